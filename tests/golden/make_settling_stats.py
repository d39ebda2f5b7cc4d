"""Packing statistics of the 4,096-sphere settling configuration run by the REFERENCE ITSELF.

Runs the reference's own substep (its headers built unmodified against the OpenMP Kokkos shim:
oracle/_ref/libref_omp.so, `make -C oracle ref`) on the configuration from its lattice start
(jittered simple-cubic lattice, seed 1, in a closed 16 x 16 x 64-cell box, e 0.5, mu 0.5, 10
position and 10 velocity iterations, 10 substeps of 1e-5 s per outer step) and records, every 100
outer steps up to 800, the bed statistics of peclet.dem.stats.packing_stats (core solids fraction,
kinetic energy, coordination number at a contact gap of +0.002, rattlers, bed height). Gauss-Seidel
trajectories diverge, so a correct solver is checked against these statistics, not positions.

    python tests/golden/make_settling_stats.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "peclet-dem_b200")]

from peclet.dem import stats as S  # noqa: E402
from peclet.dem import workloads as W  # noqa: E402
from peclet.dem._capi import CApi, CApiSimulation  # noqa: E402

STEPS = (100, 200, 400, 600, 800)


def main():
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    api = CApi(os.path.join(ROOT, "oracle", "_ref", "libref_omp.so"), "ref")
    sc = W.plain_settling()
    sim = sc.apply(CApiSimulation(api, sc.n + 8, "fp32"))
    out = {"what": "reference OpenMP shim build, float; plain settling 4096 spheres from the lattice start",
           "stats": {}}
    t0 = time.time()
    for step in range(1, max(STEPS) + 1):
        for _ in range(sc.substeps):
            sim.step(sc.dt)
        if step in STEPS:
            st = S.packing_stats(sim.get_positions(), np.full(sc.n, sc.global_scale), 1.0 / sc.inv_mass,
                                 sim.get_velocities(), sim.get_angular_velocities(), 1.0 / sc.inv_inertia[:, 0],
                                 sc.domain[0], sc.domain[1])
            out["stats"][str(step)] = st
            print(step, round(time.time() - t0, 1), st, flush=True)
    with open(os.path.join(HERE, "settling_stats_ref.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
