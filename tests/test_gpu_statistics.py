"""Long-run statistical parity: the B200 step settles the 4,096-sphere configuration to the same bed
as the reference.

Gauss-Seidel trajectories part ways chaotically within a few hundred substeps (the float and
double steps already differ by 1e-2 radii after 25), so a long run is judged by the statistics of
the bed it builds, as the reference judges its packings (docs/packing_investigation.md:139-146):
solids fraction of the bed core, kinetic energy, mean coordination number at a contact gap of
+0.002 and the bed height (peclet.dem.stats.packing_stats). The reference's own code settled the
same configuration from the same lattice start (tests/golden/make_settling_stats.py, its OpenMP
shim build, float); the B200 step runs it in FP64 and FP32 through the C ABI. Stated tolerances:

* after 400 outer steps (the bed still compacting): solids fraction within 0.03, coordination
  within 0.6, bed height within 1.5 mm;
* after 800 outer steps (at rest): solids fraction within 0.01, coordination within 0.3, bed
  height within 0.5 mm, kinetic energy below 2e-2 of the initial and within a factor 10 of the
  reference's, and the same rattler count to within 5.

The saved restart state of the benchmark (after 800 steps, FP64) is checked against the same bar.
"""
import json
import os

import numpy as np
import pytest

import parity as P
from peclet.dem import stats as S
from peclet.dem import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "tests", "golden", "settling_stats_ref.json")
TOL = {400: dict(phi=0.03, z=0.6, bed_height=1.5e-3), 800: dict(phi=0.01, z=0.3, bed_height=0.5e-3)}


def _ref():
    with open(REF) as f:
        return {int(k): v for k, v in json.load(f)["stats"].items()}


def _stats(sim, sc):
    return S.packing_stats(sim.get_positions(), np.full(sc.n, sc.global_scale), 1.0 / sc.inv_mass,
                           sim.get_velocities(), sim.get_angular_velocities(), 1.0 / sc.inv_inertia[:, 0],
                           sc.domain[0], sc.domain[1])


def _check(got, ref, step, ke0):
    for k, tol in TOL[step].items():
        assert abs(got[k] - ref[k]) <= tol, f"step {step}: {k} {got[k]} vs the reference's {ref[k]}"
    if step == 800:
        assert got["ke"] < 2e-2 * ke0 and ref["ke"] < 2e-2 * ke0
        assert 0.1 <= got["ke"] / ref["ke"] <= 10.0, f"kinetic energy {got['ke']} vs {ref['ke']}"
        assert abs(got["rattlers"] - ref["rattlers"]) <= 5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_settled_bed_statistics_match_reference(gpu_api, precision):
    ref = _ref()
    sc = W.plain_settling()
    ke0 = 0.5 * ((1.0 / sc.inv_mass) * (sc.vel ** 2).sum(1)).sum()
    sim = P.build(gpu_api, sc, None, precision)
    for step in range(1, 801):
        for _ in range(sc.substeps):
            sim.step(sc.dt)
        if step in TOL:
            _check(_stats(sim, sc), ref[step], step, ke0)
    assert sim.counters()["status"] == 0
    sim.close()


def test_saved_restart_state_matches_reference_statistics():
    ref = _ref()[800]
    sc = W.plain_settled()
    ke0 = 0.5 * ((1.0 / sc.inv_mass) * (W.plain_settling().vel ** 2).sum(1)).sum()
    got = S.packing_stats(sc.pos, np.full(sc.n, sc.global_scale), 1.0 / sc.inv_mass, sc.vel, sc.angvel,
                          1.0 / sc.inv_inertia[:, 0], sc.domain[0], sc.domain[1])
    _check(got, ref, 800, ke0)
