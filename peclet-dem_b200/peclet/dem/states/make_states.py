"""Saved states that the benchmark restarts from, made by the FP64 B200 step.

    python peclet-dem_b200/peclet/dem/states/make_states.py [out_dir]

plain_settling_4096_step800.npz: the 4,096-sphere settling configuration (jittered simple-cubic
lattice in a closed 16 x 16 x 64-cell box, e 0.5, mu 0.5, 10 position and 10 velocity iterations,
10 substeps of 1e-5 s per outer step) after 800 of its 1,000 outer steps from the lattice start:
positions, velocities, orientations and spins in float64, plus the packing statistics at that
point (solids fraction of the bed below its 95th-percentile height, kinetic energy, mean
coordination number at a gap of +0.002 r). Both arms of the benchmark restart from it, so the timed
window is the configuration's final 200 steps, at rest in dense contact.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(HERE))))


def settle_plain(steps, precision="fp64"):
    import peclet.dem as dem
    from peclet.dem import workloads as W
    from peclet.dem import stats as S
    sc = W.plain_settling()
    sim = sc.apply(dem.Simulation(sc.n + 8, precision))
    for _ in range(steps):
        for _ in range(sc.substeps):
            sim.step(sc.dt)
    out = dict(pos=sim.get_positions(), vel=sim.get_velocities(), quat=sim.get_quaternions(),
               angvel=sim.get_angular_velocities(), steps=np.int64(steps))
    st = S.packing_stats(out["pos"], np.full(sc.n, sc.global_scale), 1.0 / sc.inv_mass, out["vel"],
                         out["angvel"], 1.0 / sc.inv_inertia[:, 0], sc.domain[0], sc.domain[1])
    sim.close()
    return out, st


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else HERE
    from peclet.dem import workloads as W
    state, st = settle_plain(W.PLAIN_SETTLED_STEPS)
    path = os.path.join(out_dir, os.path.basename(W.plain_settling_state_path()))
    np.savez_compressed(path, **state, **{f"stat_{k}": v for k, v in st.items()})
    print(path, {k: float(v) for k, v in st.items()})


if __name__ == "__main__":
    main()
