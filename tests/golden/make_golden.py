"""Generate the golden vectors of the parity tests from the REFERENCE ITSELF.

Runs the reference's own substep (its headers compiled unmodified against the serial Kokkos shim:
oracle/_ref/libref_serial.so, built by `make -C oracle ref`) on small seeded scenes and stores, per
scene, the state after each substep and the substep's intermediate products after the first and
last substep (candidate pairs, contacts, manifolds, colours, warm-start ledger). The reference
computes in float; everything is stored as float32 / int32 (exact).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "peclet-dem_b200"), os.path.join(ROOT, "tests")]

import parity as P  # noqa: E402
import scenes as S  # noqa: E402
from peclet.dem._capi import CApi  # noqa: E402

CASES = {
    "dense_spheres": (lambda: S.dense_spheres(n=120, box=((0, 0, 0), (6e-3, 6e-3, 6e-3))), None, 6),
    "settled_column": (lambda: S.settled_column(nx=4, ny=4, nz=8), None, 12),
    "periodic_polydisperse": (lambda: S.polydisperse_periodic(n=90, L=7e-3, H=5e-3), None, 5),
    "hollow_cylinders": (lambda: S.cylinders(n=10, L=6e-3), None, 4),
    "g0_friction": (lambda: S.dense_spheres(n=120, box=((0, 0, 0), (6e-3, 6e-3, 6e-3)), gravity=(0, 0, 0)), None, 5),
}


def f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def record(sim, prefix, out):
    s = P.snapshot(sim)
    for k, v in s.items():
        if v.dtype.kind == "f":
            out[f"{prefix}{k}"] = f32(v)
        elif v.dtype == np.uint64:
            out[f"{prefix}{k}"] = v
        else:
            out[f"{prefix}{k}"] = v.astype(np.int32)


def main():
    api = CApi(os.path.join(ROOT, "oracle", "_ref", "libref_serial.so"), "ref")
    for name, (mk, extra, steps) in CASES.items():
        sc = mk()
        sim = P.build(api, sc, extra, "fp32")
        out = {"steps": np.array(steps)}
        for k in range(steps):
            sim.step(sc.dt)
            st = P.snapshot(sim, products=False)
            for key in P.STATE_KEYS:
                out[f"s{k}_{key}"] = f32(st[key])
            if k in (0, steps - 1):
                record(sim, f"p{k}_", out)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, sc.n, "particles", steps, "substeps", sim.debug_counts())


if __name__ == "__main__":
    main()
