"""Golden vectors from two of the reference's own unit-test fixtures, run through its own kernels.

The fixtures of tests/arborx/test_broadphase_arborx.cpp:23-101 (seed 12345) and
tests/kokkos/test_narrowphase.cpp:56-96 (seed 7) are regenerated with their seeds and
distributions by oracle/fixtures.cpp, which runs the reference's unmodified
findCollisionsArborX, detectContactsKokkos and detectBoundaryKokkos (headers compiled against the
serial Kokkos shim: `make -C oracle fixtures`) and writes inputs and outputs; this script stores
them as

    ref_broadphase_seed12345.npz: xyzr (n, 4) float32, n_real, margin, brute (P, 2) the fixture's
        brute-force pair set (its pass criterion), pairs (P, 2) the broadphase's output
    ref_narrowphase_seed7.npz: state (n, 8) float32 (x y z qx qy qz qw shape id), global_scale,
        margin, radii of shapes 0 and 1, ab (C, 2) int32, geo (C, 10) float32 (n rA rB dist)

    python tests/golden/make_fixtures.py
"""
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "fixtures"], check=True)
    with tempfile.TemporaryDirectory() as d:
        subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_fixtures"), d], check=True)
        rd = lambda name, dt: np.fromfile(os.path.join(d, name), dtype=dt)
        meta = rd("bp_meta.f32", np.float32)
        np.savez_compressed(os.path.join(HERE, "ref_broadphase_seed12345.npz"),
                            xyzr=rd("bp_xyzr.f32", np.float32).reshape(-1, 4), n_real=np.int32(meta[1]),
                            margin=np.float32(meta[2]), brute=rd("bp_brute.i32", np.int32).reshape(-1, 2),
                            pairs=rd("bp_pairs.i32", np.int32).reshape(-1, 2))
        meta = rd("np_meta.f32", np.float32)
        np.savez_compressed(os.path.join(HERE, "ref_narrowphase_seed7.npz"),
                            state=rd("np_state.f32", np.float32).reshape(-1, 8), global_scale=np.float32(meta[1]),
                            margin=np.float32(meta[2]), shape_radii=meta[3:5].copy(),
                            ab=rd("np_ab.i32", np.int32).reshape(-1, 2), geo=rd("np_geo.f32", np.float32).reshape(-1, 10))


if __name__ == "__main__":
    main()
