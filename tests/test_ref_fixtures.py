"""The reference's own unit-test fixtures as golden vectors, and its own unit tests on the shim.

* The reference's unit tests (tests/kokkos/*.cpp, tests/arborx/*.cpp), compiled unmodified
  against the Kokkos shim (`make -C oracle reftests`), pass: the shim provides what the reference's
  kernels expect of Kokkos and ArborX. (test_solver_velocity.cpp does not compile against the
  current headers: it calls computeVn0Kokkos with an argument list the header no longer has.)
* Broadphase fixture (tests/arborx/test_broadphase_arborx.cpp:23-101, seed 12345: 4,000 bodies,
  the last 400 ghosts, margin 0.05): its pass criterion is the brute-force pair set {i real, i < j,
  closed padded boxes overlap}. The stored set is checked here, and the B200 broadphase
  (`pdem_find_pairs_static`, the same box predicate and canonical order over caller arrays) must
  return exactly it, in (i, j) order.
* Narrowphase fixture (tests/kokkos/test_narrowphase.cpp:56-96, seed 7: a 6 x 6 x 6 jittered
  grid of spheres of two radii at global scale 0.7 with random orientations on a z = 0 plane): the
  reference's detectContactsKokkos / detectBoundaryKokkos contacts. The facade has one shape per
  simulation, so the two sphere shapes (radius 1.0 and 1.02) become radius-1 spheres with scales
  1.0 and 1.02: the same geometry through other rounding, compared (as the fixture compares its
  own device and host runs) by (bodyA, bodyB) with the fixture's tolerances, dist 1e-4 and normal
  and lever arms 5e-3 relative, in the oracle restatement here and in the B200 step on the GPU.
"""
import ctypes
import glob
import os
import subprocess

import numpy as np
import pytest

import parity as P
from peclet.dem import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


def _bp():
    return np.load(os.path.join(GOLD, "ref_broadphase_seed12345.npz"))


def _np():
    return np.load(os.path.join(GOLD, "ref_narrowphase_seed7.npz"))


# ---------------------------------------------------------------------------------------------- CPU
def test_reference_unit_tests_pass_on_shim():
    tests = sorted(glob.glob(os.path.join(ROOT, "oracle", "_ref", "reftest_*")))
    if not tests:
        pytest.skip("reference unit tests not built (make -C oracle reftests needs the reference sources)")
    for t in tests:
        r = subprocess.run([t], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0 and "PASS" in r.stdout, f"{os.path.basename(t)}: {r.stdout}{r.stderr}"


def test_broadphase_fixture_is_the_brute_force_set():
    z = _bp()
    xyzr, nr, m = z["xyzr"], int(z["n_real"]), np.float32(z["margin"])
    x, r = xyzr[:, :3], xyzr[:, 3]
    b = r + m  # float32, as the fixture computes it
    want = []
    for i in range(nr):
        d = np.abs(x[i + 1:] - x[i])
        ok = np.all(d <= (b[i] + b[i + 1:])[:, None], axis=1)
        want.extend((i, i + 1 + j) for j in np.nonzero(ok)[0])
    want = np.array(want, dtype=np.int32)
    np.testing.assert_array_equal(z["brute"], want)  # canonical (i, j) order
    np.testing.assert_array_equal(z["pairs"], want)  # the reference's broadphase returned exactly it
    assert want.shape[0] == 10227


def _fixture_scene():
    """The narrowphase fixture as a facade scene: radius-1 spheres with scales 1 / 1.02 at global
    scale 0.7, at rest without gravity (the first substep's detection sees the fixture's state)."""
    z = _np()
    st = z["state"].astype(np.float64)
    n = st.shape[0]
    gs = float(z["global_scale"])
    radii = z["shape_radii"].astype(np.float64)
    sc = W.Scene(name="ref_narrowphase_seed7", pos=st[:, :3], vel=np.zeros((n, 3)), inv_mass=np.ones(n),
                 inv_inertia=np.full((n, 3), 2.5), quat=st[:, 3:7], scales=radii[st[:, 7].astype(int)],
                 shape=(W.SPHERE, 1.0, 0.0, 0.0), global_scale=gs, domain=((-5.0, -5.0, -1.0), (12.0, 12.0, 12.0),
                                                                          (False, False, False)),
                 planes=[(0.0, 0.0, 0.0, 0.0, 0.0, 1.0)], gravity=(0.0, 0.0, 0.0), material=(0.5, 0.0, 0.0),
                 iterations=(1, 1), dt=1e-6)
    return sc, z


def _contacts_match(sim, z):
    c = sim.debug_contacts()
    ab = c[:, :2].astype(np.int64)
    geo = np.concatenate([c[:, 2:5], c[:, 5:8], c[:, 8:11], c[:, 11:12]], axis=1)
    # planes: the fixture stores bodyB = -1 and the plane point as rB
    order_got = np.lexsort((ab[:, 1], ab[:, 0]))
    zab = z["ab"].astype(np.int64)
    order_want = np.lexsort((zab[:, 1], zab[:, 0]))
    assert ab.shape[0] == zab.shape[0], f"{ab.shape[0]} contacts vs the fixture's {zab.shape[0]}"
    np.testing.assert_array_equal(ab[order_got], zab[order_want])
    g, w = geo[order_got], z["geo"].astype(np.float64)[order_want]
    close = lambda a, b, tol: np.abs(a - b) <= tol * (1.0 + np.abs(b))
    assert np.all(close(g[:, 9], w[:, 9], 1e-4)), "dist"
    assert np.all(close(g[:, :9], w[:, :9], 5e-3)), "normal / lever arms"


def test_narrowphase_fixture_oracle(orc_api):
    sc, z = _fixture_scene()
    for prec in ("fp32", "fp64"):
        sim = P.build(orc_api, sc, None, prec)
        sim.step(sc.dt)
        _contacts_match(sim, z)
        sim.close()


# ---------------------------------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_broadphase_fixture_b200(gpu_api):
    import torch
    z = _bp()
    xyzr, nr, m = z["xyzr"].astype(np.float64), int(z["n_real"]), float(z["margin"])
    d_pos = torch.as_tensor(np.ascontiguousarray(xyzr[:, :3]), device="cuda")
    d_rad = torch.as_tensor(np.ascontiguousarray(xyzr[:, 3]), device="cuda")
    cap = 64 * xyzr.shape[0]
    d_out = torch.full((cap, 2), -1, dtype=torch.int32, device="cuda")
    count = ctypes.c_long(-1)
    st = gpu_api.fn["find_pairs_static"](ctypes.c_void_p(d_pos.data_ptr()), ctypes.c_void_p(d_rad.data_ptr()),
                                         xyzr.shape[0], m, 0.0, ctypes.c_void_p(d_out.data_ptr()), cap,
                                         ctypes.byref(count), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert st == 0, gpu_api.error()
    got = d_out[: count.value].cpu().numpy()
    got = got[got[:, 0] < nr]  # the fixture's last 400 bodies issue no query
    np.testing.assert_array_equal(got, z["brute"])


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_narrowphase_fixture_b200(gpu_api, prec):
    sc, z = _fixture_scene()
    sim = P.build(gpu_api, sc, None, prec)
    sim.step(sc.dt)
    _contacts_match(sim, z)
    sim.close()
