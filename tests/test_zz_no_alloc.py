"""The allocation-free candidate-pair entry point (`pdem_find_pairs_static`) against the
simulation's own broadphase.

`compute_overlaps` runs the simulation's broadphase on the current positions (margin 0.1 x the
largest radius, boxes capped at the largest domain extent); `debug_pairs` then returns its
canonical pair list. The same positions and radii, copied to caller-owned device arrays, go through
`pdem_find_pairs_static`, whose scratch lives in a fixed device buffer. The lists must be identical
(integer data: exact), on two different scenes called back to back, so nothing carries over from
the first call into the second. Sizes above the fixed limit must be refused before any launch.
"""
import ctypes

import numpy as np
import pytest

import scenes as S

pytestmark = pytest.mark.gpu

MAX_BODIES = 16384


def _reference_pairs(api, scene):
    from peclet.dem._capi import CApiSimulation
    sim = scene.apply(CApiSimulation(api, scene.n + 8, "fp64"))
    sim.compute_overlaps()
    pairs = sim.debug_pairs().reshape(-1, 2)
    sim.close()
    scales = scene.scales if scene.scales is not None else np.ones(scene.n)
    radius = (np.asarray(scales, np.float64) * scene.global_scale) * scene.shape[1]
    max_rad = (np.max(scales) * scene.global_scale) * scene.shape[1]
    margin = 0.1 * max_rad
    mn, mx, _ = scene.domain
    box_cap = float(np.max(np.asarray(mx, np.float64) - np.asarray(mn, np.float64)))
    return pairs, radius, margin, box_cap


def _static_pairs(api, pos, radius, margin, box_cap, cap):
    import torch
    d_pos = torch.as_tensor(np.ascontiguousarray(pos, np.float64), device="cuda")
    d_rad = torch.as_tensor(np.ascontiguousarray(radius, np.float64), device="cuda")
    d_out = torch.full((max(cap, 1), 2), -1, dtype=torch.int32, device="cuda")
    count = ctypes.c_long(-1)
    stream = torch.cuda.current_stream().cuda_stream
    st = api.fn["find_pairs_static"](ctypes.c_void_p(d_pos.data_ptr()), ctypes.c_void_p(d_rad.data_ptr()),
                                     int(pos.shape[0]), float(margin), float(box_cap),
                                     ctypes.c_void_p(d_out.data_ptr()), int(cap), ctypes.byref(count),
                                     ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return st, count.value, d_out[: max(0, min(count.value, cap))].cpu().numpy()


def test_static_pairs_match_simulation_broadphase(gpu_api):
    scene_a = S.dense_spheres(seed=101, n=600)
    scene_b = S.dense_spheres(seed=202, n=1500, box=((0, 0, 0), (12e-3, 12e-3, 12e-3)))
    for scene in (scene_a, scene_b):  # two calls in a row, different sizes
        want, radius, margin, box_cap = _reference_pairs(gpu_api, scene)
        assert want.shape[0] > 0
        st, n, got = _static_pairs(gpu_api, scene.pos, radius, margin, box_cap, cap=4 * want.shape[0] + 16)
        assert st == 0, gpu_api.error()
        assert n == want.shape[0]
        np.testing.assert_array_equal(got, want)


def test_static_pairs_polydisperse_and_repeat(gpu_api):
    scene = S.dense_spheres(seed=303, n=800)
    rng = np.random.default_rng(5)
    scene.scales = np.clip(rng.lognormal(0.0, 0.25, scene.n), 0.5, 2.0)
    want, radius, margin, box_cap = _reference_pairs(gpu_api, scene)
    first = _static_pairs(gpu_api, scene.pos, radius, margin, box_cap, cap=4 * want.shape[0] + 16)
    second = _static_pairs(gpu_api, scene.pos, radius, margin, box_cap, cap=4 * want.shape[0] + 16)
    for st, n, got in (first, second):
        assert st == 0, gpu_api.error()
        assert n == want.shape[0]
        np.testing.assert_array_equal(got, want)


def test_static_pairs_capacity_and_limits(gpu_api):
    scene = S.dense_spheres(seed=404, n=400)
    want, radius, margin, box_cap = _reference_pairs(gpu_api, scene)
    # too small an output buffer: the count is returned and nothing is written
    st, n, _ = _static_pairs(gpu_api, scene.pos, radius, margin, box_cap, cap=0)
    assert st == 0 and n == want.shape[0]
    # above the fixed scratch size: refused with a clear message, nothing launched
    big = MAX_BODIES + 1
    count = ctypes.c_long(-1)
    st = gpu_api.fn["find_pairs_static"](ctypes.c_void_p(1), ctypes.c_void_p(1), big, 0.0, 0.0,
                                         ctypes.c_void_p(1), 0, ctypes.byref(count), None)
    assert st == 2
    assert str(MAX_BODIES) in gpu_api.error()


def _brute_pairs(pos, radius, margin, box_cap):
    """The closed-box predicate of the broadphase over all i < j, with the parking rule: a body
    whose padded half-width b = r + margin or position is not finite, or whose b exceeds box_cap,
    sits at (-1e30)^3 with b = 0 (parked bodies meet only each other)."""
    x = np.array(pos, np.float64)
    b = np.asarray(radius, np.float64) + margin
    park = ~np.isfinite(b) | np.any(np.isnan(x), axis=1) | ((box_cap > 0) & (b > box_cap))
    x[park] = -1.0e30
    b = np.where(park, 0.0, b)
    lo, hi = x - b[:, None], x + b[:, None]
    out = []
    for i in range(x.shape[0] - 1):
        ok = np.all((lo[i] <= hi[i + 1:]) & (lo[i + 1:] <= hi[i]), axis=1)
        out.extend((i, i + 1 + j) for j in np.nonzero(ok)[0])
    return np.array(out, dtype=np.int32).reshape(-1, 2)


def test_static_pairs_at_the_limit_parked_bodies_and_no_allocation(gpu_api):
    """16,384 bodies (the fixed limit) with non-finite and oversized radii and a non-finite position
    among them, then 9,000 bodies, called back to back: each list equals the brute-force predicate
    with the parking rule. After a first call, further calls leave this library's allocation count
    and the device's free memory unchanged."""
    import torch
    rng = np.random.default_rng(77)
    cases = []
    for n, L in ((MAX_BODIES, 60e-3), (9000, 50e-3)):
        pos = rng.uniform(0.0, L, (n, 3))
        radius = rng.uniform(0.5e-3, 1.5e-3, n)
        radius[rng.choice(n, 5, replace=False)] = np.nan
        radius[rng.choice(n, 3, replace=False)] = np.inf
        radius[rng.choice(n, 4, replace=False)] = 0.5  # far above box_cap
        pos[rng.choice(n, 2, replace=False), 1] = np.nan
        cases.append((pos, radius, 0.15e-3, 0.05))
    want = [_brute_pairs(*c) for c in cases]
    # every device array the calls use is made before the allocation baseline
    dev = [(torch.as_tensor(p, device="cuda"), torch.as_tensor(r, device="cuda"),
            torch.full((4 * w.shape[0] + 16, 2), -1, dtype=torch.int32, device="cuda")) for (p, r, _, _), w in zip(cases, want)]
    stream = torch.cuda.current_stream().cuda_stream

    def call(k):
        (p, r, m, cap), (dp, dr, do) = cases[k], dev[k]
        count = ctypes.c_long(-1)
        st = gpu_api.fn["find_pairs_static"](ctypes.c_void_p(dp.data_ptr()), ctypes.c_void_p(dr.data_ptr()), p.shape[0],
                                             m, cap, ctypes.c_void_p(do.data_ptr()), do.shape[0], ctypes.byref(count),
                                             ctypes.c_void_p(stream))
        torch.cuda.synchronize()
        assert st == 0, gpu_api.error()
        return count.value, do[: count.value].cpu().numpy()

    call(1)  # set-up call
    torch.cuda.synchronize()
    allocs0, free0 = gpu_api.fn["debug_allocs"](), torch.cuda.mem_get_info()[0]
    for k in (0, 1, 0):
        n, got = call(k)
        assert n == want[k].shape[0]
        np.testing.assert_array_equal(got, want[k])
    assert gpu_api.fn["debug_allocs"]() == allocs0
    assert torch.cuda.mem_get_info()[0] == free0
