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
