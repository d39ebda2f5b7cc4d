"""The broadphase's own radix sort (the Morton sort of the LBVH build) against a stable sort.

Random 64-bit keys with many repeats, sorted by their low end_bit bits with int values carried
along: keys and values must equal numpy's stable argsort of the masked keys, for sizes around the
2,048-key tile (ragged last tile, one key, several tiles) and digit widths that end mid-digit."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 7, 2047, 2048, 2049, 5000, 100003])
@pytest.mark.parametrize("end_bit", [63, 64, 20, 8, 5])
def test_radix_sort_is_stable_sort(gpu_api, n, end_bit):
    rng = np.random.default_rng(n * 131 + end_bit)
    keys = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64) | (rng.integers(0, 2, size=n, dtype=np.uint64) << 63)
    keys[rng.integers(0, n, size=n // 3)] = keys[0]  # repeated keys: stability shows
    vals = np.arange(n, dtype=np.int32)[::-1].copy()
    ok_, ov = np.zeros(n, np.uint64), np.zeros(n, np.int32)
    st = gpu_api.fn["debug_radix_sort"](keys.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p), n, end_bit,
                                        ok_.ctypes.data_as(C.c_void_p), ov.ctypes.data_as(C.c_void_p))
    gpu_api.check(st, "debug_radix_sort")
    masked = keys if end_bit == 64 else keys & np.uint64((1 << end_bit) - 1)
    order = np.argsort(masked, kind="stable")
    np.testing.assert_array_equal(ok_, keys[order])
    np.testing.assert_array_equal(ov, vals[order])
