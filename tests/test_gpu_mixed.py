"""The FP32-mixed precision form: the step computes in float, the positions and orientations are
kept in FP64 (each substep's float increment is added to the FP64 master). In contact-rich scenes
the float and double steps part ways within a few substeps (the adaptive stops and contact margins
are discrete decisions), so the error against FP64 is measured and reported by the benchmark; here
the mechanics are checked: the mixed run follows the float step and returns the FP64 master."""
import numpy as np
import pytest

import parity as P
import scenes as S

pytestmark = pytest.mark.gpu


def test_mixed_follows_fp32_step(gpu_api):
    """The mixed form runs the float step; only the stored state differs (FP64 master), so over a
    few substeps it stays within float rounding of the pure FP32 run."""
    sc = S.settled_column()
    a = P.build(gpu_api, sc, None, "mixed")
    b = P.build(gpu_api, sc, None, "fp32")
    for _ in range(3):
        a.step(sc.dt)
        b.step(sc.dt)
    err = np.max(np.abs(a.get_positions() - b.get_positions().astype(np.float64))) / sc.global_scale
    assert err < 1e-4, f"mixed vs fp32: {err:.3e} r"


def test_mixed_master_is_fp64(gpu_api):
    """Positions set in FP64 come back unrounded before any step (the master holds them)."""
    sc = S.dense_spheres()
    sim = P.build(gpu_api, sc, None, "mixed")
    x = sim.get_positions()
    np.testing.assert_array_equal(x, sc.pos)
