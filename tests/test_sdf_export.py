"""The packed-bed SDF export (get_sdf_grid / export_sdf, src/output_sdf.hpp, src/io.hpp:86-110):
the oracle restatement against the reference's own build (CPU, float: bit-exact), and the B200
library against both (GPU)."""
import os

import numpy as np
import pytest

import parity as P
import scenes as S

SCENES = [
    ("dense_spheres", lambda: S.dense_spheres(), (24, 24, 24), 3),
    ("periodic_polydisperse", lambda: S.polydisperse_periodic(), (20, 20, 16), 2),
    ("hollow_cylinders", lambda: S.cylinders(), (20, 20, 20), 2),
    ("grid_sdf_capsules", lambda: S.sdf_capsules(), (16, 18, 20), 2),
]


def _unit_scale(sc):
    """The reference splats with the particle scale alone (no global scale): give the shapes their
    size in metres through the scales so the field is a packed bed, not a box of overlaps."""
    sc.scales = (sc.scales if sc.scales is not None else np.ones(sc.n)) * sc.global_scale
    return sc


@pytest.mark.parametrize("name,mk,res,steps", SCENES, ids=[s[0] for s in SCENES])
def test_oracle_sdf_bitexact_vs_reference(ref_api, orc_api, name, mk, res, steps):
    sc = _unit_scale(mk())
    a = P.build(ref_api, sc, None, "fp32")
    b = P.build(orc_api, sc, None, "fp32")
    for _ in range(steps):
        a.step(sc.dt)
        b.step(sc.dt)
    ga, gb = a.get_sdf_grid(res), b.get_sdf_grid(res)
    assert ga.shape == res and np.isfinite(ga).all()
    assert (ga < 0).any() and (ga > 0).any(), "no solid or no void in the field"
    np.testing.assert_array_equal(ga, gb)


@pytest.mark.gpu
@pytest.mark.parametrize("name,mk,res,steps", SCENES, ids=[s[0] for s in SCENES])
def test_gpu_sdf_vs_oracle(gpu_api, orc_api, name, mk, res, steps):
    for precision, rtol in (("fp32", 0.0), ("fp64", 1e-12)):
        sc = _unit_scale(mk())
        a = P.build(gpu_api, sc, None, precision)
        b = P.build(orc_api, sc, None, precision)
        for _ in range(steps):
            a.step(sc.dt)
            b.step(sc.dt)
        ga, gb = a.get_sdf_grid(res), b.get_sdf_grid(res)
        np.testing.assert_allclose(ga, gb, rtol=rtol, atol=0, err_msg=f"{name} {precision}")


@pytest.mark.gpu
def test_gpu_export_sdf_matches_reference_file(gpu_api, ref_api, tmp_path):
    sc = _unit_scale(S.dense_spheres())
    a = P.build(gpu_api, sc, None, "fp32")
    b = P.build(ref_api, sc, None, "fp32")
    a.step(sc.dt)
    b.step(sc.dt)
    fa, fb = os.path.join(tmp_path, "a.vti"), os.path.join(tmp_path, "b.vti")
    a.export_sdf(fa, (12, 10, 14))
    b.export_sdf(fb, (12, 10, 14))
    assert open(fa).read() == open(fb).read()


def test_sdf_rejects_bad_resolution(orc_api):
    sc = S.dense_spheres()
    a = P.build(orc_api, sc, None, "fp32")
    with pytest.raises(ValueError):
        a.get_sdf_grid((0, 4, 4))
