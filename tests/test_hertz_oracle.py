"""The CPU restatement of the Hertz sphere substep (oracle/hertz_spheres.py), pinned two ways:
its forward against the C++ oracle's Hertz engine (`step_hertz`, itself pinned to the reference's
engine), and its forward-mode dual numbers against converged central finite differences."""
import os
import sys

import numpy as np
import pytest

import hertz_cases as HC
from peclet.dem import workloads as W
from peclet.dem._capi import CApiSimulation

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import hertz_spheres as H  # noqa: E402


def _model(c):
    return H.Model(c["r"], c["m"], c["I"], c["first"], c["planes"], HC.NU, HC.DT, c["g"])


def _floor_grid(h=0.5e-3):
    """The plane z = 0 (normal +z) as an SDF grid over |x|, |y| <= 5 mm, -2 mm <= z <= 5 mm."""
    nx = ny = 21
    nz = 15
    origin = np.array([-5e-3, -5e-3, -2e-3])
    z = origin[2] + h * np.arange(nz)
    grid = np.broadcast_to(z[:, None, None], (nz, ny, nx))  # x-fastest after ravel of (z, y, x)
    return np.ascontiguousarray(grid).ravel(), nx, ny, nz, origin, (h, h, h)


def _engine(api, c, theta):
    """The same scene on the Hertz engine of the C++ oracle (a floor plane as an SDF wall: the
    engine takes no analytic planes)."""
    n = len(c["r"])
    sc = W.Scene(name="hz", pos=c["x0"], vel=c["v0"], inv_mass=1.0 / c["m"], inv_inertia=np.repeat((1.0 / c["I"])[:, None], 3, 1),
                 global_scale=float(c["r"][0]), domain=((-0.02, -0.02, -0.02), (0.03, 0.03, 0.03), (False,) * 3),
                 gravity=c["g"], material=(theta[1], 0.0, theta[2]), dt=HC.DT, hertz=(theta[0], HC.NU))
    sim = sc.apply(CApiSimulation(api, n + 8, "fp64"))
    sim.set_angular_velocities(c["w0"])
    if c["planes"]:
        assert c["planes"] == [[0, 0, 0, 0, 0, 1]]
        sim.add_sdf_wall(*_floor_grid(), theta[1], theta[2])
    return sim


@pytest.mark.parametrize("case,steps", [("pair", 60), ("gas", 100)])
def test_forward_matches_hertz_engine(orc_api, case, steps):
    c = getattr(HC, case)(scenes=1, gap=0.05e-3) if case == "gas" else getattr(HC, case)()
    if case == "gas":
        c["planes"] = []  # sphere pairs only (one scene: the engine has no scenes)
    sim = _engine(orc_api, c, HC.THETA)
    x, v, w = _model(c).rollout(c["x0"], c["v0"], c["w0"], *HC.THETA, steps)
    sim.step_hertz(HC.DT, steps, 0.5)
    if case == "gas":
        assert len(sim.debug_hertz()[0]) > 0, "no sphere pair touched"
    np.testing.assert_allclose(sim.get_positions(), x, rtol=0, atol=1e-15)
    np.testing.assert_allclose(sim.get_velocities(), v, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(sim.get_angular_velocities(), w, rtol=1e-10, atol=1e-9)


def test_forward_plane_matches_hertz_engine(orc_api):
    """A sphere bouncing on a floor plane: the engine's plane is a sampled SDF with a finite-
    difference normal, so agreement is to the grid's rounding, not bit-exact."""
    c = HC.floor()
    sim = _engine(orc_api, c, HC.THETA)
    x, v, w = _model(c).rollout(c["x0"], c["v0"], c["w0"], *HC.THETA, 50)
    sim.step_hertz(HC.DT, 50, 0.5)
    np.testing.assert_allclose(sim.get_positions(), x, rtol=0, atol=1e-12)
    np.testing.assert_allclose(sim.get_velocities(), v, rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(sim.get_angular_velocities(), w, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("case,steps", [("pair", 100), ("floor", 100), ("gas", 60)])
def test_dual_matches_finite_differences(case, steps):
    c = getattr(HC, case)()
    M = _model(c)
    n = len(c["r"])
    rng = np.random.default_rng(11)
    cx = rng.standard_normal((n, 3))
    dv, dx, dw = (rng.standard_normal((n, 3)) for _ in range(3))
    tans = [{"theta": np.eye(3)[k]} for k in range(3)] + [{"v": dv}, {"x": dx}, {"w": dw}]
    xd, _, _ = H.jvp(M, c["x0"], c["v0"], c["w0"], HC.THETA, tans, steps)
    jv = (xd.d * cx[..., None]).sum((0, 1))

    def loss(th=HC.THETA, x0=c["x0"], v0=c["v0"], w0=c["w0"]):
        return float((M.rollout(x0, v0, w0, *th, steps)[0] * cx).sum())

    fd = []
    for k in range(3):
        h = 1e-6 * HC.THETA[k]
        tp, tm = HC.THETA.copy(), HC.THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd.append((loss(th=tp) - loss(th=tm)) / (2 * h))
    fd.append((loss(v0=c["v0"] + 1e-7 * dv) - loss(v0=c["v0"] - 1e-7 * dv)) / 2e-7)
    fd.append((loss(x0=c["x0"] + 1e-11 * dx) - loss(x0=c["x0"] - 1e-11 * dx)) / 2e-11)
    fd.append((loss(w0=c["w0"] + 1e-5 * dw) - loss(w0=c["w0"] - 1e-5 * dw)) / 2e-5)
    for k, (a, b) in enumerate(zip(jv, fd)):
        assert abs(a - b) <= 1e-4 * abs(b) + 1e-14, f"{case}: tangent {k}: dual {a} vs FD {b}"
