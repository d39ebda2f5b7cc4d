"""The oracle on dual numbers (the forward-mode check of the XPBD adjoint), pinned on the CPU:
its value run is the FP64 oracle's bit for bit, and its tangents are the FP64 oracle's central
finite differences over a window whose branches (contact and manifold sets, the active normal
impulses, the active position contacts) are the same at +h and -h."""
import numpy as np
import pytest

import dual_oracle as DO
import parity as P
import scenes as S

T = 10


def _scene():
    sc = S.settled_column(seed=21, nx=3, ny=3, nz=4)
    sc.material = (0.5, 0.3, 0.5)
    return sc


def _loss_weights(n, seed=5):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=(n, 3)), rng.normal(size=(n, 4))


def _loss(sim, W):
    a, b, c, d = W
    return (np.sum(a * sim.get_positions()) + np.sum(b * sim.get_velocities())
            + np.sum(c * sim.get_angular_velocities()) + np.sum(d * sim.get_quaternions()))


def _pattern(sim):
    # the sets, and the impulses that are active by more than rounding (an impulse at the level of
    # rounding noise may flip with h, and moves the result by as little)
    lam, pl = sim.debug_lambda()[:, 0], np.abs(sim.debug_pos_lambda())
    return (sim.num_contacts(), sim.num_manifolds(), tuple(np.flatnonzero(lam > 1e-9 * max(lam.max(initial=0), 1e-300))),
            tuple(np.flatnonzero(pl > 1e-9 * max(pl.max(initial=0), 1e-300))))


def _run(orc_api, sc, material=None, vel=None):
    sim = P.build(orc_api, sc, None, "fp64")
    if material is not None:
        sim.set_material_params(*material)
    if vel is not None:
        sim.set_velocities(vel)
    pats = []
    for _ in range(T):
        sim.step(sc.dt)
        pats.append(_pattern(sim))
    return sim, pats


def test_dual_value_run_is_the_fp64_oracle(orc_api):
    sc = _scene()
    a = P.build(orc_api, sc, None, "fp64")
    d = sc.apply(DO.dual_sim(orc_api, sc.n + 8))
    for _ in range(T):
        a.step(sc.dt)
        d.step(sc.dt)
    for get in ("get_positions", "get_velocities", "get_quaternions", "get_angular_velocities"):
        np.testing.assert_array_equal(getattr(d, get)(), getattr(a, get)())


def test_dual_tangents_are_the_central_differences(orc_api):
    sc = _scene()
    W = _loss_weights(sc.n)
    rng = np.random.default_rng(9)
    dv = rng.normal(size=(sc.n, 3))
    d = sc.apply(DO.dual_sim(orc_api, sc.n + 8))
    for lane in range(3):  # eN, eT, mu
        DO.seed(d, DO.MATERIAL, lane, np.eye(3)[lane])
    DO.seed(d, DO.VEL, 3, dv)
    for _ in range(T):
        d.step(sc.dt)
    got = []
    for lane in range(4):
        a, b, c, q = W
        got.append(np.sum(a * DO.tangent(d, DO.POS, lane, sc.n)) + np.sum(b * DO.tangent(d, DO.VEL, lane, sc.n))
                   + np.sum(c * DO.tangent(d, DO.ANGVEL, lane, sc.n)) + np.sum(q * DO.tangent(d, DO.QUAT, lane, sc.n)))
    e0 = np.array(sc.material, np.float64)
    for lane in range(4):
        h = 1e-5 if lane < 3 else 1e-5 * 0.05  # below this the rounding of the loss dominates
        plus = minus = None
        if lane < 3:
            up, dn = e0.copy(), e0.copy()
            up[lane] += h
            dn[lane] -= h
            sp, pp = _run(orc_api, sc, material=up)
            sm, pm = _run(orc_api, sc, material=dn)
        else:
            sp, pp = _run(orc_api, sc, vel=sc.vel + h * dv)
            sm, pm = _run(orc_api, sc, vel=sc.vel - h * dv)
        assert pp == pm, f"lane {lane}: the branches differ at +h and -h"
        fd = (_loss(sp, W) - _loss(sm, W)) / (2 * h)
        assert abs(got[lane] - fd) <= 1e-5 * max(abs(fd), 1e-3), (lane, got[lane], fd)
