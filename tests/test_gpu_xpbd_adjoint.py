"""The adjoint of the XPBD substep on the GPU against the oracle on dual numbers.

The GPU forward is the production FP64 step (recorded); the backward replays and reverses it. The
oracle on dual numbers (tests/dual_oracle.py, pinned against central differences on the CPU) runs
the same scene with tangents seeded on (eN, eT, mu) and on a direction of the start state; its
output tangents contracted with the loss weights are the directional derivatives that the
adjoint's gradients must reproduce. Both are exact derivatives of the same piecewise-smooth map
along the branch the forward took, so they agree to rounding: 1e-7 relative here."""
import numpy as np
import pytest
import torch

import dual_oracle as DO
import parity as P
import scenes as S

pytestmark = pytest.mark.gpu

RTOL = 1e-7


def _column():
    sc = S.settled_column(seed=21, nx=3, ny=3, nz=4)
    sc.material = (0.5, 0.3, 0.5)
    return sc


def _impacts():
    """Spheres thrown at each other and the walls: restitution and friction branches active."""
    sc = S.dense_spheres(seed=31, n=48, box=((0, 0, 0), (10e-3, 10e-3, 10e-3)), vmax=0.4, e=0.7, mu=0.4)
    sc.material = (0.7, 0.2, 0.4)
    return sc


def _settled():
    """The benchmark's bed: 4,096 spheres of the plain settling configuration at its saved restart."""
    from peclet.dem import workloads as W
    return W.plain_settled()


def _weights(n, seed=5):
    rng = np.random.default_rng(seed)
    return [rng.normal(size=(n, c)) for c in (3, 4, 3, 3)]  # x, q, v, w


def _start(sc):
    q = sc.quat if sc.quat is not None else np.tile([0.0, 0.0, 0.0, 1.0], (sc.n, 1))
    w = sc.angvel if sc.angvel is not None else np.zeros((sc.n, 3))
    return [np.asarray(a, np.float64) for a in (sc.pos, q, sc.vel, w)]


def _gpu(gpu_api, sc, T, extra=None):
    from peclet.dem.xpbd_adjoint import XpbdRollout
    sim = P.build(gpu_api, sc, extra, "fp64")
    roll = XpbdRollout(sim)
    dev = torch.device("cuda")
    start = [torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True) for a in _start(sc)]
    theta = torch.tensor(sc.material, dtype=torch.float64, requires_grad=True)
    out = roll(*start, theta, T)
    W = _weights(sc.n)
    L = sum((torch.tensor(w, dtype=torch.float64, device=dev) * o).sum() for w, o in zip(W, out))
    L.backward()
    grads = [t.grad.cpu().numpy() for t in start]
    return [o.detach().cpu().numpy() for o in out], grads, theta.grad.numpy(), roll.info(), roll


def _dual(orc_api, sc, T, direction, extra=None):
    d = sc.apply(DO.dual_sim(orc_api, sc.n + 8))
    if extra:
        extra(d)
    for lane in range(3):
        DO.seed(d, DO.MATERIAL, lane, np.eye(3)[lane])
    dx, dq, dv, dw = direction
    DO.seed(d, DO.POS, 3, dx)
    DO.seed(d, DO.QUAT, 3, dq)
    DO.seed(d, DO.VEL, 3, dv)
    DO.seed(d, DO.ANGVEL, 3, dw)
    for _ in range(T):
        d.step(sc.dt)
    W = _weights(sc.n)
    which = (DO.POS, DO.QUAT, DO.VEL, DO.ANGVEL)
    tans = [sum(np.sum(w * DO.tangent(d, k, lane, sc.n)) for w, k in zip(W, which)) for lane in range(4)]
    end = [d.get_positions(), d.get_quaternions(), d.get_velocities(), d.get_angular_velocities()]
    return np.array(tans), end


@pytest.mark.parametrize("name,mk,T", [("column", _column, 10), ("column", _column, 40), ("impacts", _impacts, 20),
                                       ("settled", _settled, 10)],
                         ids=["column-10", "column-40", "impacts-20", "settled4096-10"])
def test_adjoint_matches_dual_numbers(gpu_api, orc_api, name, mk, T):
    sc = mk()
    rng = np.random.default_rng(17)
    direction = [rng.normal(size=(sc.n, c)) * s for c, s in ((3, 1e-3), (4, 1e-2), (3, 0.1), (3, 10.0))]
    end, grads, dtheta, info, _ = _gpu(gpu_api, sc, T)
    tans, end_o = _dual(orc_api, sc, T, direction)
    # the forward is the production step: within 1e-12 of the oracle (relative to the scale)
    assert np.max(np.abs(end[0] - end_o[0])) <= 1e-12 * 10 * sc.global_scale
    # the replay reproduces the recorded forward
    assert info["substeps"] == T and info["replay_dx"] <= 1e-9, info
    for k in range(3):
        assert abs(dtheta[k] - tans[k]) <= RTOL * max(abs(tans[k]), 1e-6 * np.abs(tans).max()), (k, dtheta, tans)
    dirderiv = sum(np.sum(g * d) for g, d in zip(grads, direction))
    assert abs(dirderiv - tans[3]) <= RTOL * max(abs(tans[3]), 1e-6), (dirderiv, tans[3])


def test_rollout_refuses_what_it_does_not_reverse(gpu_api):
    from peclet.dem.xpbd_adjoint import XpbdRollout
    sc = S.polydisperse_periodic()
    sim = P.build(gpu_api, sc, None, "fp64")
    roll = XpbdRollout(sim)
    start = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in _start(sc)]
    with pytest.raises(ValueError):
        roll(*start, torch.tensor(sc.material, dtype=torch.float64), 2)
    with pytest.raises(ValueError):
        XpbdRollout(P.build(gpu_api, _column(), None, "fp32"))


def test_hand_reverse_equals_dual_jacobians(gpu_api, monkeypatch):
    """The hand-written reverse of the PGS update against the same update reversed through its
    forward-mode local Jacobian (PDEM_XADJ_DUAL=1): the same gradients to rounding."""
    sc = _impacts()
    _, g0, t0, _, _ = _gpu(gpu_api, sc, 20)
    monkeypatch.setenv("PDEM_XADJ_DUAL", "1")
    _, g1, t1, _, _ = _gpu(gpu_api, sc, 20)
    np.testing.assert_allclose(t0, t1, rtol=1e-10)
    for a, b in zip(g0, g1):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-12 * np.abs(b).max())


def test_branch_signature_certifies_differences(gpu_api):
    """The record's branch hash is a function of the rollout's branches: the same rollout twice gives
    the same hash; a large change of friction changes it (the cone clamps move)."""
    from peclet.dem.xpbd_adjoint import XpbdRollout
    sc = _impacts()
    sim = P.build(gpu_api, sc, None, "fp64")
    roll = XpbdRollout(sim)
    start = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in _start(sc)]
    hashes = []
    for mu in (0.4, 0.4, 0.05):
        roll(*start, torch.tensor([0.7, 0.2, mu], dtype=torch.float64), 10)
        hashes.append((roll.signature(), roll.branches()))
    assert np.array_equal(hashes[0][0], hashes[1][0]) and hashes[0][1] == hashes[1][1]
    assert hashes[0][1] != hashes[2][1]


def test_backward_uses_the_rollouts_material(gpu_api):
    """The backward differentiates the rollout that ran: a material set on the simulation after the
    forward (before the backward) changes nothing in the gradients (beyond the rounding of the
    reverse's atomic sums, which vary from run to run)."""
    from peclet.dem.xpbd_adjoint import XpbdRollout
    sc = _impacts()
    out = []
    for later in (None, (0.1, 0.0, 0.9)):
        sim = P.build(gpu_api, sc, None, "fp64")
        roll = XpbdRollout(sim)
        start = [torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=True) for a in _start(sc)]
        theta = torch.tensor(sc.material, dtype=torch.float64, requires_grad=True)
        x, q, v, w = roll(*start, theta, 10)
        if later:
            sim.set_material_params(*later)
        (x.sum() + v.sum()).backward()
        out.append((theta.grad.numpy().copy(), start[2].grad.cpu().numpy()))
    np.testing.assert_allclose(out[0][0], out[1][0], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-12, atol=1e-12 * np.abs(out[0][1]).max())


def test_adjoint_with_escalate_stabilization(gpu_api, orc_api):
    """The escalate stabilization mode (up to 256 PGS sweeps at the stabilization threshold, no
    side flags) reversed like the one-sided pass: against the dual numbers as above."""
    sc = _column()
    escalate = lambda sim: sim.set_stabilization_mode("escalate")
    rng = np.random.default_rng(19)
    direction = [rng.normal(size=(sc.n, c)) * s for c, s in ((3, 1e-3), (4, 1e-2), (3, 0.1), (3, 10.0))]
    end, grads, dtheta, info, roll = _gpu(gpu_api, sc, 20, escalate)
    tans, _ = _dual(orc_api, sc, 20, direction, escalate)
    assert info["replay_dx"] <= 1e-9, info
    assert roll.signature()[:, 5].sum() > 0, "the stabilization pass did not run"
    for k in range(3):
        assert abs(dtheta[k] - tans[k]) <= RTOL * max(abs(tans[k]), 1e-6 * np.abs(tans).max()), (k, dtheta, tans)
    dirderiv = sum(np.sum(g * d) for g, d in zip(grads, direction))
    assert abs(dirderiv - tans[3]) <= RTOL * max(abs(tans[3]), 1e-6), (dirderiv, tans[3])
