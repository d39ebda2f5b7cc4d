"""The differentiable Hertz rollout on the GPU (peclet.dem.adjoint, pdem_hz_* C ABI): its forward
against the CPU restatement, its adjoint gradients against the restatement's forward-mode dual
numbers and against central finite differences of the GPU forward (relative step 1e-4, FP64), the
checkpointed windows against one long window, the FP32 form against FP64, and the
torch.autograd.Function path."""
import os
import sys

import numpy as np
import pytest

import hertz_cases as HC

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import hertz_spheres as H  # noqa: E402

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _sim(c, precision="fp64", checkpoint=20, skin=None, list_every=25):
    from peclet.dem.adjoint import HertzSpheres
    return HertzSpheres(c["r"], c["m"], c["I"], c["first"], c["planes"], HC.NU, HC.DT, c["g"], precision,
                        checkpoint, skin, list_every=list_every)


def _oracle(c):
    return H.Model(c["r"], c["m"], c["I"], c["first"], c["planes"], HC.NU, HC.DT, c["g"])


def _t(a, sim):
    return torch.as_tensor(np.asarray(a), dtype=sim.dtype, device=sim.device)


def _grads(sim, c, steps, cx, cv, theta=HC.THETA):
    """Gradients of L = sum(cx * x_T) + sum(cv * v_T) through the adjoint."""
    (x, v, w), tape = sim.run(_t(c["x0"], sim), _t(c["v0"], sim), _t(c["w0"], sim), theta, steps, record=True)
    gx, gv, gw, gt = sim.adjoint(tape, theta, _t(cx, sim), _t(cv, sim), torch.zeros_like(w))
    return [a.double().cpu().numpy() for a in (gx, gv, gw, gt)]


def _loss(sim, c, steps, cx, cv, theta=HC.THETA, x0=None, v0=None, w0=None):
    (x, v, _), _ = sim.run(_t(c["x0"] if x0 is None else x0, sim), _t(c["v0"] if v0 is None else v0, sim),
                           _t(c["w0"] if w0 is None else w0, sim), theta, steps)
    return float((x.double().cpu().numpy() * cx).sum() + (v.double().cpu().numpy() * cv).sum())


CASES = [("pair", 100), ("floor", 100), ("gas", 60)]


@pytest.mark.parametrize("case,steps", CASES)
def test_forward_matches_oracle(gpu_api, case, steps):
    c = getattr(HC, case)()
    sim = _sim(c)
    (x, v, w), _ = sim.run(_t(c["x0"], sim), _t(c["v0"], sim), _t(c["w0"], sim), HC.THETA, steps)
    xo, vo, wo = _oracle(c).rollout(c["x0"], c["v0"], c["w0"], *HC.THETA, steps)
    # force sums are atomics on the GPU: agreement to rounding, not bit-exact
    np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=0, atol=1e-14)
    np.testing.assert_allclose(v.cpu().numpy(), vo, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(w.cpu().numpy(), wo, rtol=1e-9, atol=1e-9)
    assert sim.stats["windows"] == -(-steps // 20)


@pytest.mark.parametrize("case,steps", CASES)
def test_adjoint_matches_dual(gpu_api, case, steps):
    """Adjoint (reverse) and dual (forward) derivatives of the same discrete map: equal to
    rounding, along theta's axes and random directions of the initial state."""
    c = getattr(HC, case)()
    n = len(c["r"])
    rng = np.random.default_rng(7)
    cx, cv = rng.standard_normal((n, 3)), 1e-3 * rng.standard_normal((n, 3))
    dx, dv, dw = (rng.standard_normal((n, 3)) for _ in range(3))
    gx, gv, gw, gt = _grads(_sim(c), c, steps, cx, cv)
    tans = [{"theta": np.eye(3)[k]} for k in range(3)] + [{"x": dx}, {"v": dv}, {"w": dw}]
    xd, vd, _ = H.jvp(_oracle(c), c["x0"], c["v0"], c["w0"], HC.THETA, tans, steps)
    want = (xd.d * cx[..., None]).sum((0, 1)) + (vd.d * cv[..., None]).sum((0, 1))
    got = np.concatenate([gt, [(gx * dx).sum(), (gv * dv).sum(), (gw * dw).sum()]])
    for k, (a, b) in enumerate(zip(got, want)):
        assert abs(a - b) <= 1e-7 * abs(b) + 1e-24, f"{case}: direction {k}: adjoint {a} vs dual {b}"


@pytest.mark.parametrize("case,steps", CASES)
def test_adjoint_matches_finite_differences(gpu_api, case, steps):
    """Central differences of the GPU forward, relative step 1e-4 on theta, within 1e-3."""
    c = getattr(HC, case)()
    n = len(c["r"])
    rng = np.random.default_rng(5)
    cx, cv = rng.standard_normal((n, 3)), np.zeros((n, 3))
    sim = _sim(c)
    _, gv, _, gt = _grads(sim, c, steps, cx, cv)
    for k in range(3):
        h = 1e-4 * HC.THETA[k]
        tp, tm = HC.THETA.copy(), HC.THETA.copy()
        tp[k] += h
        tm[k] -= h
        fd = (_loss(sim, c, steps, cx, cv, tp) - _loss(sim, c, steps, cx, cv, tm)) / (2 * h)
        assert abs(gt[k] - fd) <= 1e-3 * abs(fd) + 1e-24, f"{case}: theta[{k}]: adjoint {gt[k]} vs FD {fd}"
    dv = rng.standard_normal((n, 3))
    h = 1e-4 * 0.1
    fd = (_loss(sim, c, steps, cx, cv, v0=c["v0"] + h * dv) - _loss(sim, c, steps, cx, cv, v0=c["v0"] - h * dv)) / (2 * h)
    got = (gv * dv).sum()
    assert abs(got - fd) <= 1e-3 * abs(fd), f"{case}: v0 direction: adjoint {got} vs FD {fd}"


@pytest.mark.parametrize("checkpoint,list_every", [(7, 3), (20, 6), (13, 13)])
def test_windows_match_one_window(gpu_api, checkpoint, list_every):
    """Contact lists rebuilt every `list_every` substeps (histories carried by key, history
    adjoints mapped back) inside checkpoints of `checkpoint` substeps give the result of one
    window over the whole rollout."""
    c = HC.gas()
    n = len(c["r"])
    rng = np.random.default_rng(9)
    cx, cv = rng.standard_normal((n, 3)), rng.standard_normal((n, 3))
    sim = _sim(c, checkpoint=checkpoint, list_every=list_every)
    a = _grads(sim, c, 60, cx, cv)
    assert sim.stats["windows"] > 60 // checkpoint
    b = _grads(_sim(c, checkpoint=1000, list_every=1000), c, 60, cx, cv)
    for ga, gb in zip(a, b):
        np.testing.assert_allclose(ga, gb, rtol=1e-9, atol=1e-12 * np.abs(gb).max())


def test_fp32_gradients_near_fp64(gpu_api):
    c = HC.gas()
    n = len(c["r"])
    rng = np.random.default_rng(4)
    cx, cv = rng.standard_normal((n, 3)), np.zeros((n, 3))
    g64 = _grads(_sim(c, "fp64"), c, 60, cx, cv)
    g32 = _grads(_sim(c, "fp32"), c, 60, cx, cv)
    for k, (a, b) in enumerate(zip(g32, g64)):
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err < 2e-2, f"gradient {k}: FP32 max error {err:.2e} of the FP64 scale"


def test_autograd_function(gpu_api):
    """loss.backward() through HertzSpheres.rollout equals the explicit adjoint."""
    c = HC.gas()
    sim = _sim(c)
    n = len(c["r"])
    rng = np.random.default_rng(2)
    target = _t(c["x0"] + 1e-4 * rng.standard_normal((n, 3)), sim)
    x0 = _t(c["x0"], sim).requires_grad_(True)
    v0 = _t(c["v0"], sim).requires_grad_(True)
    w0 = _t(c["w0"], sim).requires_grad_(True)
    theta = torch.tensor(HC.THETA, dtype=torch.float64, requires_grad=True)
    x, v, w = sim.rollout(x0, v0, w0, theta, 40)
    loss = ((x - target) ** 2).sum(dim=1).mean()
    loss.backward()
    gx = (2.0 / n) * (x.detach() - target)
    bx, bv, bw, bt = _grads(sim, c, 40, gx.cpu().numpy(), np.zeros((n, 3)))
    np.testing.assert_allclose(v0.grad.cpu().numpy(), bv, rtol=1e-9, atol=1e-12 * np.abs(bv).max())
    np.testing.assert_allclose(theta.grad.numpy(), bt, rtol=1e-9)
    assert theta.grad.dtype == torch.float64 and v0.grad.shape == (n, 3)


def test_rejects_bad_arguments(gpu_api):
    from peclet.dem.adjoint import HertzSpheres
    c = HC.pair()
    with pytest.raises(ValueError):
        HertzSpheres(c["r"], c["m"][:1], c["I"], precision="fp64")
    with pytest.raises(ValueError):
        HertzSpheres(c["r"], c["m"], c["I"], scene_first=[0, 3])
    sim = _sim(c)
    with pytest.raises(ValueError):
        sim.run(_t(c["x0"], sim), _t(c["v0"], sim), _t(c["w0"], sim), (0.0, 0.7, 0.35), 5)


def test_hand_reversal_matches_dual_jacobians(gpu_api):
    """The hand reversal of each contact law (mode 0) against the contact's local Jacobian taken by
    dual numbers through the engine's hertzForce (mode 1), on the same recorded rollout."""
    c = HC.gas()
    n = len(c["r"])
    rng = np.random.default_rng(8)
    sim = _sim(c)
    (x, v, w), tape = sim.run(_t(c["x0"], sim), _t(c["v0"], sim), _t(c["w0"], sim), HC.THETA, 60, record=True)
    g = [_t(rng.standard_normal((n, 3)), sim) for _ in range(3)]
    a = [t.cpu().numpy() for t in sim.adjoint(tape, HC.THETA, *g, mode=0)]
    b = [t.cpu().numpy() for t in sim.adjoint(tape, HC.THETA, *g, mode=1)]
    for k, (ga, gb) in enumerate(zip(a, b)):
        np.testing.assert_allclose(ga, gb, rtol=1e-10, atol=1e-12 * np.abs(gb).max(), err_msg=f"gradient {k}")


@pytest.mark.parametrize("case,steps", CASES)
def test_jvp_matches_oracle_dual(gpu_api, case, steps):
    """The GPU tangent-linear run against the restatement's dual numbers, same direction."""
    c = getattr(HC, case)()
    n = len(c["r"])
    rng = np.random.default_rng(12)
    dx, dv, dw = (rng.standard_normal((n, 3)) for _ in range(3))
    dth = np.array([1e5, 0.01, 0.01])
    sim = _sim(c)
    (x, v, w), (xd, vd, wd) = sim.jvp(_t(c["x0"], sim), _t(c["v0"], sim), _t(c["w0"], sim), HC.THETA,
                                      _t(dx, sim), _t(dv, sim), _t(dw, sim), dth, steps)
    ox, ov, ow = H.jvp(_oracle(c), c["x0"], c["v0"], c["w0"], HC.THETA, [{"x": dx, "v": dv, "w": dw, "theta": dth}],
                       steps)
    for got, want in ((xd, ox), (vd, ov), (wd, ow)):
        want = want.d[..., 0]
        np.testing.assert_allclose(got.cpu().numpy(), want, rtol=1e-8, atol=1e-10 * np.abs(want).max())
    np.testing.assert_allclose(x.cpu().numpy(), ox.v, rtol=0, atol=1e-14)


def test_adjoint_matches_jvp(gpu_api):
    """<adjoint gradient, direction> = tangent-linear derivative along it, on the GPU alone."""
    c = HC.gas()
    n = len(c["r"])
    rng = np.random.default_rng(13)
    cx, cv = rng.standard_normal((n, 3)), rng.standard_normal((n, 3))
    dx, dv, dw = (rng.standard_normal((n, 3)) for _ in range(3))
    dth = np.array([1e5, 0.01, 0.01])
    sim = _sim(c, checkpoint=13)
    gx, gv, gw, gt = _grads(sim, c, 60, cx, cv)
    _, (xd, vd, _) = sim.jvp(_t(c["x0"], sim), _t(c["v0"], sim), _t(c["w0"], sim), HC.THETA, _t(dx, sim),
                             _t(dv, sim), _t(dw, sim), dth, 60)
    lhs = (gx * dx).sum() + (gv * dv).sum() + (gw * dw).sum() + (gt * dth).sum()
    rhs = (xd.cpu().numpy() * cx).sum() + (vd.cpu().numpy() * cv).sum()
    assert abs(lhs - rhs) <= 1e-9 * abs(rhs), (lhs, rhs)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("scenes,per", [(3, 40), (2, 3000), (1, 9000)])
def test_contact_candidates_match_brute_force(gpu_api, precision, scenes, per):
    """Candidate lists (cell grid in shared memory, or the global-memory scan for scenes too large
    for it) equal a brute-force enumeration, in (i, j) order with planes after spheres."""
    rng = np.random.default_rng(scenes * 1000 + per)
    L = 0.02 * (per / 40) ** (1 / 3)
    n = scenes * per
    x = rng.uniform(0, L, (n, 3))
    r = rng.uniform(0.5e-3, 1e-3, n)
    m, I = HC.props(r)
    c = dict(x0=x, v0=np.zeros((n, 3)), w0=np.zeros((n, 3)), r=r, m=m, I=I, first=[per * s for s in range(scenes + 1)],
             planes=HC.box(L), g=(0.0, 0.0, 0.0))
    sim = _sim(c, precision)
    skin = 0.3e-3
    got = sim.contacts(_t(x, sim), skin).cpu().numpy()
    xs = x.astype(np.float32).astype(np.float64) if precision == "fp32" else x
    want = []
    for s in range(scenes):
        a, b = per * s, per * (s + 1)
        for i in range(a, b):
            d = np.linalg.norm(xs[i + 1:b] - xs[i], axis=1)
            lim = r[i] + r[i + 1:b] + skin
            for j in np.nonzero(d < lim)[0]:
                want.append((i, i + 1 + j))
            dist = [(xs[i] - np.array(p[:3])) @ np.array(p[3:]) for p in HC.box(L)]
            for k, dk in enumerate(dist):
                if dk < r[i] + skin:
                    want.append((i, -k - 1))
    want = np.array(want, dtype=np.int64).reshape(-1, 2)
    if precision == "fp32":  # rounding at the threshold may differ: compare away from it
        assert abs(len(got) - len(want)) <= max(3, len(want) // 1000)
    else:
        np.testing.assert_array_equal(got, want)


def test_fd_on_certified_window_calibration(gpu_api):
    """The calibration workload (4 boxes of 2,048 spheres, 64 substeps, loss = mean squared distance
    to targets made at the hidden parameters): central differences at relative step 1e-4 along E,
    e, mu and along a random direction of the first box's initial velocities, each on a window that
    the test certifies: the +h and -h rollouts touch exactly the nominal rollout's contacts in every
    substep. There the rollout is smooth and the adjoint agrees with the differences within 1e-3.
    On the 64-box workload a direction over all spheres at that step is not certified (contacts
    begin or end between the rollouts: the 51 % disagreement once reported there); here such a
    direction is checked at a 100 times smaller step, and only when certified."""
    from peclet.dem import workloads as W
    from peclet.dem.adjoint import HertzSpheres
    c = W.calibration_boxes(scenes=4)
    n = len(c["r"])
    sim = HertzSpheres(c["r"], c["m"], c["I"], c["first"], c["planes"], 0.3, 2e-5, (0.0, 0.0, -9.81), "fp64", 100)
    dev = torch.device("cuda")
    x0, v0, w0 = (torch.as_tensor(c[k], device=dev) for k in ("x0", "v0", "w0"))
    hidden, guess, steps = (5e6, 0.7, 0.35), (4e6, 0.6, 0.3), 64
    (xt, _, _), _ = sim.run(x0, v0, w0, hidden, steps)

    def loss(theta, vv):
        (x, _, _), _ = sim.run(x0, vv, w0, theta, steps)
        return float(((x - xt) ** 2).sum()) / n

    th = torch.tensor(guess, dtype=torch.float64, requires_grad=True)
    vr = v0.clone().requires_grad_(True)
    x, _, _ = sim.rollout(x0, vr, w0, th, steps)
    (((x - xt) ** 2).sum() / n).backward()
    g, gv = th.grad.numpy(), vr.grad
    base = sim.active_sets(x0, v0, w0, guess, steps)
    assert sum(a.numel() for a in base) > 0  # contacts are touching inside the window

    def certified(theta, vv):
        return HertzSpheres.same_branches(sim.active_sets(x0, vv, w0, theta, steps), base)

    for k in range(3):
        h = 1e-4 * guess[k]
        tp, tm = list(guess), list(guess)
        tp[k] += h
        tm[k] -= h
        assert certified(tp, v0) and certified(tm, v0), f"theta[{k}]: the window is not certified"
        fd = (loss(tp, v0) - loss(tm, v0)) / (2 * h)
        assert abs(g[k] - fd) <= 1e-3 * abs(fd), f"theta[{k}]: adjoint {g[k]} vs FD {fd}"
    gen = torch.Generator(device="cpu").manual_seed(5)
    dv = torch.randn(v0.shape, generator=gen, dtype=torch.float64).to(dev)
    dv1 = dv.clone()
    dv1[2048:] = 0.0
    h = 1e-4 * 0.2
    assert certified(guess, v0 + h * dv1) and certified(guess, v0 - h * dv1)
    fd = (loss(guess, v0 + h * dv1) - loss(guess, v0 - h * dv1)) / (2 * h)
    got = float((gv * dv1).sum())
    assert abs(got - fd) <= 1e-3 * abs(fd), f"v0 (first box): adjoint {got} vs FD {fd}"
    h = 1e-6 * 0.2
    if certified(guess, v0 + h * dv) and certified(guess, v0 - h * dv):
        fd = (loss(guess, v0 + h * dv) - loss(guess, v0 - h * dv)) / (2 * h)
        got = float((gv * dv).sum())
        assert abs(got - fd) <= 2e-3 * abs(fd), f"v0 (all boxes, step 1e-6): adjoint {got} vs FD {fd}"
