"""Differentiable rollout of the plain FP64 XPBD step: forward and hand-written adjoint on the B200.

`XpbdRollout(sim)` wraps a configured FP64 `Simulation` (spheres without point shells, planes,
gravity on with the Gauss-Seidel velocity solve, stabilization "off", "onesided" or "escalate"; no
periodicity, growth, thermostat or pair materials). `rollout(x0, q0, v0, w0, theta, substeps)`
runs `substeps` substeps of the production step (src/sim.hpp:97-488, `pdem_step`) from the start
state (positions, quaternions x y z w, velocities, angular velocities) with
theta = (eN, eT, mu) of `set_material_params`, as a `torch.autograd.Function`: the outputs are the
end state, and `backward` returns the gradients with respect to the start state and theta.

Scheme (the library's pdem_xa_* entry points, include/pdem.h):
- the forward records, for every substep, its start state and warm-start ledger (a checkpoint of
  the compact state) and the decisions the step took: contacts, manifolds, both colourings, the
  side flags of the stabilization pass and the three sweep counts;
- the backward replays each substep from its checkpoint with the forward's expressions, keeping the
  input of every sweep update, and reverses it: the position sweeps, the velocity commit, the
  stabilization and main PGS sweeps in reverse colour and sweep order over the frozen colouring,
  the warm start, the approach velocities, the ledger gather, the manifold sums, the contact
  geometry and the velocity prediction. The friction, restitution and impulse-clamp branches are
  the ones the forward took; the gradient is that of the branch taken (the step is piecewise
  smooth: a contact onset or release inside the rollout is a jump the gradient does not see).
Young's modulus does not enter the XPBD step; its gradient is defined on the Hertz path
(`peclet.dem.adjoint.HertzSpheres`).

One record per simulation: a second forward on the same simulation before the first one's
backward makes that backward raise RuntimeError. There is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._capi import CApiSimulation


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class XpbdRollout:
    """Recorded, differentiable rollouts of one FP64 simulation."""

    def __init__(self, sim: CApiSimulation, device=None):
        if sim.precision != "fp64":
            raise ValueError("the XPBD adjoint runs on the FP64 plain path (precision 'fp64')")
        if not torch.cuda.is_available():
            raise RuntimeError("XpbdRollout needs a CUDA device (there is no CPU path)")
        if not sim._api.has("xa_begin"):
            raise RuntimeError("this library has no XPBD adjoint entry points")
        self.sim = sim
        self.device = torch.device(device or "cuda")
        self.generation = 0

    def _check(self, status, what):
        self.sim._api.check(status, what)

    def info(self):
        """Record statistics: substeps, record bytes, workspace bytes, largest sweep count, and the
        replay's largest deviation from the recorded next state in the last backward (positions in
        global-scale units, velocities in m/s)."""
        out = (C.c_long * 4)()
        err = (C.c_double * 2)()
        self._check(self.sim._f["xa_info"](self.sim._h, out, err), "xa_info")
        return {"substeps": out[0], "record_bytes": out[1], "work_bytes": out[2], "max_sweeps": out[3],
                "replay_dx": err[0], "replay_dv": err[1]}

    def signature(self):
        """The last rollout's discrete decisions, one row per substep: contacts, manifolds, colours
        of the velocity and position colourings, main / stabilization / position sweeps. Two
        rollouts with equal signatures took the same contact sets, colourings and adaptive stops."""
        n = int(self.sim._f["xa_signature"](self.sim._h, None, 0))
        if n < 0:
            self._check(1, "xa_signature")
        out = np.zeros(7 * max(n, 1), np.int64)
        self.sim._f["xa_signature"](self.sim._h, out.ctypes.data_as(C.POINTER(C.c_long)), out.size)
        return out[: 7 * n].reshape(n, 7)

    def branches(self):
        """Hash of the branch decisions of every sweep update of the last rollout (impulse clamps,
        restitution cut-off, friction cone, active position contacts), from a replay of its record.
        Equal `signature()` and equal `branches()` mean two rollouts ran the same smooth piece of the
        step, so their central difference certifies the gradient."""
        h = C.c_ulonglong(0)
        self._check(self.sim._f["xa_branches"](self.sim._h, C.byref(h)), "xa_branches")
        return int(h.value)

    def rollout(self, x0, q0, v0, w0, theta, substeps: int, dt: float = 0.0):
        """End state (x, q, v, w) after `substeps` substeps of length dt (0: the simulation's)."""
        if substeps < 1:
            raise ValueError("substeps must be at least 1")
        return _XpbdFn.apply(self, int(substeps), float(dt), x0, q0, v0, w0, theta)

    __call__ = rollout


class _XpbdFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, roll, substeps, dt, x0, q0, v0, w0, theta):
        sim = roll.sim
        dev = roll.device
        rows = [t.detach().to(device=dev, dtype=torch.float64).contiguous() for t in (x0, q0, v0, w0)]
        n = int(rows[0].shape[0])
        for t, cols in zip(rows, (3, 4, 3, 3)):
            if t.shape != (n, cols):
                raise ValueError("start state rows: x, v, w (n, 3) and q (n, 4)")
        th = np.asarray(theta.detach().cpu().double().numpy() if torch.is_tensor(theta) else theta, np.float64)
        if th.shape != (3,):
            raise ValueError("theta = (eN, eT, mu)")
        sim.set_material_params(float(th[0]), float(th[1]), float(th[2]))
        torch.cuda.synchronize(dev)
        h, f = sim._h, sim._f
        roll._check(f["xa_begin"](h, *[_ptr(t) for t in rows], n), "xa_begin")
        roll._check(f["xa_step"](h, dt, substeps), "xa_step")
        out = [torch.empty((n, c), dtype=torch.float64, device=dev) for c in (3, 4, 3, 3)]
        roll._check(f["xa_state"](h, *[_ptr(t) for t in out]), "xa_state")
        roll.generation += 1
        ctx.roll, ctx.gen, ctx.n = roll, roll.generation, n
        ctx.theta_dtype = theta.dtype if torch.is_tensor(theta) else torch.float64
        ctx.theta_device = theta.device if torch.is_tensor(theta) else torch.device("cpu")
        ctx.in_dtypes = [t.dtype for t in (x0, q0, v0, w0)]
        return tuple(out)

    @staticmethod
    def backward(ctx, gx, gq, gv, gw):
        roll = ctx.roll
        if roll.generation != ctx.gen:
            raise RuntimeError("XpbdRollout: the record was replaced by a later forward on the same simulation")
        dev, n = roll.device, ctx.n
        grads = []
        for g, cols in zip((gx, gq, gv, gw), (3, 4, 3, 3)):
            if g is None:
                g = torch.zeros((n, cols), dtype=torch.float64, device=dev)
            grads.append(g.to(device=dev, dtype=torch.float64).contiguous())
        d = [torch.empty((n, c), dtype=torch.float64, device=dev) for c in (3, 4, 3, 3)]
        dth = (C.c_double * 3)()
        torch.cuda.synchronize(dev)
        roll._check(roll.sim._f["xa_backward"](roll.sim._h, *[_ptr(t) for t in grads], *[_ptr(t) for t in d], dth),
                    "xa_backward")
        dtheta = torch.tensor(list(dth), dtype=ctx.theta_dtype, device=ctx.theta_device)
        dx, dq, dv, dw = [t.to(dt) for t, dt in zip(d, ctx.in_dtypes)]
        return None, None, None, dx, dq, dv, dw, dtheta
