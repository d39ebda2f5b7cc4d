"""Differentiable Hertz-Mindlin rollout of spheres: forward and hand-written adjoint on the B200.

`HertzSpheres` holds the static description (radii, masses, moments of inertia, scenes, planes,
Poisson ratio, dt, gravity) and `rollout(x0, v0, w0, theta, steps)` runs the explicit Hertz
substep of the reference's engine (src/solver_hertz.hpp:88-144 pair law, the wall branch of
src/solver_hertz.hpp:300-372 for planes at rest, the kick-drift of src/solver_hertz.hpp:374-425)
as a `torch.autograd.Function`: the outputs are the final positions, velocities and angular
velocities, and `backward` returns the gradients with respect to the initial state and
theta = (Young's modulus E, restitution e, friction mu).

Scheme:
- substeps run in windows of `checkpoint` substeps; at each window start the candidate pairs of
  each scene are rebuilt with a skin that covers the window's motion (checked after the window:
  if a sphere moved more than half the skin, the window is rerun with twice the skin), and the
  Mindlin histories are carried to the new list by pair key;
- the forward keeps only each window's start state (the checkpoint), its pair list and the key
  map; the backward recomputes each window's substeps from its checkpoint, stores them, and runs
  the adjoint kernels over them in reverse (pdem_hz_backward), then maps the history adjoints
  back through the key map to the previous window's list.
The CUDA library does all the arithmetic; torch provides device memory and the stream. There is no
CPU path: without a CUDA device construction raises RuntimeError.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _API
from ._capi import HzModel

_CODES = {torch.float64: 64, torch.float32: 32}


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None and t.numel() else None


class HertzSpheres:
    """Spheres (radius, mass, scalar moment of inertia) in independent scenes [first[s], first[s+1])
    with planes (point, normal into the domain) shared by every scene."""

    def __init__(self, radius, mass, inertia, scene_first=None, planes=(), poisson=0.3, dt=2e-5,
                 gravity=(0.0, 0.0, -9.81), precision="fp64", checkpoint=100, skin=None, device=None):
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if not torch.cuda.is_available():
            raise RuntimeError("HertzSpheres needs a CUDA device (there is no CPU path)")
        if checkpoint < 1:
            raise ValueError("checkpoint must be at least 1 substep")
        self.api = _API
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.code = _CODES[self.dtype]
        self.device = torch.device(device or "cuda")
        as_t = lambda a: torch.as_tensor(np.asarray(a, np.float64).ravel(), dtype=self.dtype,
                                          device=self.device).contiguous()
        self.r, self.m, self.I = as_t(radius), as_t(mass), as_t(inertia)
        self.n = int(self.r.numel())
        if self.m.numel() != self.n or self.I.numel() != self.n:
            raise ValueError("radius, mass and inertia must have one value per sphere")
        first = np.asarray(scene_first if scene_first is not None else [0, self.n], np.int64)
        if first[0] != 0 or first[-1] != self.n or np.any(np.diff(first) < 0):
            raise ValueError("scene_first must rise from 0 to the number of spheres")
        end = np.repeat(first[1:], np.diff(first)).astype(np.int32)
        self.scene_first = first
        self.end = torch.as_tensor(end, device=self.device)
        pl = np.asarray(planes, np.float64).reshape(-1, 6).copy()
        if pl.size:
            pl[:, 3:] /= np.linalg.norm(pl[:, 3:], axis=1, keepdims=True)
        self.nplane = int(pl.shape[0])
        self.planes = torch.as_tensor(pl.ravel(), dtype=self.dtype, device=self.device).contiguous()
        self.poisson, self.dt = float(poisson), float(dt)
        self.gravity = tuple(float(g) for g in gravity)
        self.checkpoint = int(checkpoint)
        self.skin_min = float(skin) if skin is not None else 0.5 * float(np.max(np.asarray(radius)))
        self._cnt = torch.empty(max(self.n, 1), dtype=torch.int32, device=self.device)
        self._off = torch.empty(self.n + 1, dtype=torch.int32, device=self.device)
        self._cap = max(1024, 4 * self.n)
        self._buf = torch.empty((self._cap, 2), dtype=torch.int32, device=self.device)
        self.stats = {"windows": 0, "reruns": 0}

    # ---- C ABI helpers ---------------------------------------------------------------------
    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _check(self, status, what):
        self.api.check(status, what)

    def state_size(self, npair):
        return int(self.api.fn["hz_state_size"](self.n, npair, self.nplane))

    def _model(self, pairs, npair, theta):
        M = HzModel()
        M.n, M.npair, M.nplane = self.n, npair, self.nplane
        M.pairs = _ptr(pairs) if npair else None
        M.planes = _ptr(self.planes) if self.nplane else None
        M.radius, M.mass, M.inertia = _ptr(self.r), _ptr(self.m), _ptr(self.I)
        M.youngs, M.restitution, M.friction = theta
        M.poisson, M.dt = self.poisson, self.dt
        M.gravity[:] = self.gravity
        return M

    def pairs(self, x, skin):
        """Candidate pairs (i < j, same scene, gap below skin) of positions x (n, 3), in (i, j) order."""
        x = x.contiguous()
        count = C.c_long(0)
        while True:
            self._check(self.api.fn["hz_pairs"](self.code, _ptr(x), _ptr(self.r), _ptr(self.end), self.n, float(skin),
                                                _ptr(self._cnt), _ptr(self._off), _ptr(self._buf), self._cap,
                                                C.byref(count), self._stream()), "hz_pairs")
            if count.value <= self._cap:
                return self._buf[:count.value].clone()
            self._cap = int(count.value * 1.5) + 1024
            self._buf = torch.empty((self._cap, 2), dtype=torch.int32, device=self.device)

    def forward_window(self, start, pairs, theta, steps, store):
        """Run `steps` substeps from the state block `start`; returns the trajectory buffer
        (steps + 1 blocks when store, else 2 blocks with the final state in block 1)."""
        npair = int(pairs.shape[0])
        S = self.state_size(npair)
        traj = torch.empty(((steps + 1) if store else 2) * S, dtype=self.dtype, device=self.device)
        traj[:S] = start
        work = torch.empty(int(self.api.fn["hz_work_size"](self.n, npair, self.nplane)), dtype=self.dtype,
                           device=self.device)
        M = self._model(pairs, npair, theta)
        self._check(self.api.fn["hz_forward"](self.code, C.byref(M), int(steps), int(bool(store)), _ptr(traj),
                                              _ptr(work), self._stream()), "hz_forward")
        return traj

    # ---- windows ------------------------------------------------------------------------------
    def _skin(self, v, steps):
        t = steps * self.dt
        vmax = float(v.norm(dim=1).max()) if v.numel() else 0.0
        g = float(np.linalg.norm(self.gravity))
        return max(self.skin_min, 3.0 * (vmax * t + 0.5 * g * t * t))

    @staticmethod
    def _keys(pairs, n):
        return pairs[:, 0].long() * n + pairs[:, 1].long()

    def run(self, x0, v0, w0, theta, steps, record=False):
        """Forward rollout. Returns (x, v, w) and, when record, the checkpoint tape."""
        n, nW = self.n, 3 * self.n * self.nplane
        theta = tuple(float(t) for t in theta)
        x, v, w = (torch.as_tensor(a, device=self.device).to(self.dtype).reshape(n, 3).contiguous()
                   for a in (x0, v0, w0))
        xiW = torch.zeros(nW, dtype=self.dtype, device=self.device)
        prev_keys = prev_xiP = None
        tape = []
        k = 0
        while k < steps:
            K = min(self.checkpoint, steps - k)
            skin = self._skin(v, K)
            while True:
                pairs = self.pairs(x, skin)
                npair = int(pairs.shape[0])
                keys = self._keys(pairs, n)
                xiP = torch.zeros((npair, 3), dtype=self.dtype, device=self.device)
                idx = valid = None
                if prev_keys is not None and npair and prev_keys.numel():
                    idx = torch.searchsorted(prev_keys, keys)
                    valid = idx < prev_keys.numel()
                    valid &= prev_keys[idx.clamp(max=prev_keys.numel() - 1)] == keys
                    xiP[valid] = prev_xiP[idx[valid]]
                start = torch.cat([x.reshape(-1), v.reshape(-1), w.reshape(-1), xiP.reshape(-1), xiW])
                traj = self.forward_window(start, pairs, theta, K, store=False)
                S = start.numel()
                end = traj[S:2 * S]
                disp = (end[:3 * n] - start[:3 * n]).reshape(n, 3).norm(dim=1).max() if n else 0.0
                if float(disp) <= 0.5 * skin:
                    break
                skin *= 2.0
                self.stats["reruns"] += 1
            self.stats["windows"] += 1
            if record:
                tape.append({"start": start, "pairs": pairs, "idx": idx, "valid": valid, "steps": K})
            x = end[:3 * n].reshape(n, 3)
            v = end[3 * n:6 * n].reshape(n, 3)
            w = end[6 * n:9 * n].reshape(n, 3)
            prev_xiP = end[9 * n:9 * n + 3 * npair].reshape(npair, 3)
            xiW = end[9 * n + 3 * npair:]
            prev_keys = keys
            k += K
        return (x.clone(), v.clone(), w.clone()), tape

    def adjoint(self, tape, theta, gx, gv, gw):
        """Reverse of a recorded rollout: gradients of the initial (x, v, w) and of theta."""
        n = self.n
        theta = tuple(float(t) for t in theta)
        grad = torch.zeros(3, dtype=torch.float64, device=self.device)
        if not tape:
            return gx, gv, gw, grad
        npair = int(tape[-1]["pairs"].shape[0])
        adj = torch.zeros(self.state_size(npair), dtype=self.dtype, device=self.device)
        adj[:3 * n] = gx.reshape(-1)
        adj[3 * n:6 * n] = gv.reshape(-1)
        adj[6 * n:9 * n] = gw.reshape(-1)
        for t in range(len(tape) - 1, -1, -1):
            win = tape[t]
            pairs, K = win["pairs"], win["steps"]
            npair = int(pairs.shape[0])
            traj = self.forward_window(win["start"], pairs, theta, K, store=True)
            work = torch.empty(int(self.api.fn["hz_work_size"](n, npair, self.nplane)), dtype=self.dtype,
                               device=self.device)
            M = self._model(pairs, npair, theta)
            self._check(self.api.fn["hz_backward"](self.code, C.byref(M), int(K), _ptr(traj), _ptr(adj), _ptr(grad),
                                                   _ptr(work), self._stream()), "hz_backward")
            del traj
            if t == 0:
                break
            prev = int(tape[t - 1]["pairs"].shape[0])
            a = torch.zeros(self.state_size(prev), dtype=self.dtype, device=self.device)
            a[:9 * n] = adj[:9 * n]
            a[9 * n + 3 * prev:] = adj[9 * n + 3 * npair:]
            if win["idx"] is not None:
                valid = win["valid"]
                xb = adj[9 * n:9 * n + 3 * npair].reshape(npair, 3)
                a[9 * n:9 * n + 3 * prev].view(prev, 3).index_add_(0, win["idx"][valid], xb[valid])
            adj = a
        return adj[:3 * n].reshape(n, 3), adj[3 * n:6 * n].reshape(n, 3), adj[6 * n:9 * n].reshape(n, 3), grad

    def rollout(self, x0, v0, w0, theta, steps):
        """Differentiable rollout: (x, v, w) after `steps` substeps; gradients flow to x0, v0, w0
        and theta = tensor([E, e, mu])."""
        return _HertzRollout.apply(x0, v0, w0, theta, self, int(steps))


class _HertzRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x0, v0, w0, theta, sim, steps):
        th = [float(t) for t in theta.detach().cpu().reshape(-1)]
        (x, v, w), tape = sim.run(x0.detach(), v0.detach(), w0.detach(), th, steps, record=True)
        ctx.sim, ctx.tape, ctx.theta = sim, tape, th
        ctx.meta = (x0.dtype, x0.device, theta.dtype, theta.device)
        return x, v, w

    @staticmethod
    def backward(ctx, gx, gv, gw):
        sim = ctx.sim
        z = lambda g: (torch.zeros((sim.n, 3), dtype=sim.dtype, device=sim.device) if g is None
                       else g.to(sim.device, sim.dtype).contiguous())
        bx, bv, bw, gt = sim.adjoint(ctx.tape, ctx.theta, z(gx), z(gv), z(gw))
        xd, xdev, td, tdev = ctx.meta
        ctx.tape = None
        return (bx.to(xdev, xd), bv.to(xdev, xd), bw.to(xdev, xd), gt.to(tdev, td), None, None)
