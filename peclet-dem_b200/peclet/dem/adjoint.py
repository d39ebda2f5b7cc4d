"""Differentiable Hertz-Mindlin rollout of spheres: forward and hand-written adjoint on the B200.

`HertzSpheres` holds the static description (radii, masses, moments of inertia, scenes, planes,
Poisson ratio, dt, gravity) and `rollout(x0, v0, w0, theta, steps)` runs the explicit Hertz
substep of the reference's engine (src/solver_hertz.hpp:88-144 pair law, the wall branch of
src/solver_hertz.hpp:300-372 for planes at rest, the kick-drift of src/solver_hertz.hpp:374-425)
as a `torch.autograd.Function`: the outputs are the final positions, velocities and angular
velocities, and `backward` returns the gradients with respect to the initial state and
theta = (Young's modulus E, restitution e, friction mu).

Scheme:
- substeps run in windows of at most `list_every` substeps that never cross a checkpoint (every
  `checkpoint` substeps); at each window start the candidate contacts (sphere pairs of each scene
  and sphere-plane couples) are rebuilt with a skin that covers the window's motion (2.5 times the
  previous window's largest displacement, a free-flight bound for the first; checked after the
  window: if a sphere moved more than half the skin, the window is rerun with twice the skin),
  and the Mindlin histories are carried to the new list by key;
- the forward keeps only each window's start state (the checkpoint), its contact list and the
  key map; the backward recomputes each window's substeps from its checkpoint, stores them, and
  runs the adjoint kernels over them in reverse (pdem_hz_backward), then maps the history
  adjoints back through the key map to the previous window's list;
- `jvp` is the tangent-linear run (one forward-mode dual tangent through the whole rollout), the
  independent check of the adjoint at full size.
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
                 gravity=(0.0, 0.0, -9.81), precision="fp64", checkpoint=100, skin=None, device=None,
                 list_every=50):
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if not torch.cuda.is_available():
            raise RuntimeError("HertzSpheres needs a CUDA device (there is no CPU path)")
        if checkpoint < 1 or list_every < 1:
            raise ValueError("checkpoint and list_every must be at least 1 substep")
        self.api = _API
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.code = _CODES[self.dtype]
        self.device = torch.device(device or "cuda")
        as_t = lambda a: torch.as_tensor(np.asarray(a, np.float64).ravel(), dtype=self.dtype,
                                          device=self.device).contiguous()
        mass, inertia = np.asarray(mass, np.float64).ravel(), np.asarray(inertia, np.float64).ravel()
        self.r = as_t(radius)
        self.n = int(self.r.numel())
        if mass.size != self.n or inertia.size != self.n:
            raise ValueError("radius, mass and inertia must have one value per sphere")
        if np.any(mass <= 0) or np.any(inertia <= 0):
            raise ValueError("masses and moments of inertia must be positive")
        # the engine's convention: inverse mass and inverse inertia, formed once in double
        self.im, self.iI = as_t(1.0 / mass), as_t(1.0 / inertia)
        first = np.asarray(scene_first if scene_first is not None else [0, self.n], np.int64)
        if first[0] != 0 or first[-1] != self.n or np.any(np.diff(first) < 0):
            raise ValueError("scene_first must rise from 0 to the number of spheres")
        self.scene_first = first
        self._first_h = np.ascontiguousarray(first, dtype=np.int32)
        self.first = torch.as_tensor(self._first_h, device=self.device)
        pl = np.asarray(planes, np.float64).reshape(-1, 6).copy()
        if pl.size:
            pl[:, 3:] /= np.linalg.norm(pl[:, 3:], axis=1, keepdims=True)
        self.nplane = int(pl.shape[0])
        self.planes = torch.as_tensor(pl.ravel(), dtype=self.dtype, device=self.device).contiguous()
        self.poisson, self.dt = float(poisson), float(dt)
        self.gravity = tuple(float(g) for g in gravity)
        self.checkpoint = int(checkpoint)
        self.list_every = int(list_every)
        self.skin_min = float(skin) if skin is not None else 0.1 * float(np.max(np.asarray(radius)))
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

    def state_size(self, ncontact):
        return int(self.api.fn["hz_state_size"](self.n, ncontact))

    def _work(self, ncontact):
        return torch.empty(int(self.api.fn["hz_work_size"](self.n, ncontact)), dtype=self.dtype, device=self.device)

    def _model(self, cont, theta):
        nc = int(cont.shape[0])
        M = HzModel()
        M.n, M.ncontact, M.nplane = self.n, nc, self.nplane
        M.contacts = _ptr(cont) if nc else None
        M.planes = _ptr(self.planes) if self.nplane else None
        M.radius, M.inv_mass, M.inv_inertia = _ptr(self.r), _ptr(self.im), _ptr(self.iI)
        M.youngs, M.restitution, M.friction = theta
        M.poisson, M.dt = self.poisson, self.dt
        M.gravity[:] = self.gravity
        return M

    def contacts(self, x, skin):
        """Candidate contacts of positions x (n, 3): per sphere i in order, the spheres j > i of its
        scene with a gap below skin, then the planes within skin of it (j = -1 - plane)."""
        x = x.contiguous()
        count = C.c_long(0)
        while True:
            self._check(self.api.fn["hz_contacts"](self.code, _ptr(x), _ptr(self.r),
                                                   self._first_h.ctypes.data_as(C.POINTER(C.c_int)), _ptr(self.first),
                                                   len(self.scene_first) - 1, _ptr(self.planes), self.nplane,
                                                   float(skin), _ptr(self._cnt),
                                                   _ptr(self._off), _ptr(self._buf), self._cap, C.byref(count),
                                                   self._stream()), "hz_contacts")
            if count.value <= self._cap:
                return self._buf[:count.value].clone()
            self._cap = int(count.value * 1.5) + 1024
            self._buf = torch.empty((self._cap, 2), dtype=torch.int32, device=self.device)

    def forward_window(self, start, cont, theta, steps, store):
        """Run `steps` substeps from the state block `start`; returns the trajectory buffer
        (steps + 1 blocks when store, else 2 blocks with the final state in block 1)."""
        S = self.state_size(int(cont.shape[0]))
        traj = torch.empty(((steps + 1) if store else 2) * S, dtype=self.dtype, device=self.device)
        traj[:S] = start
        M = self._model(cont, theta)
        self._check(self.api.fn["hz_forward"](self.code, C.byref(M), int(steps), int(bool(store)), _ptr(traj),
                                              _ptr(self._work(int(cont.shape[0]))), self._stream()), "hz_forward")
        return traj

    # ---- windows ------------------------------------------------------------------------------
    def _skin(self, v, steps):
        t = steps * self.dt
        vmax = float(v.norm(dim=1).max()) if v.numel() else 0.0
        g = float(np.linalg.norm(self.gravity))
        return max(self.skin_min, 2.2 * (vmax * t + 0.5 * g * t * t))

    def _keys(self, cont):
        j = cont[:, 1].long()
        return cont[:, 0].long() * (self.n + self.nplane) + torch.where(j >= 0, j, self.n - 1 - j)

    @staticmethod
    def _remap(prev_keys, keys):
        """Index of each new contact in the previous list (keys sorted), or None when none can match."""
        if prev_keys is None or not keys.numel() or not prev_keys.numel():
            return None, None
        idx = torch.searchsorted(prev_keys, keys)
        valid = idx < prev_keys.numel()
        valid &= prev_keys[idx.clamp(max=prev_keys.numel() - 1)] == keys
        return idx, valid

    def _state(self, x, v, w, xi):
        return torch.cat([x.reshape(-1), v.reshape(-1), w.reshape(-1), xi.reshape(-1)])

    def _split(self, block, nc):
        n = self.n
        return (block[:3 * n].reshape(n, 3), block[3 * n:6 * n].reshape(n, 3), block[6 * n:9 * n].reshape(n, 3),
                block[9 * n:9 * n + 3 * nc].reshape(nc, 3))

    def _carry(self, prev, idx, valid, nc):
        xi = torch.zeros((nc, 3), dtype=self.dtype, device=self.device)
        if idx is not None:
            xi[valid] = prev[idx[valid]]
        return xi

    def _window_len(self, k, steps):
        """Substeps of the window starting at substep k: at most list_every, never across a
        checkpoint boundary."""
        return min(self.list_every, steps - k, self.checkpoint - k % self.checkpoint)

    def _start(self, x, v, w, skin, prev_keys, prev_xi):
        cont = self.contacts(x, skin)
        keys = self._keys(cont)
        idx, valid = self._remap(prev_keys, keys)
        return cont, keys, idx, valid, self._state(x, v, w, self._carry(prev_xi, idx, valid, int(cont.shape[0])))

    def run(self, x0, v0, w0, theta, steps, record=False):
        """Forward rollout. Returns (x, v, w) and, when record, the tape: per window its contact
        list, key map and length, and at every checkpoint the window's start state."""
        n = self.n
        theta = tuple(float(t) for t in theta)
        x, v, w = (torch.as_tensor(a, device=self.device).to(self.dtype).reshape(n, 3).contiguous()
                   for a in (x0, v0, w0))
        prev_keys = prev_xi = None
        tape = []
        k, rate = 0, None
        while k < steps:
            K = self._window_len(k, steps)
            skin = self._skin(v, K) if rate is None else max(self.skin_min, 2.5 * rate * K)
            while True:
                cont, keys, idx, valid, start = self._start(x, v, w, skin, prev_keys, prev_xi)
                traj = self.forward_window(start, cont, theta, K, store=False)
                S = start.numel()
                end = traj[S:2 * S]
                disp = float((end[:3 * n] - start[:3 * n]).reshape(n, 3).norm(dim=1).max()) if n else 0.0
                if disp <= 0.5 * skin:
                    break
                skin *= 2.0
                self.stats["reruns"] += 1
            rate = disp / K  # the next window's skin: 2.5 times this window's largest displacement
            self.stats["windows"] += 1
            if record:
                tape.append({"start": start if k % self.checkpoint == 0 else None, "cont": cont, "idx": idx,
                             "valid": valid, "steps": K})
            x, v, w, prev_xi = self._split(end, int(cont.shape[0]))
            prev_keys = keys
            k += K
        return (x.clone(), v.clone(), w.clone()), tape

    def _adjoint_map(self, adj, win, prev):
        """Adjoint of the previous window's final state from that of this window's start: the
        bodies' parts carry over, the history adjoints go back through the key map."""
        n = self.n
        nc = int(win["cont"].shape[0])
        a = torch.zeros(self.state_size(prev), dtype=self.dtype, device=self.device)
        a[:9 * n] = adj[:9 * n]
        if win["idx"] is not None:
            valid = win["valid"]
            xb = adj[9 * n:].reshape(nc, 3)
            a[9 * n:].view(prev, 3).index_add_(0, win["idx"][valid], xb[valid])
        return a

    def adjoint(self, tape, theta, gx, gv, gw, mode=0):
        """Reverse of a recorded rollout: gradients of the initial (x, v, w) and of theta.
        Each checkpoint's windows are recomputed from its stored state (all their substeps kept),
        then reversed window by window. mode 0 reverses each contact law by hand; mode 1 uses
        dual-number local Jacobians."""
        n = self.n
        theta = tuple(float(t) for t in theta)
        grad = torch.zeros(3, dtype=torch.float64, device=self.device)
        if not tape:
            return gx, gv, gw, grad
        adj = torch.zeros(self.state_size(int(tape[-1]["cont"].shape[0])), dtype=self.dtype, device=self.device)
        adj[:3 * n] = gx.reshape(-1)
        adj[3 * n:6 * n] = gv.reshape(-1)
        adj[6 * n:9 * n] = gw.reshape(-1)
        heads = [t for t, win in enumerate(tape) if win["start"] is not None]
        for g in range(len(heads) - 1, -1, -1):
            lo, hi = heads[g], (heads[g + 1] if g + 1 < len(heads) else len(tape))
            trajs, start = [], tape[lo]["start"]
            for t in range(lo, hi):  # recompute the checkpoint's windows, keeping every substep
                win = tape[t]
                if t > lo:
                    x, v, w, xi = self._split(end, int(tape[t - 1]["cont"].shape[0]))
                    start = self._state(x, v, w, self._carry(xi, win["idx"], win["valid"], int(win["cont"].shape[0])))
                traj = self.forward_window(start, win["cont"], theta, win["steps"], store=True)
                S = start.numel()
                end = traj[win["steps"] * S:(win["steps"] + 1) * S]
                trajs.append(traj)
            for t in range(hi - 1, lo - 1, -1):
                win = tape[t]
                M = self._model(win["cont"], theta)
                self._check(self.api.fn["hz_backward"](self.code, C.byref(M), int(win["steps"]), _ptr(trajs[t - lo]),
                                                       _ptr(adj), _ptr(grad), _ptr(self._work(int(win["cont"].shape[0]))),
                                                       int(mode), self._stream()), "hz_backward")
                trajs[t - lo] = None
                if t > 0:
                    adj = self._adjoint_map(adj, win, int(tape[t - 1]["cont"].shape[0]))
        return adj[:3 * n].reshape(n, 3), adj[3 * n:6 * n].reshape(n, 3), adj[6 * n:9 * n].reshape(n, 3), grad

    def jvp(self, x0, v0, w0, theta, dx0, dv0, dw0, dtheta, steps):
        """Tangent-linear (forward-mode dual-number) rollout: the final (x, v, w) and their
        directional derivatives along (dx0, dv0, dw0, dtheta). Windows and contact lists as in
        `run`; tangent histories are carried by key like the histories."""
        n = self.n
        theta = tuple(float(t) for t in theta)
        cast = lambda a: torch.as_tensor(a, device=self.device).to(self.dtype).reshape(n, 3).contiguous()
        x, v, w = cast(x0), cast(v0), cast(w0)
        xd, vd, wd = cast(dx0), cast(dv0), cast(dw0)
        td = (C.c_double * 3)(*[float(a) for a in dtheta])
        prev_keys = prev_xi = prev_xid = None
        k, rate = 0, None
        while k < steps:
            K = self._window_len(k, steps)
            skin = self._skin(v, K) if rate is None else max(self.skin_min, 2.5 * rate * K)
            while True:
                cont, keys, idx, valid, start = self._start(x, v, w, skin, prev_keys, prev_xi)
                nc = int(cont.shape[0])
                S = start.numel()
                st = torch.empty(2 * S, dtype=self.dtype, device=self.device)
                tg = torch.empty(2 * S, dtype=self.dtype, device=self.device)
                st[:S] = start
                tg[:S] = self._state(xd, vd, wd, self._carry(prev_xid, idx, valid, nc))
                M = self._model(cont, theta)
                self._check(self.api.fn["hz_jvp"](self.code, C.byref(M), int(K), _ptr(st), _ptr(tg), td,
                                                  _ptr(self._work(nc)), self._stream()), "hz_jvp")
                disp = float((st[S:S + 3 * n] - start[:3 * n]).reshape(n, 3).norm(dim=1).max()) if n else 0.0
                if disp <= 0.5 * skin:
                    break
                skin *= 2.0
                self.stats["reruns"] += 1
            rate = disp / K
            x, v, w, prev_xi = self._split(st[S:], nc)
            xd, vd, wd, prev_xid = self._split(tg[S:], nc)
            prev_keys = keys
            k += K
        return (x.clone(), v.clone(), w.clone()), (xd.clone(), vd.clone(), wd.clone())

    def active_sets(self, x0, v0, w0, theta, steps):
        """The touching contacts of every substep of a rollout (the branches its force law takes):
        a list of `steps` sorted int64 key tensors (key i (n + nplane) + j of a sphere pair i < j,
        i (n + nplane) + n + p of sphere i on plane p), each from the state the substep starts from:
        overlap r_i + r_j - |x_i - x_j| > 0 (and |x_i - x_j| >= 1e-12) for a pair,
        r_i - (x_i - p0) . n > 0 for a plane. Two rollouts with equal lists take the same branches
        everywhere, so central differences between them see no contact onset or release."""
        n = self.n
        theta = tuple(float(t) for t in theta)
        x, v, w = (torch.as_tensor(a, device=self.device).to(self.dtype).reshape(n, 3).contiguous()
                   for a in (x0, v0, w0))
        pl = self.planes.view(-1, 6)
        prev_keys = prev_xi = None
        out = []
        k, rate = 0, None
        while k < steps:
            K = self._window_len(k, steps)
            skin = self._skin(v, K) if rate is None else max(self.skin_min, 2.5 * rate * K)
            while True:
                cont, keys, idx, valid, start = self._start(x, v, w, skin, prev_keys, prev_xi)
                traj = self.forward_window(start, cont, theta, K, store=True)
                S = start.numel()
                end = traj[K * S:(K + 1) * S]
                disp = float((end[:3 * n] - start[:3 * n]).reshape(n, 3).norm(dim=1).max()) if n else 0.0
                if disp <= 0.5 * skin:
                    break
                skin *= 2.0
            rate = disp / K
            i, j = cont[:, 0].long(), cont[:, 1].long()
            pair = j >= 0
            for q in range(K):
                xq = traj[q * S:q * S + 3 * n].view(n, 3)
                delta = torch.empty(i.shape, dtype=self.dtype, device=self.device)
                if bool(pair.any()):
                    d = (xq[i[pair]] - xq[j[pair]]).norm(dim=1)
                    delta[pair] = torch.where(d >= 1e-12, self.r[i[pair]] + self.r[j[pair]] - d,
                                              torch.zeros_like(d))
                if bool((~pair).any()):
                    p = -1 - j[~pair]
                    dist = ((xq[i[~pair]] - pl[p, :3]) * pl[p, 3:]).sum(dim=1)
                    delta[~pair] = self.r[i[~pair]] - dist
                out.append(torch.sort(keys[delta > 0]).values)
            x, v, w, prev_xi = self._split(end, int(cont.shape[0]))
            prev_keys = keys
            k += K
        return out

    @staticmethod
    def same_branches(a, b):
        """True when two active_sets lists are equal substep by substep."""
        return len(a) == len(b) and all(p.numel() == q.numel() and bool(torch.equal(p, q)) for p, q in zip(a, b))

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
