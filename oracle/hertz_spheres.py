"""CPU restatement of the explicit Hertz-Mindlin sphere substep, with forward-mode dual numbers.

TEST INFRASTRUCTURE ONLY: this module is the checker of the differentiable Hertz rollout
(`peclet.dem.adjoint`); only tests and the benchmark's baseline leg import it.

The substep follows the reference's Hertz engine:
- pair law (src/solver_hertz.hpp:88-144): overlap d = r_i + r_j - |x_i - x_j|, normal n from j to i,
  lever arms r_A = -n (r_i - d/2), r_B = n (r_j - d/2), relative contact velocity
  v_r = v_i + w_i x r_A - (v_j + w_j x r_B); Hertz stiffnesses from E* = 1 / (2 (1 - nu^2) / E),
  G* = 1 / (4 (2 - nu)(1 + nu) / E), R* = r_i r_j / (r_i + r_j), m* = 1 / (1/m_i + 1/m_j);
  damping from beta(e) = ln e / sqrt(ln^2 e + pi^2) (e <= 0 -> -1, e >= 1 -> 0); the Mindlin
  history xi grows by v_t dt, is projected onto the tangent plane, and is rescaled when the
  tangential force exceeds the Coulomb cone mu |f_s|;
- sphere-plane contacts: the same law against a plane at rest (point p0, unit normal n), with
  R* = r_i and m* = m_i (the wall branch of src/solver_hertz.hpp:300-372);
- integration (src/solver_hertz.hpp:374-425): v' = v + (F/m + g) dt, w' = w + T/I dt,
  x' = x + v' dt.
All pairs of one scene are evaluated every substep (no candidate list); separated pairs have a
zero force and a cleared history, so this equals any list that contains every touching pair.

`Dual` carries tangents along the last axis, so `rollout` with dual inputs is the forward-mode
(tangent-linear) run used to check adjoint gradients.
"""
from __future__ import annotations

import numpy as np

PI2 = 9.8696044  # the constant of the damping ratio, as the engine writes it


class Dual:
    """Value array `v` with tangents `d` (shape v.shape + (T,))."""

    __slots__ = ("v", "d")
    __array_ufunc__ = None  # numpy arrays defer to Dual's reflected operators

    def __init__(self, v, d):
        self.v = np.asarray(v, dtype=np.float64)
        self.d = np.asarray(d, dtype=np.float64)

    @staticmethod
    def const(v, nt):
        v = np.asarray(v, dtype=np.float64)
        return Dual(v, np.zeros(v.shape + (nt,)))

    def _wrap(self, o):
        return o if isinstance(o, Dual) else Dual.const(o, self.d.shape[-1])

    def __add__(self, o):
        o = self._wrap(o)
        return Dual(self.v + o.v, self.d + o.d)

    __radd__ = __add__

    def __sub__(self, o):
        o = self._wrap(o)
        return Dual(self.v - o.v, self.d - o.d)

    def __rsub__(self, o):
        return self._wrap(o) - self

    def __neg__(self):
        return Dual(-self.v, -self.d)

    def __mul__(self, o):
        o = self._wrap(o)
        return Dual(self.v * o.v, self.d * o.v[..., None] + self.v[..., None] * o.d)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = self._wrap(o)
        q = self.v / o.v
        return Dual(q, (self.d - q[..., None] * o.d) / o.v[..., None])

    def __rtruediv__(self, o):
        return self._wrap(o) / self

    def __getitem__(self, idx):
        return Dual(self.v[idx], self.d[idx])


def _nt(*xs):
    for x in xs:
        if isinstance(x, Dual):
            return x.d.shape[-1]
    return None


def sqrt(a):
    if not isinstance(a, Dual):
        return np.sqrt(a)
    s = np.sqrt(a.v)
    g = np.where(s > 0, 0.5 / np.where(s > 0, s, 1.0), 0.0)
    return Dual(s, g[..., None] * a.d)


def log(a):
    if not isinstance(a, Dual):
        return np.log(a)
    return Dual(np.log(a.v), a.d / a.v[..., None])


def val(a):
    return a.v if isinstance(a, Dual) else np.asarray(a, dtype=np.float64)


def where(mask, a, b):
    nt = _nt(a, b)
    if nt is None:
        return np.where(mask, a, b)
    a = a if isinstance(a, Dual) else Dual.const(a, nt)
    b = b if isinstance(b, Dual) else Dual.const(b, nt)
    shape = np.broadcast_shapes(mask.shape, a.v.shape, b.v.shape)
    av, bv = np.broadcast_to(a.v, shape), np.broadcast_to(b.v, shape)
    ad, bd = np.broadcast_to(a.d, shape + (nt,)), np.broadcast_to(b.d, shape + (nt,))
    return Dual(np.where(mask, av, bv), np.where(mask[..., None], ad, bd))


# ---- 3-vectors as lists of three arrays (or Duals) ----
def dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def cross(a, b):
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def beta_d(e):
    """src/solver_hertz.hpp:94-98 (the damping ratio's beta of the restitution)."""
    ev = float(val(e))
    if ev <= 0:
        return -1.0
    if ev >= 1:
        return 0.0
    le = log(e)
    return le / sqrt(le * le + PI2)


def stars(E, nu):
    eS = 1.0 / ((1.0 - nu * nu) / E + (1.0 - nu * nu) / E)
    b = (2.0 - nu) * (1.0 + nu)
    gS = 1.0 / (2.0 * b / E + 2.0 * b / E)
    return eS, gS


def hertz_force(delta, nh, vr, rS, mS, eS, gS, e, mu, dt, xi):
    """Contact force and new history (src/solver_hertz.hpp:99-144), elementwise over contacts."""
    sq = sqrt(rS * delta)
    sn = 2.0 * eS * sq
    st = 8.0 * gS * sq
    kn = (4.0 / 3.0) * eS * sq
    bd = beta_d(e)
    etaN = -2.0 * 0.9128709 * bd * sqrt(sn * mS)
    etaT = -2.0 * 0.9128709 * bd * sqrt(st * mS)
    vn = dot(vr, nh)
    fs = kn * delta
    fn = fs - etaN * vn
    vt = [vr[a] - nh[a] * vn for a in range(3)]
    xi = [xi[a] + vt[a] * dt for a in range(3)]
    xn = dot(xi, nh)
    xi = [xi[a] - nh[a] * xn for a in range(3)]
    ft = [xi[a] * (-st) + vt[a] * (-etaT) for a in range(3)]
    fl = sqrt(dot(ft, ft))
    fm = mu * where(val(fs) < 0, -fs, fs) if isinstance(fs, Dual) else mu * np.abs(fs)
    slip = val(fl) > val(fm)
    safe = where(val(fl) > 1e-20, fl, 1.0)
    s = where(val(fl) > 1e-20, fm / safe, 0.0)
    ft_c = [ft[a] * s for a in range(3)]
    st_safe = where(val(st) > 1e-20, st, 1.0)
    xi_c = [(ft_c[a] + vt[a] * etaT) * (-1.0 / st_safe) for a in range(3)]
    xi_new = [where(slip & (val(st) > 1e-20), xi_c[a], xi[a]) for a in range(3)]
    ft_new = [where(slip, ft_c[a], ft[a]) for a in range(3)]
    return [nh[a] * fn + ft_new[a] for a in range(3)], xi_new


def _rows(a, idx):
    """Rows idx of an (n, 3) array or Dual as a list of three columns."""
    return [a[idx, k] for k in range(3)]


def _scatter(n, idx, vals, nt):
    """Sum of vals (list of three columns) into n rows at idx (np.add.at, values and tangents)."""
    if nt is None:
        out = np.zeros((n, 3))
        for k in range(3):
            np.add.at(out[:, k], idx, vals[k])
        return out
    v, d = np.zeros((n, 3)), np.zeros((n, 3, nt))
    for k in range(3):
        c = vals[k] if isinstance(vals[k], Dual) else Dual.const(vals[k], nt)
        c = Dual(np.broadcast_to(c.v, idx.shape), np.broadcast_to(c.d, idx.shape + (nt,)))
        np.add.at(v[:, k], idx, c.v)
        np.add.at(d[:, k], idx, c.d)
    return Dual(v, d)


def _stack(cols):
    if isinstance(cols[0], Dual):
        return Dual(np.stack([c.v for c in cols], -1), np.stack([c.d for c in cols], -2))
    return np.stack(cols, -1)


def _mask_rows(active, cols, nt):
    return [where(active, c, 0.0) for c in cols]


class Model:
    """Spheres (radius r, mass m, scalar inertia I) in scenes [first[s], first[s+1]), planes
    (p0, n), Poisson ratio nu, time step dt, gravity g."""

    def __init__(self, r, m, I, first, planes, nu, dt, g):
        self.r = np.asarray(r, np.float64)
        self.m = np.asarray(m, np.float64)
        self.I = np.asarray(I, np.float64)
        self.n = self.r.size
        self.planes = np.asarray(planes, np.float64).reshape(-1, 6)
        self.nu, self.dt, self.g = float(nu), float(dt), np.asarray(g, np.float64)
        pi, pj = [], []
        for s in range(len(first) - 1):
            a, b = int(first[s]), int(first[s + 1])
            ii, jj = np.triu_indices(b - a, 1)
            pi.append(ii + a)
            pj.append(jj + a)
        self.pi = np.concatenate(pi) if pi else np.zeros(0, int)
        self.pj = np.concatenate(pj) if pj else np.zeros(0, int)

    def substep(self, x, v, w, xiP, xiW, E, e, mu):
        """One substep; x, v, w (n, 3), xiP (npairs, 3) over all scene pairs, xiW (n, nplane, 3).
        Any argument may be a Dual (all Duals share the tangent count)."""
        nt = _nt(x, v, w, xiP, xiW, E, e, mu)
        n, dt = self.n, self.dt
        eS, gS = stars(E, self.nu)
        F = T = None
        # sphere pairs
        i, j = self.pi, self.pj
        if i.size:
            xi_, xj_ = _rows(x, i), _rows(x, j)
            dx = [xi_[k] - xj_[k] for k in range(3)]
            dd = sqrt(dot(dx, dx))
            ri, rj = self.r[i], self.r[j]
            delta = (ri + rj) - dd
            active = (val(delta) > 0) & (val(dd) >= 1e-12)
            dd_s = where(active, dd, 1.0)
            delta_s = where(active, delta, 1e-30)
            nh = [dx[k] / dd_s for k in range(3)]
            rA = [nh[k] * (-(ri - 0.5 * delta_s)) for k in range(3)]
            rB = [nh[k] * (rj - 0.5 * delta_s) for k in range(3)]
            vi, vj, wi, wj = _rows(v, i), _rows(v, j), _rows(w, i), _rows(w, j)
            ca, cb = cross(wi, rA), cross(wj, rB)
            vr = [vi[k] + ca[k] - (vj[k] + cb[k]) for k in range(3)]
            rS = ri * rj / (ri + rj)
            mS = 1.0 / (1.0 / self.m[i] + 1.0 / self.m[j])
            f, xin = hertz_force(delta_s, nh, vr, rS, mS, eS, gS, e, mu, dt, [xiP[:, k] for k in range(3)])
            f = _mask_rows(active, f, nt)
            xin = _mask_rows(active, xin, nt)
            ti = cross(rA, f)
            tj = cross(rB, [-c for c in f])
            ti, tj = _mask_rows(active, ti, nt), _mask_rows(active, tj, nt)
            F = _scatter(n, i, f, nt) + _scatter(n, j, [-c for c in f], nt)
            T = _scatter(n, i, ti, nt) + _scatter(n, j, tj, nt)
            xiP = _stack(xin)
        # planes: per sphere, in plane order
        xiW_new = []
        for k in range(self.planes.shape[0]):
            p0, nn = self.planes[k, :3], self.planes[k, 3:]
            xc = [x[:, a] for a in range(3)]
            dist = (xc[0] - p0[0]) * nn[0] + (xc[1] - p0[1]) * nn[1] + (xc[2] - p0[2]) * nn[2]
            delta = self.r - dist
            active = val(delta) > 0
            delta_s = where(active, delta, 1e-30)
            nh = [np.full(n, nn[a]) for a in range(3)]
            rA = [nh[a] * (-(self.r - 0.5 * delta_s)) for a in range(3)]
            wc = [w[:, a] for a in range(3)]
            cw = cross(wc, rA)
            vr = [v[:, a] + cw[a] for a in range(3)]
            f, xin = hertz_force(delta_s, nh, vr, self.r, self.m, eS, gS, e, mu, dt, [xiW[:, k, a] for a in range(3)])
            f = _mask_rows(active, f, nt)
            xin = _mask_rows(active, xin, nt)
            t = _mask_rows(active, cross(rA, f), nt)
            Fk, Tk = _stack(f), _stack(t)
            F = Fk if F is None else F + Fk
            T = Tk if T is None else T + Tk
            xiW_new.append(_stack(xin))
        if F is None:
            F, T = np.zeros((n, 3)), np.zeros((n, 3))
        if xiW_new:
            if isinstance(xiW_new[0], Dual):
                xiW = Dual(np.stack([q.v for q in xiW_new], 1), np.stack([q.d for q in xiW_new], 1))
            else:
                xiW = np.stack(xiW_new, 1)
        inv_m, inv_I = (1.0 / self.m)[:, None], (1.0 / self.I)[:, None]
        v = v + (F * inv_m + self.g[None, :]) * dt
        w = w + T * inv_I * dt
        x = x + v * dt
        return x, v, w, xiP, xiW

    def rollout(self, x, v, w, E, e, mu, steps):
        """`steps` substeps from rest histories; returns the final (x, v, w)."""
        nt = _nt(x, v, w, E, e, mu)
        zP = np.zeros((self.pi.size, 3))
        zW = np.zeros((self.n, self.planes.shape[0], 3))
        xiP = zP if nt is None else Dual.const(zP, nt)
        xiW = zW if nt is None else Dual.const(zW, nt)
        if nt is not None:
            x, v, w = (a if isinstance(a, Dual) else Dual.const(a, nt) for a in (x, v, w))
        for _ in range(steps):
            x, v, w, xiP, xiW = self.substep(x, v, w, xiP, xiW, E, e, mu)
        return x, v, w


def jvp(model, x0, v0, w0, theta, tangents, steps):
    """Directional derivatives of the final state: tangents = list of dicts with optional keys
    'x', 'v', 'w' ((n, 3) arrays) and 'theta' (3,) for (E, e, mu). Returns (x, v, w) Duals."""
    nt = len(tangents)
    n = model.n

    def seed(base, key, shape):
        d = np.zeros(shape + (nt,))
        for t, tan in enumerate(tangents):
            if key in tan:
                d[..., t] = tan[key]
        return Dual(base, d)

    x = seed(x0, "x", (n, 3))
    v = seed(v0, "v", (n, 3))
    w = seed(w0, "w", (n, 3))
    th = [Dual(np.float64(theta[k]), np.array([tan.get("theta", np.zeros(3))[k] for tan in tangents]))
          for k in range(3)]
    return model.rollout(x, v, w, th[0], th[1], th[2], steps)
