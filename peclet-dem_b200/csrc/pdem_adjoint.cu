// Forward, adjoint and tangent-linear runs of the explicit Hertz-Mindlin substep for spheres, for
// differentiable calibration: gradients of a loss on the final state with respect to Young's
// modulus E, the restitution e, the friction mu and the initial state.
//
// The force law is the Hertz engine's (src/solver_hertz.hpp:88-144 for sphere pairs, the same law
// against a wall at rest for the planes, src/solver_hertz.hpp:300-372), the integration its
// symplectic kick-drift (src/solver_hertz.hpp:374-425) without orientation update:
//   per contact with overlap d > 0 (pair: d = r_i + r_j - |x_i - x_j|, normal from j to i; plane:
//   d = r_i - (x_i - p0).n): force f(d, n, v_rel, xi; E, e, mu) and the new Mindlin history xi',
//   torques r_A x f on i (and r_B x (-f) on j); then v' = v + (F / m + g) dt, w' = w + T / I dt,
//   x' = x + v' dt.
// Contacts are candidates (sphere pairs of one scene and sphere-plane couples within a skin) built
// by the caller at each window start; they stay fixed over the window's substeps.
//
// State of a substep (one contiguous block): x, v, w (3 n each), then the history of every
// contact (3 each). The forward stores every substep of a window (or ping-pongs two states); the
// backward walks the stored window in reverse.
//
// Adjoint of one substep, given the adjoint of S_{k+1}: the integration is linear and reversed by
// hand; each contact's law is re-evaluated from the stored state with its intermediates kept in
// registers (the same arithmetic as the forward, so the active set and the stick/slip branch are
// the forward's) and reversed statement by statement. A second mode takes the contact's local
// Jacobian with forward-mode dual numbers through the engine's own hertzForce instead; it is the
// cross-check of the hand reversal. The tangent-linear run carries one dual tangent through the
// whole rollout. Accumulation into bodies and parameters uses atomics, so sums come in an
// unspecified order (forward forces too: the forward is deterministic up to summation order).
#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include <cub/cub.cuh>

#include "../../include/pdem.h"
#include "pdem_hertz.cuh"

namespace pdem {
void setLastError(const std::string& msg);  // pdem_capi.cu
}

namespace {

using pdem::add;
using pdem::cross;
using pdem::dot;
using pdem::mul;
using pdem::sub;
using pdem::V3;
using std::fabs;  // the plain overloads stay visible beside the dual-number ones below
using std::log;
using std::sqrt;

// ---------------------------------------------------------------------------------------------
// forward-mode dual number over scalar S with N tangents
template <class S, int N>
struct Dn {
  S v;
  S d[N];
  __device__ Dn() : v(0) {
#pragma unroll
    for (int k = 0; k < N; ++k)
      d[k] = 0;
  }
  __device__ Dn(double x) : v(S(x)) {  // NOLINT: literals and R(2)-style casts of the shared law
#pragma unroll
    for (int k = 0; k < N; ++k)
      d[k] = 0;
  }
};
template <class S, int N>
__device__ Dn<S, N> operator+(const Dn<S, N>& a, const Dn<S, N>& b) {
  Dn<S, N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <class S, int N>
__device__ Dn<S, N> operator-(const Dn<S, N>& a, const Dn<S, N>& b) {
  Dn<S, N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <class S, int N>
__device__ Dn<S, N> operator-(const Dn<S, N>& a) {
  Dn<S, N> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = -a.d[k];
  return r;
}
template <class S, int N>
__device__ Dn<S, N> operator*(const Dn<S, N>& a, const Dn<S, N>& b) {
  Dn<S, N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <class S, int N>
__device__ Dn<S, N> operator/(const Dn<S, N>& a, const Dn<S, N>& b) {
  Dn<S, N> r;
  r.v = a.v / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
template <class S, int N>
__device__ bool operator<(const Dn<S, N>& a, const Dn<S, N>& b) { return a.v < b.v; }
template <class S, int N>
__device__ bool operator>(const Dn<S, N>& a, const Dn<S, N>& b) { return a.v > b.v; }
template <class S, int N>
__device__ bool operator<=(const Dn<S, N>& a, const Dn<S, N>& b) { return a.v <= b.v; }
template <class S, int N>
__device__ bool operator>=(const Dn<S, N>& a, const Dn<S, N>& b) { return a.v >= b.v; }
template <class S, int N>
__device__ Dn<S, N> sqrt(const Dn<S, N>& a) {
  Dn<S, N> r;
  r.v = ::sqrt(a.v);
  const S g = r.v > S(0) ? S(0.5) / r.v : S(0);
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = g * a.d[k];
  return r;
}
template <class S, int N>
__device__ Dn<S, N> log(const Dn<S, N>& a) {
  Dn<S, N> r;
  r.v = ::log(a.v);
#pragma unroll
  for (int k = 0; k < N; ++k)
    r.d[k] = a.d[k] / a.v;
  return r;
}
template <class S, int N>
__device__ Dn<S, N> fabs(const Dn<S, N>& a) {
  return a.v < S(0) ? -a : a;
}

// ---------------------------------------------------------------------------------------------
template <class R>
struct Model {
  int n, nc, nplane;
  const int* cont;  // [nc] (i, j): j >= 0 the sphere j (> i); j < 0 the plane -j - 1
  const R *planes, *r, *im, *iI;  // radius, inverse mass, inverse (scalar) moment of inertia
  R E, e, mu, dt, g[3];
  double nu;
};
template <class R>
struct StateView {
  R *x, *v, *w, *xi;
};
inline size_t stateSize(long n, long nc) { return (size_t)(9 * n + 3 * nc); }
template <class R>
StateView<R> view(R* base, long n) {
  return StateView<R>{base, base + 3 * n, base + 6 * n, base + 9 * n};
}
template <class R>
__device__ V3<R> ld3(const R* p, long i) {
  return V3<R>{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
}
template <class R>
__device__ void st3(R* p, long i, V3<R> a) {
  p[3 * i] = a.x, p[3 * i + 1] = a.y, p[3 * i + 2] = a.z;
}
template <class R>
__device__ void atomicAdd3(R* p, long i, V3<R> a) {
  atomicAdd(&p[3 * i], a.x);
  atomicAdd(&p[3 * i + 1], a.y);
  atomicAdd(&p[3 * i + 2], a.z);
}

// material stars of one material against itself (hertzStars with E_i = E_j, nu_i = nu_j):
// E* = E / (2 (1 - nu^2)), G* = E / (4 (2 - nu)(1 + nu))
template <class T>
__device__ void stars(T E, double nu, T& eS, T& gS) {
  const T one(1.0), two(2.0), a(1.0 - nu * nu), b((2.0 - nu) * (1.0 + nu));
  eS = one / (a / E + a / E);
  gS = one / (two * b / E + two * b / E);
}

// ---------------------------------------------------------------------------------------------
// One contact with its intermediates: the engine's hertzForce statement by statement (same
// operations in the same order), kept for the reversal.
template <class R>
struct Contact {
  int i, j, k;  // spheres i, j (j < 0 for a plane k)
  bool active, slip, sOk, stOk;
  R ri, rj, rS, mS, dd, delta, eS, gS, sq, sn, st, kn, bd, qN, qT, etaN, etaT, vn, fs, fn, p, fl, fm, s;
  V3<R> dx, nh, rA, rB, wi, wj, vr, vt, xi1, xi2, ft0, ft, f, xi3;
};
template <class R>
constexpr R kEtaC() {
  return R(-2) * R(0.9128709);
}

// contactPrimal's activity test alone (the same operations): touching spheres, or a sphere
// overlapping its plane
template <class R>
__device__ bool contactActive(const Model<R>& M, long c, const StateView<R>& s) {
  const int i = M.cont[2 * c], j = M.cont[2 * c + 1];
  const R ri = M.r[i];
  if (j >= 0) {
    const R rj = M.r[j];
    const V3<R> dx = sub(ld3(s.x, i), ld3(s.x, j));
    const R d2 = dot(dx, dx), rr = ri + rj;
    if (d2 > rr * rr * R(1.0001))
      return false;
    const R dd = sqrt(d2);
    const R delta = rr - dd;
    return !(delta <= R(0) || dd < R(1e-12));
  }
  const R* pl = M.planes + 6 * (-j - 1);
  const V3<R> nh{pl[3], pl[4], pl[5]};
  const R delta = ri - dot(sub(ld3(s.x, i), V3<R>{pl[0], pl[1], pl[2]}), nh);
  return !(delta <= R(0));
}

template <class R>
__device__ void contactPrimal(const Model<R>& M, long c, const StateView<R>& s, Contact<R>& C) {
  C.i = M.cont[2 * c];
  C.j = M.cont[2 * c + 1];
  C.k = C.j < 0 ? -C.j - 1 : -1;
  const int i = C.i;
  C.ri = M.r[i];
  // the activity test first, from positions and radii only (most candidates are apart)
  if (C.j >= 0) {
    const int j = C.j;
    C.rj = M.r[j];
    C.dx = sub(ld3(s.x, i), ld3(s.x, j));
    const R d2 = dot(C.dx, C.dx), rr = C.ri + C.rj;
    if (d2 > rr * rr * R(1.0001)) {  // certainly apart: sqrt(d2) > rr whatever the rounding
      C.active = false;
      return;
    }
    C.dd = sqrt(d2);
    C.delta = rr - C.dd;
    C.active = !(C.delta <= R(0) || C.dd < R(1e-12));
    if (!C.active)
      return;
    C.wi = ld3(s.w, i);
    C.nh = mul(C.dx, R(1) / C.dd);
    C.rA = mul(C.nh, -(C.ri - R(0.5) * C.delta));
    C.rB = mul(C.nh, (C.rj - R(0.5) * C.delta));
    C.wj = ld3(s.w, j);
    C.vr = sub(add(ld3(s.v, i), cross(C.wi, C.rA)), add(ld3(s.v, j), cross(C.wj, C.rB)));
    C.rS = C.ri * C.rj / (C.ri + C.rj);
    const R imS = M.im[i] + M.im[j];
    C.mS = imS > R(0) ? R(1) / imS : R(0);
  } else {
    const R* pl = M.planes + 6 * C.k;
    C.nh = V3<R>{pl[3], pl[4], pl[5]};
    C.delta = C.ri - dot(sub(ld3(s.x, i), V3<R>{pl[0], pl[1], pl[2]}), C.nh);
    C.active = !(C.delta <= R(0));
    if (!C.active)
      return;
    C.wi = ld3(s.w, i);
    C.rA = mul(C.nh, -(C.ri - R(0.5) * C.delta));
    C.vr = add(ld3(s.v, i), cross(C.wi, C.rA));
    C.rS = C.ri;
    C.mS = M.im[i] > R(0) ? R(1) / M.im[i] : R(0);
  }
  const V3<R> xi0 = ld3(s.xi, c);
  stars(M.E, M.nu, C.eS, C.gS);
  C.sq = sqrt(C.rS * C.delta);
  C.sn = R(2) * C.eS * C.sq;
  C.st = R(8) * C.gS * C.sq;
  C.kn = (R(4) / R(3)) * C.eS * C.sq;
  C.bd = pdem::hertzBetaD(M.e);
  C.qN = sqrt(C.sn * C.mS);
  C.qT = sqrt(C.st * C.mS);
  C.etaN = kEtaC<R>() * C.bd * C.qN;
  C.etaT = kEtaC<R>() * C.bd * C.qT;
  C.vn = dot(C.vr, C.nh);
  C.fs = C.kn * C.delta;
  C.fn = C.fs - C.etaN * C.vn;
  C.vt = sub(C.vr, mul(C.nh, C.vn));
  C.xi1 = add(xi0, mul(C.vt, M.dt));
  C.p = dot(C.xi1, C.nh);
  C.xi2 = sub(C.xi1, mul(C.nh, C.p));
  C.ft0 = add(mul(C.xi2, -C.st), mul(C.vt, -C.etaT));
  C.fl = sqrt(dot(C.ft0, C.ft0));
  C.fm = M.mu * fabs(C.fs);
  C.slip = C.fl > C.fm;
  C.ft = C.ft0;
  C.xi3 = C.xi2;
  if (C.slip) {
    C.sOk = C.fl > R(1e-20);
    C.s = C.sOk ? C.fm / C.fl : R(0);
    C.ft = mul(C.ft0, C.s);
    C.stOk = C.st > R(1e-20);
    if (C.stOk)
      C.xi3 = mul(add(C.ft, mul(C.vt, C.etaT)), R(-1) / C.st);
  }
  C.f = add(mul(C.nh, C.fn), C.ft);
}

// Reverse of one active contact. In: fb (adjoint of f, the force on i), tAb, tBb (adjoints of
// the torques on i and j), xib (adjoint of the new history). Out: adjoints of x_i, x_j, v_i, v_j,
// w_i, w_j (pair: the j parts are the negated dx / dv ones), of the old history, and of E, e, mu.
template <class R>
struct ContactBar {
  V3<R> dx, dv, wi, wj, xi;
  R E, e, mu;
};
template <class R>
__device__ ContactBar<R> contactReverse(const Model<R>& M, const Contact<R>& C, V3<R> fb, V3<R> tAb, V3<R> tBb,
                                        V3<R> xi3b) {
  const V3<R> zero{R(0), R(0), R(0)};
  ContactBar<R> B;
  // torques: tA = rA x f, tB = rB x (-f)
  V3<R> rAb = cross(C.f, tAb);
  fb = add(fb, cross(tAb, C.rA));
  V3<R> rBb = zero;
  if (C.j >= 0) {
    rBb = cross(tBb, C.f);
    fb = add(fb, cross(C.rB, tBb));
  }
  // f = nh fn + ft
  V3<R> nhb = mul(fb, C.fn);
  const R fnb = dot(C.nh, fb);
  V3<R> ftb = fb, ft0b = zero, xi2b = zero, vtb = zero;
  R stb = 0, etaTb = 0, fmb = 0, flb = 0;
  if (C.slip) {
    if (C.stOk) {  // xi3 = (ft + vt etaT) (-1 / st)
      const R inv = R(-1) / C.st;
      ftb = add(ftb, mul(xi3b, inv));
      etaTb += dot(xi3b, C.vt) * inv;
      vtb = add(vtb, mul(xi3b, C.etaT * inv));
      stb += -dot(xi3b, C.xi3) / C.st;
    } else {
      xi2b = add(xi2b, xi3b);
    }
    // ft = ft0 s, s = fm / fl
    ft0b = add(ft0b, mul(ftb, C.s));
    const R sb = dot(C.ft0, ftb);
    if (C.sOk) {
      fmb += sb / C.fl;
      flb += -sb * C.s / C.fl;
    }
  } else {
    ft0b = add(ft0b, ftb);
    xi2b = add(xi2b, xi3b);
  }
  // fm = mu |fs|
  const R mub = fabs(C.fs) * fmb;
  R fsb = (C.fs >= R(0) ? M.mu : -M.mu) * fmb;
  // fl = |ft0|
  if (C.fl > R(0))
    ft0b = add(ft0b, mul(C.ft0, flb / C.fl));
  // ft0 = xi2 (-st) + vt (-etaT)
  stb += -dot(C.xi2, ft0b);
  xi2b = add(xi2b, mul(ft0b, -C.st));
  etaTb += -dot(C.vt, ft0b);
  vtb = add(vtb, mul(ft0b, -C.etaT));
  // xi2 = xi1 - nh p, p = xi1 . nh
  const R pb = -dot(C.nh, xi2b);
  const V3<R> xi1b = add(xi2b, mul(C.nh, pb));
  nhb = add(nhb, add(mul(xi2b, -C.p), mul(C.xi1, pb)));
  // xi1 = xi0 + vt dt
  B.xi = xi1b;
  vtb = add(vtb, mul(xi1b, M.dt));
  // vt = vr - nh vn
  V3<R> vrb = vtb;
  nhb = add(nhb, mul(vtb, -C.vn));
  R vnb = -dot(C.nh, vtb);
  // fn = fs - etaN vn
  fsb += fnb;
  const R etaNb = -C.vn * fnb;
  vnb += -C.etaN * fnb;
  // fs = kn delta
  const R knb = C.delta * fsb;
  R deltab = C.kn * fsb;
  // vn = vr . nh
  vrb = add(vrb, mul(C.nh, vnb));
  nhb = add(nhb, mul(C.vr, vnb));
  // etaN = c bd qN, etaT = c bd qT, q = sqrt(s mS)
  const R bdb = kEtaC<R>() * (C.qT * etaTb + C.qN * etaNb);
  R snb = 0;
  if (C.qT > R(0))
    stb += kEtaC<R>() * C.bd * etaTb * C.mS / (R(2) * C.qT);
  if (C.qN > R(0))
    snb += kEtaC<R>() * C.bd * etaNb * C.mS / (R(2) * C.qN);
  // bd = ln e / sqrt(ln^2 e + pi^2) on 0 < e < 1, constant outside
  B.e = 0;
  if (M.e > R(0) && M.e < R(1)) {
    const R le = log(M.e), den = le * le + R(9.8696044);
    B.e = bdb * R(9.8696044) / (den * sqrt(den)) / M.e;
  }
  // kn = (4/3) eS sq, st = 8 gS sq, sn = 2 eS sq
  const R eSb = (R(4) / R(3)) * C.sq * knb + R(2) * C.sq * snb;
  const R gSb = R(8) * C.sq * stb;
  const R sqb = (R(4) / R(3)) * C.eS * knb + R(8) * C.gS * stb + R(2) * C.eS * snb;
  // sq = sqrt(rS delta)
  if (C.sq > R(0))
    deltab += sqb * C.rS / (R(2) * C.sq);
  // eS, gS proportional to E
  B.E = (eSb * C.eS + gSb * C.gS) / M.E;
  B.mu = mub;
  if (C.j >= 0) {
    // vr = (v_i + wi x rA) - (v_j + wj x rB)
    B.dv = vrb;
    B.wi = cross(C.rA, vrb);
    rAb = add(rAb, cross(vrb, C.wi));
    B.wj = mul(cross(C.rB, vrb), R(-1));
    rBb = add(rBb, mul(cross(vrb, C.wj), R(-1)));
    // rA = nh (-(ri - delta / 2)), rB = nh (rj - delta / 2)
    nhb = add(nhb, mul(rAb, -(C.ri - R(0.5) * C.delta)));
    deltab += R(0.5) * dot(C.nh, rAb);
    nhb = add(nhb, mul(rBb, C.rj - R(0.5) * C.delta));
    deltab += R(-0.5) * dot(C.nh, rBb);
    // delta = ri + rj - dd; nh = dx / dd; dd = |dx|
    R ddb = -deltab;
    B.dx = mul(nhb, R(1) / C.dd);
    ddb += -dot(nhb, C.nh) / C.dd;
    B.dx = add(B.dx, mul(C.nh, ddb));
  } else {
    // vr = v + wi x rA; rA = n (-(ri - delta / 2)); delta = ri - (x - p0) . n
    B.dv = vrb;
    B.wi = cross(C.rA, vrb);
    rAb = add(rAb, cross(vrb, C.wi));
    deltab += R(0.5) * dot(C.nh, rAb);
    B.dx = mul(C.nh, -deltab);
    B.wj = zero;
  }
  return B;
}

// ---------------------------------------------------------------------------------------------
// the same contact through the engine's hertzForce on any scalar type T (plain, or dual numbers):
// in = x_i(3) x_j(3) v_i(3) v_j(3) w_i(3) w_j(3) xi(3) E e mu; out = f(3) T_i(3) T_j(3) xi'(3)
constexpr int kIn = 24, kOut = 12;
template <class T, class R>
__device__ bool contactLaw(const Model<R>& M, int i, int j, int k, const T* in, T* out) {
  const V3<T> xi_{in[0], in[1], in[2]}, xj{in[3], in[4], in[5]}, vi{in[6], in[7], in[8]}, vj{in[9], in[10], in[11]};
  const V3<T> wi{in[12], in[13], in[14]}, wj{in[15], in[16], in[17]};
  V3<T> h{in[18], in[19], in[20]};
  const T E = in[21], e = in[22], mu = in[23];
  T eS, gS;
  stars(E, M.nu, eS, gS);
  const R ri = M.r[i];
  if (j >= 0) {
    const R rj = M.r[j];
    const V3<T> dx = sub(xi_, xj);
    const T dd = sqrt(dot(dx, dx));
    const T delta = T(ri + rj) - dd;
    if (delta <= T(0.0) || dd < T(1e-12))
      return false;
    const V3<T> nh = mul(dx, T(1.0) / dd);
    const V3<T> rA = mul(nh, -(T(ri) - T(0.5) * delta));
    const V3<T> rB = mul(nh, T(rj) - T(0.5) * delta);
    const V3<T> vr = sub(add(vi, cross(wi, rA)), add(vj, cross(wj, rB)));
    const R imS = M.im[i] + M.im[j];
    const R mS = imS > R(0) ? R(1) / imS : R(0);
    const V3<T> f = pdem::hertzForce(delta, nh, vr, T(ri * rj / (ri + rj)), T(mS), eS, gS, e, mu, T(M.dt), h);
    const V3<T> ti = cross(rA, f), tj = cross(rB, mul(f, T(-1.0)));
    out[0] = f.x, out[1] = f.y, out[2] = f.z, out[3] = ti.x, out[4] = ti.y, out[5] = ti.z;
    out[6] = tj.x, out[7] = tj.y, out[8] = tj.z, out[9] = h.x, out[10] = h.y, out[11] = h.z;
    return true;
  }
  const R* pl = M.planes + 6 * k;
  const V3<T> n{T(pl[3]), T(pl[4]), T(pl[5])};
  const T delta = T(ri) - dot(sub(xi_, V3<T>{T(pl[0]), T(pl[1]), T(pl[2])}), n);
  if (delta <= T(0.0))
    return false;
  const V3<T> rA = mul(n, -(T(ri) - T(0.5) * delta));
  const V3<T> vr = add(vi, cross(wi, rA));
  const R mS = M.im[i] > R(0) ? R(1) / M.im[i] : R(0);
  const V3<T> f = pdem::hertzForce(delta, n, vr, T(ri), T(mS), eS, gS, e, mu, T(M.dt), h);
  const V3<T> t = cross(rA, f);
  out[0] = f.x, out[1] = f.y, out[2] = f.z, out[3] = t.x, out[4] = t.y, out[5] = t.z;
  out[6] = out[7] = out[8] = T(0.0);
  out[9] = h.x, out[10] = h.y, out[11] = h.z;
  return true;
}

// ---------------------------------------------------------------------------------------------
// forward: contact forces into F, T (atomics), new histories; then the kick-drift, which also
// clears F, T for the next substep (they are cleared once at the window start)
template <class R>
__global__ void kContacts(Model<R> M, StateView<R> s, StateView<R> t, R* F, R* T) {
  GRID_STRIDE(c, M.nc) {
    Contact<R> C;
    contactPrimal(M, c, s, C);
    if (!C.active) {
      st3(t.xi, c, V3<R>{R(0), R(0), R(0)});
      continue;
    }
    st3(t.xi, c, C.xi3);
    atomicAdd3(F, C.i, C.f);
    atomicAdd3(T, C.i, cross(C.rA, C.f));
    if (C.j >= 0) {
      atomicAdd3(F, C.j, mul(C.f, R(-1)));
      atomicAdd3(T, C.j, cross(C.rB, mul(C.f, R(-1))));
    }
  }
}
// one thread per component (coalesced, three times the threads of one per sphere); the
// arithmetic per component is the engine's
template <class R>
__global__ void kIntegrate(Model<R> M, StateView<R> s, StateView<R> t, R* F, R* T) {
  GRID_STRIDE(q, 3L * M.n) {
    const int qi = (int)q, i = qi / 3, a = qi - 3 * i;  // 32-bit: the divide is a multiply
    const R im = M.im[i], iI = M.iI[i];
    const R x = s.x[q], v = s.v[q], w = s.w[q], f = F[q], tq = T[q];
    const R ga = a == 0 ? M.g[0] : (a == 1 ? M.g[1] : M.g[2]);  // no dynamic index into the parameters
    const R v1 = v + (f * im + ga) * M.dt;
    t.v[q] = v1;
    t.w[q] = w + tq * iI * M.dt;
    t.x[q] = x + v1 * M.dt;
    F[q] = R(0);
    T[q] = R(0);
  }
}

// ---- adjoint ----
// b0.{x,v,w} = b1 carried back through x' = x + v' dt, v' = v + ..., w' = w + ...;
// Fb, Tb = adjoints of the substep's force and torque sums
template <class R>
__global__ void kIntegrateAdj(Model<R> M, StateView<R> b1, StateView<R> b0, R* Fb, R* Tb) {
  GRID_STRIDE(q, 3L * M.n) {
    const int i = (int)q / 3;
    const R im = M.im[i], iI = M.iI[i];
    const R xb = b1.x[q], vb = b1.v[q], wb = b1.w[q];
    const R vbt = vb + xb * M.dt;  // v' feeds x' = x + v' dt
    b0.x[q] = xb;
    b0.v[q] = vbt;
    b0.w[q] = wb;
    Fb[q] = vbt * im * M.dt;
    Tb[q] = wb * iI * M.dt;
  }
}
__device__ inline void flushParams(double* thetaB, double gE, double ge, double gmu) {
  for (int o = 16; o > 0; o >>= 1) {
    gE += __shfl_xor_sync(0xffffffffu, gE, o);
    ge += __shfl_xor_sync(0xffffffffu, ge, o);
    gmu += __shfl_xor_sync(0xffffffffu, gmu, o);
  }
  if ((threadIdx.x & 31) == 0 && (gE != 0 || ge != 0 || gmu != 0)) {
    atomicAdd(&thetaB[0], gE);
    atomicAdd(&thetaB[1], ge);
    atomicAdd(&thetaB[2], gmu);
  }
}
// contact adjoints (hand reversal), in two passes so that the few touching contacts do not set
// the occupancy of the many apart: the scan clears the history adjoint of every apart contact
// and lists the touching ones (count[slot]); the second pass reverses the listed contacts, its
// warps in lockstep so the parameter sums reduce with shuffles, and clears the other counter
// slot for the next substep's scan
template <class R>
__global__ void kContactsAdjScan(Model<R> M, StateView<R> s, StateView<R> b0, int* list, int* count) {
  GRID_STRIDE(c, M.nc) {
    if (contactActive(M, c, s))
      list[atomicAdd(count, 1)] = (int)c;
    else
      st3(b0.xi, c, V3<R>{R(0), R(0), R(0)});  // cleared history: no dependence on the old one
  }
}
template <class R>
__global__ void kContactsAdj(Model<R> M, StateView<R> s, StateView<R> b1, StateView<R> b0, const R* Fb,
                             const R* Tb, double* thetaB, const int* list, const int* count, int* nextCount) {
  double gE = 0, ge = 0, gmu = 0;
  const long na = *count;
  if ((blockIdx.x | threadIdx.x) == 0)
    *nextCount = 0;
  for (long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x - (threadIdx.x & 31); t0 < na;
       t0 += (long)gridDim.x * blockDim.x) {
    const long t = t0 + (threadIdx.x & 31);
    if (t < na) {
      const long c = list[t];
      Contact<R> C;
      contactPrimal(M, c, s, C);
      if (!C.active) {  // cannot happen (the scan ran the same test); kept for safety
        st3(b0.xi, c, V3<R>{R(0), R(0), R(0)});
      } else {
        const int i = C.i, j = C.j;
        V3<R> fb = ld3(Fb, i);
        V3<R> tBb{R(0), R(0), R(0)};
        if (j >= 0) {
          fb = sub(fb, ld3(Fb, j));  // f acts on i, -f on j
          tBb = ld3(Tb, j);
        }
        const ContactBar<R> B = contactReverse(M, C, fb, ld3(Tb, i), tBb, ld3(b1.xi, c));
        st3(b0.xi, c, B.xi);
        atomicAdd3(b0.x, i, B.dx);
        atomicAdd3(b0.v, i, B.dv);
        atomicAdd3(b0.w, i, B.wi);
        if (j >= 0) {
          atomicAdd3(b0.x, j, mul(B.dx, R(-1)));
          atomicAdd3(b0.v, j, mul(B.dv, R(-1)));
          atomicAdd3(b0.w, j, B.wj);
        }
        gE += B.E, ge += B.e, gmu += B.mu;
      }
    }
  }
  flushParams(thetaB, gE, ge, gmu);
}
// contact adjoints from the local Jacobian by dual numbers through hertzForce (the cross-check)
template <class R>
__global__ void kContactsAdjDual(Model<R> M, StateView<R> s, StateView<R> b1, StateView<R> b0, const R* Fb,
                                 const R* Tb, double* thetaB) {
  double gE = 0, ge = 0, gmu = 0;
  for (long c0 = (long)blockIdx.x * blockDim.x + threadIdx.x - (threadIdx.x & 31); c0 < M.nc;
       c0 += (long)gridDim.x * blockDim.x) {
    const long c = c0 + (threadIdx.x & 31);
    if (c < M.nc) {
      const int i = M.cont[2 * c], j = M.cont[2 * c + 1], k = j < 0 ? -j - 1 : -1;
      const int jj = j >= 0 ? j : i;  // a plane reads sphere i in the j slots (unused)
      Dn<R, kIn> in[kIn], out[kOut];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        in[a] = Dn<R, kIn>(s.x[3 * i + a]);
        in[3 + a] = Dn<R, kIn>(s.x[3 * jj + a]);
        in[6 + a] = Dn<R, kIn>(s.v[3 * i + a]);
        in[9 + a] = Dn<R, kIn>(s.v[3 * jj + a]);
        in[12 + a] = Dn<R, kIn>(s.w[3 * i + a]);
        in[15 + a] = Dn<R, kIn>(s.w[3 * jj + a]);
        in[18 + a] = Dn<R, kIn>(s.xi[3 * c + a]);
      }
      in[21] = Dn<R, kIn>(M.E), in[22] = Dn<R, kIn>(M.e), in[23] = Dn<R, kIn>(M.mu);
#pragma unroll
      for (int q = 0; q < kIn; ++q)
        in[q].d[q] = R(1);
      if (!contactLaw<Dn<R, kIn>, R>(M, i, j, k, in, out)) {
        st3(b0.xi, c, V3<R>{R(0), R(0), R(0)});
      } else {
        R yb[kOut];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          yb[a] = Fb[3 * i + a] - (j >= 0 ? Fb[3 * j + a] : R(0));
          yb[3 + a] = Tb[3 * i + a];
          yb[6 + a] = j >= 0 ? Tb[3 * j + a] : R(0);
          yb[9 + a] = b1.xi[3 * c + a];
        }
        R cb[kIn];
#pragma unroll
        for (int q = 0; q < kIn; ++q) {
          R acc = 0;
#pragma unroll
          for (int o = 0; o < kOut; ++o)
            acc += out[o].d[q] * yb[o];
          cb[q] = acc;
        }
        atomicAdd3(b0.x, i, V3<R>{cb[0], cb[1], cb[2]});
        atomicAdd3(b0.v, i, V3<R>{cb[6], cb[7], cb[8]});
        atomicAdd3(b0.w, i, V3<R>{cb[12], cb[13], cb[14]});
        if (j >= 0) {
          atomicAdd3(b0.x, j, V3<R>{cb[3], cb[4], cb[5]});
          atomicAdd3(b0.v, j, V3<R>{cb[9], cb[10], cb[11]});
          atomicAdd3(b0.w, j, V3<R>{cb[15], cb[16], cb[17]});
        }
        st3(b0.xi, c, V3<R>{cb[18], cb[19], cb[20]});
        gE += cb[21], ge += cb[22], gmu += cb[23];
      }
    }
  }
  flushParams(thetaB, gE, ge, gmu);
}

// ---- tangent-linear (forward mode, one tangent) ----
template <class R>
__global__ void kContactsJvp(Model<R> M, StateView<R> s, StateView<R> sd, StateView<R> t, StateView<R> td, R Ed,
                             R ed, R mud, R* F, R* T, R* Fd, R* Td) {
  GRID_STRIDE(c, M.nc) {
    const int i = M.cont[2 * c], j = M.cont[2 * c + 1], k = j < 0 ? -j - 1 : -1;
    const int jj = j >= 0 ? j : i;
    Dn<R, 1> in[kIn], out[kOut];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      in[a].v = s.x[3 * i + a], in[a].d[0] = sd.x[3 * i + a];
      in[3 + a].v = s.x[3 * jj + a], in[3 + a].d[0] = sd.x[3 * jj + a];
      in[6 + a].v = s.v[3 * i + a], in[6 + a].d[0] = sd.v[3 * i + a];
      in[9 + a].v = s.v[3 * jj + a], in[9 + a].d[0] = sd.v[3 * jj + a];
      in[12 + a].v = s.w[3 * i + a], in[12 + a].d[0] = sd.w[3 * i + a];
      in[15 + a].v = s.w[3 * jj + a], in[15 + a].d[0] = sd.w[3 * jj + a];
      in[18 + a].v = s.xi[3 * c + a], in[18 + a].d[0] = sd.xi[3 * c + a];
    }
    in[21].v = M.E, in[21].d[0] = Ed;
    in[22].v = M.e, in[22].d[0] = ed;
    in[23].v = M.mu, in[23].d[0] = mud;
    if (!contactLaw<Dn<R, 1>, R>(M, i, j, k, in, out)) {
      st3(t.xi, c, V3<R>{R(0), R(0), R(0)});
      st3(td.xi, c, V3<R>{R(0), R(0), R(0)});
      continue;
    }
    st3(t.xi, c, V3<R>{out[9].v, out[10].v, out[11].v});
    st3(td.xi, c, V3<R>{out[9].d[0], out[10].d[0], out[11].d[0]});
    atomicAdd3(F, i, V3<R>{out[0].v, out[1].v, out[2].v});
    atomicAdd3(Fd, i, V3<R>{out[0].d[0], out[1].d[0], out[2].d[0]});
    atomicAdd3(T, i, V3<R>{out[3].v, out[4].v, out[5].v});
    atomicAdd3(Td, i, V3<R>{out[3].d[0], out[4].d[0], out[5].d[0]});
    if (j >= 0) {
      atomicAdd3(F, j, V3<R>{-out[0].v, -out[1].v, -out[2].v});
      atomicAdd3(Fd, j, V3<R>{-out[0].d[0], -out[1].d[0], -out[2].d[0]});
      atomicAdd3(T, j, V3<R>{out[6].v, out[7].v, out[8].v});
      atomicAdd3(Td, j, V3<R>{out[6].d[0], out[7].d[0], out[8].d[0]});
    }
  }
}
template <class R>
__global__ void kIntegrateJvp(Model<R> M, StateView<R> s, StateView<R> sd, StateView<R> t, StateView<R> td, R* F,
                              R* T, R* Fd, R* Td) {
  GRID_STRIDE(i, M.n) {
    const R im = M.im[i], iI = M.iI[i];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const long q = 3 * i + a;
      const R v = s.v[q] + (F[q] * im + M.g[a]) * M.dt;
      const R vd = sd.v[q] + Fd[q] * im * M.dt;
      t.v[q] = v, td.v[q] = vd;
      t.w[q] = s.w[q] + T[q] * iI * M.dt, td.w[q] = sd.w[q] + Td[q] * iI * M.dt;
      t.x[q] = s.x[q] + v * M.dt, td.x[q] = sd.x[q] + vd * M.dt;
      F[q] = T[q] = Fd[q] = Td[q] = R(0);
    }
  }
}

// Candidate contacts, `split` blocks per scene [first[s], first[s + 1]): for each sphere i of the
// scene, the spheres i < j of the scene with |x_i - x_j| < r_i + r_j + skin, then the planes k with
// (x_i - p0_k).n_k < r_i + skin, in that order. Each block stages the scene's positions and radii
// in shared memory (structure of arrays: a warp reads consecutive entries) when they fit (SMEM),
// else reads global memory. Rows are dealt in pairs (q, ns - 1 - q) so every thread scans about
// ns / 2 partners; block b of a scene takes the pairs q = b, b + split, ... Pass 1 (off ==
// nullptr) writes each sphere's count; pass 2 writes its contacts at off[i].
constexpr int kCandBlock = 256;
template <class R, bool SMEM>
__global__ void __launch_bounds__(kCandBlock) kCandScene(const R* x, const R* r, const int* first, int split,
                                                         const R* planes, int nplane, R skin, int* cnt, const int* off,
                                                         int* out) {
  extern __shared__ __align__(16) unsigned char smRaw[];
  const int scene = blockIdx.x / split, part = blockIdx.x % split;
  const int a = first[scene], ns = first[scene + 1] - a;
  R* sx = reinterpret_cast<R*>(smRaw);
  R *sy = sx + ns, *sz = sy + ns, *sr = sz + ns;
  if (SMEM) {
    for (int q = threadIdx.x; q < ns; q += blockDim.x) {
      sx[q] = x[3 * (a + q)], sy[q] = x[3 * (a + q) + 1], sz[q] = x[3 * (a + q) + 2];
      sr[q] = r[a + q];
    }
    __syncthreads();
  }
  auto px = [&](int q) { return SMEM ? sx[q] : x[3 * (a + q)]; };
  auto py = [&](int q) { return SMEM ? sy[q] : x[3 * (a + q) + 1]; };
  auto pz = [&](int q) { return SMEM ? sz[q] : x[3 * (a + q) + 2]; };
  auto pr = [&](int q) { return SMEM ? sr[q] : r[a + q]; };
  const int half = (ns + 1) / 2;
  for (int q = part * blockDim.x + threadIdx.x; q < half; q += split * blockDim.x) {
    for (int h = 0; h < 2; ++h) {
      const int li = h == 0 ? q : ns - 1 - q;
      if (h == 1 && li == q)
        break;
      const int i = a + li;
      const R xi = px(li), yi = py(li), zi = pz(li), ri = pr(li) + skin;
      int c = 0;
      const int base = off ? off[i] : 0;
      for (int lj = li + 1; lj < ns; ++lj) {
        const R dx = xi - px(lj), dy = yi - py(lj), dz = zi - pz(lj);
        const R lim = ri + pr(lj);
        if (dx * dx + dy * dy + dz * dz < lim * lim) {
          if (off) {
            out[2 * (base + c)] = i;
            out[2 * (base + c) + 1] = a + lj;
          }
          ++c;
        }
      }
      for (int k = 0; k < nplane; ++k) {
        const R* pl = planes + 6 * k;
        const R dist = (xi - pl[0]) * pl[3] + (yi - pl[1]) * pl[4] + (zi - pl[2]) * pl[5];
        if (dist < ri) {
          if (off) {
            out[2 * (base + c)] = i;
            out[2 * (base + c) + 1] = -k - 1;
          }
          ++c;
        }
      }
      if (!off)
        cnt[i] = c;
    }
  }
}
// Candidate contacts on a cell grid, `split` blocks per scene, for scenes that fit in shared memory:
// each block stages its scene (positions and radii as structure of arrays), bins the spheres into
// cells of side h >= 2 r_max + skin over the scene's bounding box (coarser when the cells would not
// fit), and takes the rows li = part, part + split, ... (strided over the block's threads). A row
// scans the 27 cells around its sphere for partners j > i within r_i + r_j + skin, then the planes
// within r_i + skin; it reserves room with one atomic and writes 64-bit keys
// i (n + nplane) + (j, or n + plane) in no particular order (sorted afterwards). Keys past `cap`
// are not written; *total counts them all.
constexpr int kGridBlock = 256, kCellCap = 4096;
template <class R>
__global__ void __launch_bounds__(kGridBlock) kCandGrid(const R* x, const R* r, const int* first, int split, int n,
                                                        const R* planes, int nplane, R skin, unsigned long long* keys,
                                                        long cap, unsigned long long* total) {
  extern __shared__ __align__(16) unsigned char smRaw[];
  __shared__ R red[6][kGridBlock / 32];
  __shared__ R redR[kGridBlock / 32];
  __shared__ int cellStart[kCellCap + 1];
  __shared__ int cursor[kCellCap];
  __shared__ R lo[3], h;
  __shared__ int dims[3];
  const int scene = blockIdx.x / split, part = blockIdx.x % split;
  const int a = first[scene], ns = first[scene + 1] - a;
  R* sx = reinterpret_cast<R*>(smRaw);
  R *sy = sx + ns, *sz = sy + ns, *sr = sz + ns;
  int* order = reinterpret_cast<int*>(sr + ns);
  R mn[3] = {R(INFINITY), R(INFINITY), R(INFINITY)}, mx[3] = {R(-INFINITY), R(-INFINITY), R(-INFINITY)}, rmax = 0;
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    const R p[3] = {x[3 * (a + q)], x[3 * (a + q) + 1], x[3 * (a + q) + 2]};
    sx[q] = p[0], sy[q] = p[1], sz[q] = p[2], sr[q] = r[a + q];
    rmax = fmax(rmax, sr[q]);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      mn[c] = fmin(mn[c], p[c]), mx[c] = fmax(mx[c], p[c]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      mn[c] = fmin(mn[c], __shfl_xor_sync(0xffffffffu, mn[c], o));
      mx[c] = fmax(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) {
    redR[wid] = rmax;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      red[c][wid] = mn[c], red[3 + c][wid] = mx[c];
  }
  for (int c = threadIdx.x; c < kCellCap; c += blockDim.x)
    cursor[c] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    R m0[3] = {red[0][0], red[1][0], red[2][0]}, m1[3] = {red[3][0], red[4][0], red[5][0]}, rm = redR[0];
    for (int w = 1; w < nw; ++w) {
      rm = fmax(rm, redR[w]);
      for (int c = 0; c < 3; ++c)
        m0[c] = fmin(m0[c], red[c][w]), m1[c] = fmax(m1[c], red[3 + c][w]);
    }
    R side = R(2) * rm + skin;
    if (!(side > R(0)))
      side = R(1);
    int d[3] = {1, 1, 1};
    bool fit = false;
    for (int it = 0; it < 64 && !fit; ++it) {  // coarser cells until they fit (a bounded search)
      long cells = 1;
      for (int c = 0; c < 3; ++c) {
        const R ext = m1[c] - m0[c];
        d[c] = ext > R(0) && ext < side * R(kCellCap) ? (int)(ext / side) + 1 : (ext > R(0) ? kCellCap : 1);
        cells *= d[c];
      }
      fit = cells <= kCellCap;
      if (!fit)
        side *= R(1.26);
    }
    if (!fit) {  // non-finite extents: one cell holds the scene (every pair is tested)
      d[0] = d[1] = d[2] = 1;
      m0[0] = m0[1] = m0[2] = R(0);
    }
    for (int c = 0; c < 3; ++c)
      lo[c] = m0[c], dims[c] = d[c];
    h = side;
  }
  __syncthreads();
  const int nx = dims[0], ny = dims[1], nz = dims[2], ncell = nx * ny * nz;
  auto cellOf = [&](int q, int& cx, int& cy, int& cz) {
    cx = min(max((int)((sx[q] - lo[0]) / h), 0), nx - 1);
    cy = min(max((int)((sy[q] - lo[1]) / h), 0), ny - 1);
    cz = min(max((int)((sz[q] - lo[2]) / h), 0), nz - 1);
  };
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    int cx, cy, cz;
    cellOf(q, cx, cy, cz);
    atomicAdd(&cursor[(cz * ny + cy) * nx + cx], 1);
  }
  __syncthreads();
  {  // exclusive scan of the cell counts: kCellCap / blockDim consecutive cells per thread
    constexpr int per = kCellCap / kGridBlock;
    const int c0 = threadIdx.x * per;
    int v = 0;
    for (int q = 0; q < per; ++q)
      v += c0 + q < ncell ? cursor[c0 + q] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o)
        incl += u;
    }
    __shared__ int wsum[kGridBlock / 32];
    if (lane == 31)
      wsum[wid] = incl;
    __syncthreads();
    int before = incl - v;
    for (int w = 0; w < wid; ++w)
      before += wsum[w];
    for (int q = 0; q < per; ++q) {
      if (c0 + q < ncell) {
        cellStart[c0 + q] = before;
        before += cursor[c0 + q];
      }
    }
    if (threadIdx.x == blockDim.x - 1)
      cellStart[ncell] = before;
    __syncthreads();
    for (int q = 0; q < per; ++q)
      if (c0 + q < ncell)
        cursor[c0 + q] = 0;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < ns; q += blockDim.x) {
    int cx, cy, cz;
    cellOf(q, cx, cy, cz);
    const int c = (cz * ny + cy) * nx + cx;
    order[cellStart[c] + atomicAdd(&cursor[c], 1)] = q;
  }
  __syncthreads();
  const unsigned long long np = (unsigned long long)(n + nplane);
  for (int li = part * blockDim.x + threadIdx.x; li < ns; li += split * blockDim.x) {
    int cx, cy, cz;
    cellOf(li, cx, cy, cz);
    const R xi = sx[li], yi = sy[li], zi = sz[li], ri = sr[li] + skin;
    const int i = a + li;
    unsigned long long base = 0;
    for (int pass = 0; pass < 2; ++pass) {
      int c = 0;
      for (int dz = -1; dz <= 1; ++dz) {
        const int zz = cz + dz;
        if (zz < 0 || zz >= nz)
          continue;
        for (int dy = -1; dy <= 1; ++dy) {
          const int yy = cy + dy;
          if (yy < 0 || yy >= ny)
            continue;
          for (int dx = -1; dx <= 1; ++dx) {
            const int xx = cx + dx;
            if (xx < 0 || xx >= nx)
              continue;
            const int cell = (zz * ny + yy) * nx + xx;
            for (int t = cellStart[cell]; t < cellStart[cell + 1]; ++t) {
              const int lj = order[t];
              if (lj <= li)
                continue;
              const R ex = xi - sx[lj], ey = yi - sy[lj], ez = zi - sz[lj];
              const R lim = ri + sr[lj];
              if (ex * ex + ey * ey + ez * ez < lim * lim) {
                if (pass == 1 && base + c < (unsigned long long)cap)
                  keys[base + c] = (unsigned long long)i * np + (unsigned long long)(a + lj);
                ++c;
              }
            }
          }
        }
      }
      for (int k = 0; k < nplane; ++k) {
        const R* pl = planes + 6 * k;
        const R dist = (xi - pl[0]) * pl[3] + (yi - pl[1]) * pl[4] + (zi - pl[2]) * pl[5];
        if (dist < ri) {
          if (pass == 1 && base + c < (unsigned long long)cap)
            keys[base + c] = (unsigned long long)i * np + (unsigned long long)(n + k);
          ++c;
        }
      }
      if (pass == 0) {
        if (c == 0)
          break;
        base = atomicAdd(total, (unsigned long long)c);
      }
    }
  }
}
// sorted keys back to (i, j) rows: j = key mod (n + nplane), a plane k when j >= n (stored -k - 1)
__global__ void kDecodeKeys(const unsigned long long* keys, long count, int n, int nplane, int* out) {
  GRID_STRIDE(p, count) {
    const unsigned long long np = (unsigned long long)(n + nplane), k = keys[p];
    const int i = (int)(k / np), j = (int)(k % np);
    out[2 * p] = i;
    out[2 * p + 1] = j < n ? j : -(j - n) - 1;
  }
}

// exclusive prefix sum of cnt[0, n) into off[0, n], off[n] = total; one block walks the array in
// chunks of blockDim x kScanItems (each thread sums kScanItems consecutive counts, the block scans
// the thread sums with warp shuffles, a running carry joins the chunks)
constexpr int kScanBlock = 1024, kScanItems = 16;
__global__ void __launch_bounds__(kScanBlock) kScanCounts(const int* cnt, int n, int* off) {
  __shared__ int warpSum[kScanBlock / 32];
  __shared__ long long carry;
  if (threadIdx.x == 0)
    carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (long base = 0; base < n; base += (long)blockDim.x * kScanItems) {
    const long first = base + (long)threadIdx.x * kScanItems;
    int item[kScanItems];
    int v = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
      item[q] = first + q < n ? cnt[first + q] : 0;
      v += item[q];
    }
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o)
        incl += u;
    }
    if (lane == 31)
      warpSum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int ws = lane < (int)(blockDim.x >> 5) ? warpSum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o)
          ws += u;
      }
      warpSum[lane] = ws;  // inclusive over warps
    }
    __syncthreads();
    long long run = carry + (wid > 0 ? warpSum[wid - 1] : 0) + incl - v;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
      if (first + q < n)
        off[first + q] = (int)run;
      run += item[q];
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1)
      carry = run;
    __syncthreads();
  }
  if (threadIdx.x == 0)
    off[n] = (int)carry;
}

// ---------------------------------------------------------------------------------------------
struct Fail {
  int status;
  std::string msg;
};
void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw Fail{PDEM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}
template <class R>
Model<R> makeModel(const pdem_hz_model* h) {
  if (!h || h->n < 0 || h->ncontact < 0 || h->nplane < 0)
    throw Fail{PDEM_ERR_INVALID, "hz model: negative sizes"};
  if (3L * h->n > (long)INT_MAX)
    throw Fail{PDEM_ERR_INVALID, "hz model: too many spheres (3 n must fit an int)"};
  if (h->n > 0 && (!h->radius || !h->inv_mass || !h->inv_inertia))
    throw Fail{PDEM_ERR_INVALID, "hz model: radius, inverse mass and inverse inertia are required"};
  if ((h->ncontact > 0 && !h->contacts) || (h->nplane > 0 && !h->planes))
    throw Fail{PDEM_ERR_INVALID, "hz model: contact list or planes missing"};
  if (!(h->youngs > 0) || !(h->dt > 0))
    throw Fail{PDEM_ERR_INVALID, "hz model: Young's modulus and dt must be positive"};
  Model<R> M;
  M.n = h->n, M.nc = h->ncontact, M.nplane = h->nplane, M.cont = h->contacts;
  M.planes = static_cast<const R*>(h->planes);
  M.r = static_cast<const R*>(h->radius);
  M.im = static_cast<const R*>(h->inv_mass);
  M.iI = static_cast<const R*>(h->inv_inertia);
  M.E = R(h->youngs), M.e = R(h->restitution), M.mu = R(h->friction), M.dt = R(h->dt), M.nu = h->poisson;
  for (int a = 0; a < 3; ++a)
    M.g[a] = R(h->gravity[a]);
  return M;
}
int precisionOf(int p) {
  if (p != 32 && p != 64)
    throw Fail{PDEM_ERR_INVALID, "hz: precision must be 32 or 64"};
  return p;
}

template <class R>
void forward(const pdem_hz_model* h, int steps, int store, R* traj, R* work, cudaStream_t st) {
  const Model<R> M = makeModel<R>(h);
  if (steps <= 0 || M.n == 0)
    return;
  if (!traj || !work)
    throw Fail{PDEM_ERR_INVALID, "hz forward: trajectory or work buffer missing"};
  const size_t S = stateSize(M.n, M.nc);
  R* F = work;
  R* T = work + 3 * (size_t)M.n;
  check(cudaMemsetAsync(F, 0, 6 * (size_t)M.n * sizeof(R), st), "memset");
  for (int k = 0; k < steps; ++k) {
    const size_t a = store ? k : (k & 1), b = store ? k + 1 : ((k + 1) & 1);
    const StateView<R> s = view(traj + S * a, M.n), t = view(traj + S * b, M.n);
    if (M.nc > 0)
      kContacts<R><<<pdem::gridFor(M.nc), pdem::kBlock, 0, st>>>(M, s, t, F, T);
    kIntegrate<R><<<pdem::gridFor(3L * M.n), pdem::kBlock, 0, st>>>(M, s, t, F, T);
  }
  if (!store && (steps & 1) == 0)  // the final state of a ping-pong run always ends in block 1
    check(cudaMemcpyAsync(traj + S, traj, S * sizeof(R), cudaMemcpyDeviceToDevice, st), "D2D");
  check(cudaGetLastError(), "hz forward");
}

template <class R>
void backward(const pdem_hz_model* h, int steps, const R* traj, R* adj, double* thetaB, R* work, int mode,
              cudaStream_t st) {
  const Model<R> M = makeModel<R>(h);
  if (steps <= 0 || M.n == 0)
    return;
  if (!traj || !adj || !work)
    throw Fail{PDEM_ERR_INVALID, "hz backward: trajectory, adjoint or work buffer missing"};
  if (mode != 0 && mode != 1)
    throw Fail{PDEM_ERR_INVALID, "hz backward: mode must be 0 (reversal) or 1 (dual Jacobians)"};
  const size_t SZ = stateSize(M.n, M.nc);
  R* Fb = work;
  R* Tb = work + 3 * (size_t)M.n;
  R* other = work + 6 * (size_t)M.n;  // second adjoint state, ping-pong with adj
  int* cnt = reinterpret_cast<int*>(other + SZ);  // two counter slots, then the active list
  int* list = cnt + 2;
  check(cudaMemsetAsync(cnt, 0, 2 * sizeof(int), st), "memset");
  R* cur = adj;
  for (int k = steps - 1; k >= 0; --k) {
    const StateView<R> s = view(const_cast<R*>(traj) + SZ * k, M.n);
    const StateView<R> b1 = view(cur, M.n), b0 = view(other, M.n);
    kIntegrateAdj<R><<<pdem::gridFor(3L * M.n), pdem::kBlock, 0, st>>>(M, b1, b0, Fb, Tb);
    if (M.nc > 0) {
      if (mode == 0) {
        kContactsAdjScan<R><<<pdem::gridFor(M.nc), pdem::kBlock, 0, st>>>(M, s, b0, list, cnt + (k & 1));
        // the active list is a small part of the contacts: a grid of a few blocks per SM strides it
        const int g = std::min(pdem::gridFor(M.nc), 4 * pdem::kNumSMs);
        kContactsAdj<R><<<g, pdem::kBlock, 0, st>>>(M, s, b1, b0, Fb, Tb, thetaB, list, cnt + (k & 1),
                                                    cnt + ((k + 1) & 1));
      } else {
        kContactsAdjDual<R><<<pdem::gridFor(M.nc), pdem::kBlock, 0, st>>>(M, s, b1, b0, Fb, Tb, thetaB);
      }
    }
    std::swap(cur, other);
  }
  if (cur != adj)
    check(cudaMemcpyAsync(adj, cur, SZ * sizeof(R), cudaMemcpyDeviceToDevice, st), "D2D");
  check(cudaGetLastError(), "hz backward");
}

template <class R>
void jvp(const pdem_hz_model* h, int steps, R* state, R* tangent, const double* thetaDot, R* work, cudaStream_t st) {
  const Model<R> M = makeModel<R>(h);
  if (steps <= 0 || M.n == 0)
    return;
  if (!state || !tangent || !thetaDot || !work)
    throw Fail{PDEM_ERR_INVALID, "hz jvp: state, tangent, parameter tangent or work buffer missing"};
  const size_t S = stateSize(M.n, M.nc), n3 = 3 * (size_t)M.n;
  R *F = work, *T = work + n3, *Fd = work + 2 * n3, *Td = work + 3 * n3;
  check(cudaMemsetAsync(work, 0, 4 * n3 * sizeof(R), st), "memset");
  for (int k = 0; k < steps; ++k) {
    const size_t a = k & 1, b = (k + 1) & 1;
    const StateView<R> s = view(state + S * a, M.n), t = view(state + S * b, M.n);
    const StateView<R> sd = view(tangent + S * a, M.n), td = view(tangent + S * b, M.n);
    if (M.nc > 0)
      kContactsJvp<R><<<pdem::gridFor(M.nc), pdem::kBlock, 0, st>>>(M, s, sd, t, td, R(thetaDot[0]), R(thetaDot[1]),
                                                                     R(thetaDot[2]), F, T, Fd, Td);
    kIntegrateJvp<R><<<pdem::gridFor(M.n), pdem::kBlock, 0, st>>>(M, s, sd, t, td, F, T, Fd, Td);
  }
  if ((steps & 1) == 0) {
    check(cudaMemcpyAsync(state + S, state, S * sizeof(R), cudaMemcpyDeviceToDevice, st), "D2D");
    check(cudaMemcpyAsync(tangent + S, tangent, S * sizeof(R), cudaMemcpyDeviceToDevice, st), "D2D");
  }
  check(cudaGetLastError(), "hz jvp");
}

// grow-only device scratch of the calling thread (one process per GPU, one stream per caller)
struct Scratch {
  void* p = nullptr;
  size_t bytes = 0;
  void* get(size_t want) {
    if (want > bytes) {
      if (p)
        cudaFree(p);
      p = nullptr;
      bytes = 0;
      check(cudaMalloc(&p, want), "hz scratch");
      bytes = want;
    }
    return p;
  }
};
thread_local Scratch gKeys, gCub, gTotal;

template <class R>
void candidates(const R* x, const R* r, const int* hFirst, const int* dFirst, int nscene, const R* planes, int nplane,
                double skin, int* cnt, int* off, int* out, long cap, long* count, cudaStream_t st) {
  *count = 0;
  if (nscene < 1)
    return;
  int maxScene = 0;
  if (hFirst[0] != 0)
    throw Fail{PDEM_ERR_INVALID, "hz contacts: scenes must start at sphere 0"};
  for (int q = 0; q < nscene; ++q) {
    if (hFirst[q + 1] < hFirst[q])
      throw Fail{PDEM_ERR_INVALID, "hz contacts: scene offsets must not decrease"};
    maxScene = std::max(maxScene, hFirst[q + 1] - hFirst[q]);
  }
  const int n = hFirst[nscene];
  if (n < 1)
    return;
  // cell-grid path: every scene staged in shared memory (positions, radii, cell order)
  constexpr size_t kGridDyn = 160 * 1024;
  const size_t gridSmem = (4 * sizeof(R) + sizeof(int)) * (size_t)maxScene;
  if (gridSmem <= kGridDyn) {
    static bool attr[2] = {false, false};
    if (!attr[sizeof(R) == 8]) {
      check(cudaFuncSetAttribute(kCandGrid<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGridDyn),
            "smem attribute");
      attr[sizeof(R) == 8] = true;
    }
    int split = std::max(1, (4 * pdem::kNumSMs + nscene - 1) / nscene);
    split = std::min(split, std::max(1, (maxScene + kGridBlock - 1) / kGridBlock));
    auto* total = static_cast<unsigned long long*>(gTotal.get(sizeof(unsigned long long)));
    check(cudaMemsetAsync(total, 0, sizeof(unsigned long long), st), "memset");
    auto* keys = reinterpret_cast<unsigned long long*>(out);  // cap x 2 ints = cap keys
    kCandGrid<R><<<nscene * split, kGridBlock, gridSmem, st>>>(x, r, dFirst, split, n, planes, nplane, R(skin), keys,
                                                               cap, total);
    check(cudaGetLastError(), "hz candidate grid");
    unsigned long long tot = 0;
    check(cudaMemcpyAsync(&tot, total, sizeof(tot), cudaMemcpyDeviceToHost, st), "D2H");
    check(cudaStreamSynchronize(st), "sync");
    *count = (long)tot;
    if ((long)tot > cap || tot == 0)
      return;
    auto* sorted = static_cast<unsigned long long*>(gKeys.get(tot * sizeof(unsigned long long)));
    const unsigned long long maxKey = (unsigned long long)n * (unsigned long long)(n + nplane);
    int endBit = 1;
    while (endBit < 64 && (maxKey >> endBit))
      ++endBit;
    size_t bytes = 0;
    check(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys, sorted, (int)tot, 0, endBit, st), "cub sort");
    check(cub::DeviceRadixSort::SortKeys(gCub.get(bytes), bytes, keys, sorted, (int)tot, 0, endBit, st), "cub sort");
    kDecodeKeys<<<pdem::gridFor((long)tot), pdem::kBlock, 0, st>>>(sorted, (long)tot, n, nplane, out);
    check(cudaGetLastError(), "hz candidate decode");
    return;
  }
  // scenes too large for shared memory: brute force over each scene from global memory, counted,
  // scanned and written in (i, j) order
  if (!cnt || !off)
    throw Fail{PDEM_ERR_INVALID, "hz contacts: scenes this large need the count and offset scratch"};
  const int rows = (maxScene + 1) / 2;
  int split = std::max(1, (4 * pdem::kNumSMs + nscene - 1) / nscene);
  split = std::min(split, std::max(1, (rows + kCandBlock - 1) / kCandBlock));
  kCandScene<R, false><<<nscene * split, kCandBlock, 0, st>>>(x, r, dFirst, split, planes, nplane, R(skin), cnt,
                                                              nullptr, out);
  check(cudaGetLastError(), "hz candidate count");
  kScanCounts<<<1, kScanBlock, 0, st>>>(cnt, n, off);
  int total = 0;
  check(cudaMemcpyAsync(&total, off + n, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  check(cudaStreamSynchronize(st), "sync");
  *count = total;
  if (total > cap || total == 0)
    return;
  kCandScene<R, false><<<nscene * split, kCandBlock, 0, st>>>(x, r, dFirst, split, planes, nplane, R(skin), cnt, off,
                                                              out);
  check(cudaGetLastError(), "hz candidate write");
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return PDEM_OK;
  } catch (const Fail& e) {
    pdem::setLastError(e.msg);
    return e.status;
  }
}

}  // namespace

extern "C" {

long pdem_hz_state_size(int n, int ncontact) {
  return (n < 0 || ncontact < 0) ? -1 : (long)stateSize(n, ncontact);
}
long pdem_hz_work_size(int n, int ncontact) {
  if (n < 0 || ncontact < 0)
    return -1;
  // backward: force/torque adjoints, a second adjoint state, then (as ints) two counters and the
  // active-contact list; jvp: four force/torque arrays
  const size_t a = 6 * (size_t)n + stateSize(n, ncontact) + (size_t)ncontact + 2, b = 12 * (size_t)n;
  return (long)(a > b ? a : b);
}

int pdem_hz_contacts(int precision, const void* d_x, const void* d_radius, const int* first, const int* d_first,
                     int nscene, const void* d_planes, int nplane, double skin, int* d_cnt, int* d_off, int* d_contacts,
                     long cap, long* count, void* stream) {
  return guarded([&] {
    if (!count || nscene < 0 || nplane < 0 || (nplane > 0 && !d_planes) || (nscene > 0 && (!d_first || !first)))
      throw Fail{PDEM_ERR_INVALID, "hz contacts: bad arguments"};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precisionOf(precision) == 64)
      candidates<double>(static_cast<const double*>(d_x), static_cast<const double*>(d_radius), first, d_first, nscene,
                         static_cast<const double*>(d_planes), nplane, skin, d_cnt, d_off, d_contacts, cap, count, st);
    else
      candidates<float>(static_cast<const float*>(d_x), static_cast<const float*>(d_radius), first, d_first, nscene,
                        static_cast<const float*>(d_planes), nplane, skin, d_cnt, d_off, d_contacts, cap, count, st);
  });
}

int pdem_hz_forward(int precision, const pdem_hz_model* model, int steps, int store, void* d_traj, void* d_work,
                    void* stream) {
  return guarded([&] {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precisionOf(precision) == 64)
      forward<double>(model, steps, store, static_cast<double*>(d_traj), static_cast<double*>(d_work), st);
    else
      forward<float>(model, steps, store, static_cast<float*>(d_traj), static_cast<float*>(d_work), st);
  });
}

int pdem_hz_backward(int precision, const pdem_hz_model* model, int steps, const void* d_traj, void* d_adj,
                     double* d_grad, void* d_work, int mode, void* stream) {
  return guarded([&] {
    if (!d_grad)
      throw Fail{PDEM_ERR_INVALID, "hz backward: parameter gradient buffer missing"};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precisionOf(precision) == 64)
      backward<double>(model, steps, static_cast<const double*>(d_traj), static_cast<double*>(d_adj), d_grad,
                       static_cast<double*>(d_work), mode, st);
    else
      backward<float>(model, steps, static_cast<const float*>(d_traj), static_cast<float*>(d_adj), d_grad,
                      static_cast<float*>(d_work), mode, st);
  });
}

int pdem_hz_jvp(int precision, const pdem_hz_model* model, int steps, void* d_state, void* d_tangent,
                const double* theta_dot, void* d_work, void* stream) {
  return guarded([&] {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precisionOf(precision) == 64)
      jvp<double>(model, steps, static_cast<double*>(d_state), static_cast<double*>(d_tangent), theta_dot,
                  static_cast<double*>(d_work), st);
    else
      jvp<float>(model, steps, static_cast<float*>(d_state), static_cast<float*>(d_tangent), theta_dot,
                 static_cast<float*>(d_work), st);
  });
}

}  // extern "C"
