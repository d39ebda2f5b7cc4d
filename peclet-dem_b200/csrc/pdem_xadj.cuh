// Adjoint of the XPBD substep (plain FP64 path, spheres and planes): the per-entry local maps
// and their vector-Jacobian products.
//
// Every stage of the substep that the reverse pass differentiates is written once here as a
// local map from a flat array of active inputs to a flat array of outputs, templated on the
// scalar type:
//   - with T = double it is the replay: the same expressions, in the same order, as the forward
//     step (src/integration.hpp:44-148, src/narrowphase.hpp:179-268 and :371-449,
//     src/contact_preprocessing.hpp:339-374, src/solver_velocity.hpp:390-605 and :641-858,
//     src/solver_position.hpp:248-331), so the replay takes the forward's branches;
//   - with T = Dd<K> (forward-mode dual numbers with K tangent lanes) it yields K columns of the
//     map's Jacobian at once; vjp() seeds the inputs K at a time and contracts the output
//     tangents with the output adjoints, which is the map's vector-Jacobian product.
// The branch decisions (active contact, clamps of the normal impulse and of the friction cone,
// restitution cut-off, side flags) are taken on the values, so the derivative is the one of the
// branch the forward took. The sweep-level reversal (colours and sweeps in reverse order over the
// frozen colouring, checkpoints and replays) is in pdem_xadj.cu.
#pragma once
#include <cuda_runtime.h>

#include "pdem_math.cuh"

namespace pdem {
namespace xadj {

// ---- forward-mode dual numbers ------------------------------------------------------------
// K = 7 lanes: sizeof(Dd<7>) = 64 B, so Q4<Dd<7>> (aligned to 4 x its element) stays a power of 2
constexpr int kLanes = 7;

template <int K>
struct Dd {
  double v;
  double d[K];
  PD Dd() : v(0.0) {
#pragma unroll
    for (int k = 0; k < K; ++k)
      d[k] = 0.0;
  }
  PD Dd(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < K; ++k)
      d[k] = 0.0;
  }
};
template <int K>
PD Dd<K> operator+(const Dd<K>& a, const Dd<K>& b) {
  Dd<K> r(a.v + b.v);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int K>
PD Dd<K> operator-(const Dd<K>& a, const Dd<K>& b) {
  Dd<K> r(a.v - b.v);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int K>
PD Dd<K> operator-(const Dd<K>& a) {
  Dd<K> r(-a.v);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = -a.d[k];
  return r;
}
template <int K>
PD Dd<K> operator*(const Dd<K>& a, const Dd<K>& b) {
  Dd<K> r(a.v * b.v);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int K>
PD Dd<K> operator/(const Dd<K>& a, const Dd<K>& b) {
  const double q = a.v / b.v;
  Dd<K> r(q);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = (a.d[k] - q * b.d[k]) / b.v;
  return r;
}
// mixed forms with a plain double (a constant of the map), value arithmetic unchanged
template <int K>
PD Dd<K> operator+(const Dd<K>& a, double b) {
  Dd<K> r = a;
  r.v = a.v + b;
  return r;
}
template <int K>
PD Dd<K> operator+(double a, const Dd<K>& b) {
  Dd<K> r = b;
  r.v = a + b.v;
  return r;
}
template <int K>
PD Dd<K> operator-(const Dd<K>& a, double b) {
  Dd<K> r = a;
  r.v = a.v - b;
  return r;
}
template <int K>
PD Dd<K> operator-(double a, const Dd<K>& b) {
  Dd<K> r(a - b.v);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = -b.d[k];
  return r;
}
template <int K>
PD Dd<K> operator*(const Dd<K>& a, double b) {
  Dd<K> r(a.v * b);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = a.d[k] * b;
  return r;
}
template <int K>
PD Dd<K> operator*(double a, const Dd<K>& b) {
  Dd<K> r(a * b.v);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = a * b.d[k];
  return r;
}
template <int K>
PD Dd<K> operator/(const Dd<K>& a, double b) {
  Dd<K> r(a.v / b);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = a.d[k] / b;
  return r;
}
template <int K>
PD Dd<K> operator/(double a, const Dd<K>& b) {
  const double q = a / b.v;
  Dd<K> r(q);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = -q * b.d[k] / b.v;
  return r;
}
template <int K>
PD Dd<K>& operator+=(Dd<K>& a, const Dd<K>& b) {
  return a = a + b;
}
template <int K>
PD bool operator<(const Dd<K>& a, const Dd<K>& b) { return a.v < b.v; }
template <int K>
PD bool operator>(const Dd<K>& a, const Dd<K>& b) { return a.v > b.v; }
template <int K>
PD bool operator<=(const Dd<K>& a, const Dd<K>& b) { return a.v <= b.v; }
template <int K>
PD bool operator>=(const Dd<K>& a, const Dd<K>& b) { return a.v >= b.v; }
template <int K>
PD bool operator==(const Dd<K>& a, const Dd<K>& b) { return a.v == b.v; }
template <int K>
PD bool operator!=(const Dd<K>& a, const Dd<K>& b) { return a.v != b.v; }
template <int K>
PD bool operator<(const Dd<K>& a, double b) { return a.v < b; }
template <int K>
PD bool operator>(const Dd<K>& a, double b) { return a.v > b; }
template <int K>
PD bool operator<=(const Dd<K>& a, double b) { return a.v <= b; }
template <int K>
PD bool operator>=(const Dd<K>& a, double b) { return a.v >= b; }
template <int K>
PD bool operator!=(const Dd<K>& a, double b) { return a.v != b; }
template <int K>
PD bool operator==(const Dd<K>& a, double b) { return a.v == b; }

template <int K>
PD Dd<K> sqrt(const Dd<K>& a) {
  const double s = ::sqrt(a.v);
  const double g = s > 0.0 ? 0.5 / s : 0.0;
  Dd<K> r(s);
#pragma unroll
  for (int k = 0; k < K; ++k)
    r.d[k] = g * a.d[k];
  return r;
}
template <int K>
PD Dd<K> fabs(const Dd<K>& a) {
  return a.v < 0.0 ? -a : a;
}
template <int K>
PD Dd<K> fmax(const Dd<K>& a, const Dd<K>& b) {
  return (b.v > a.v) ? b : a;
}

// the same functions on plain doubles (the replay instantiation), which the templates above hide
PD double sqrt(double a) { return ::sqrt(a); }
PD double fabs(double a) { return ::fabs(a); }
PD double fmax(double a, double b) { return ::fmax(a, b); }

// value of a scalar of either kind
PD double val(double x) { return x; }
template <int K>
PD double val(const Dd<K>& x) {
  return x.v;
}

// ---- constants of the maps (not differentiated) ---------------------------------------------
struct BodyC {     // one body
  double im;       // inverse mass
  V3<double> iI;   // inverse inertia (body frame)
};
struct StepC {     // the substep
  double dt;
  V3<double> g;
  double vRest;    // 2 dt |g| (main sweeps) or the stabilization threshold
  double eps;      // central-difference step of the SDF normal (canonical units)
};

// flat views of vectors in an input/output array
template <class T>
PD V3<T> ld3(const T* a, int o) {
  return V3<T>{a[o], a[o + 1], a[o + 2]};
}
template <class T>
PD Q4<T> ld4(const T* a, int o) {
  return Q4<T>{a[o], a[o + 1], a[o + 2], a[o + 3]};
}
template <class T>
PD void st3(T* a, int o, V3<T> v) {
  a[o] = v.x, a[o + 1] = v.y, a[o + 2] = v.z;
}
template <class T>
PD void st4(T* a, int o, Q4<T> v) {
  a[o] = v.x, a[o + 1] = v.y, a[o + 2] = v.z, a[o + 3] = v.w;
}
template <class T>
PD V3<T> cv3(V3<double> a) {
  return V3<T>{T(a.x), T(a.y), T(a.z)};
}

// ---- predictVelocity (src/integration.hpp:44-93) ------------------------------------------
// in: x[0..3) q[3..7) v[7..10) w[10..13)   out: vP[0..3) wP[3..6) xP[6..9)
constexpr int kPredIn = 13, kPredOut = 9;
template <class T>
PD void predictMap(const T* in, T* out, const BodyC& b, const StepC& s, V3<double> F) {
  const double im = b.im, dtt = s.dt;
  V3<T> v = ld3(in, 7);
  if (im > 0.0) {
    v = add(v, cv3<T>(mul(s.g, dtt)));
    v = add(v, cv3<T>(mul(F, im * dtt)));
  }
  V3<T> wp = ld3(in, 10);
  if (im > 0.0) {
    const V3<double> ii = b.iI;
    if (ii.x > 0.0 || ii.y > 0.0 || ii.z > 0.0) {
      const Q4<T> q = ld4(in, 3);
      V3<T> wb = invrot(q, ld3(in, 10));
      const V3<double> Ib{(ii.x > 1e-9) ? 1.0 / ii.x : 0.0, (ii.y > 1e-9) ? 1.0 / ii.y : 0.0,
                          (ii.z > 1e-9) ? 1.0 / ii.z : 0.0};
      const V3<T> Lb{T(Ib.x) * wb.x, T(Ib.y) * wb.y, T(Ib.z) * wb.z};
      const V3<T> wxL = cross(wb, Lb);
      const V3<T> al{T(-ii.x) * wxL.x, T(-ii.y) * wxL.y, T(-ii.z) * wxL.z};
      wb = add(wb, mul(al, T(dtt)));
      wp = rot(q, wb);
    }
  }
  V3<T> x = ld3(in, 0);
  if (im > 0.0)
    x = add(x, mul(v, T(dtt)));
  st3(out, 0, v);
  st3(out, 3, wp);
  st3(out, 6, x);
}

// ---- sphere-sphere contact (src/narrowphase.hpp:179-268, spheres: no shell points) ----------
// in: xA[0..3) qA[3..7) xB[7..10) qB[10..14)   out: n[0..3) rA[3..6) rB[6..9) dist[9]
constexpr int kConIn = 14, kConOut = 10;
struct ConC {
  double sA, sB;     // scale x global scale of each body
  double parA, parB; // canonical sphere radii
  double eps;
};
template <class T>
PD T sdfSph(V3<T> p, double r) {
  return vlen(p) - T(r);
}
template <class T>
PD void contactMap(const T* in, T* out, const ConC& c) {
  const V3<T> pA = ld3(in, 0), pB = ld3(in, 7);
  const Q4<T> qA = ld4(in, 3), qB = ld4(in, 10);
  const T sA(c.sA), sB(c.sB);
  const T prad = T(c.parA) * sA;
  const V3<T> pl{T(0.0), T(0.0), T(0.0)};
  const V3<T> pw = add(pA, rot(qA, mul(pl, sA)));
  const V3<T> plB = invrot(qB, sub(pw, pB));
  const V3<T> pc = mul(plB, T(1.0) / sB);
  const T dist = sdfSph(pc, c.parB) * sB;
  const T eff = dist - prad;
  const T eps(c.eps);
  V3<T> nl{sdfSph(V3<T>{pc.x + eps, pc.y, pc.z}, c.parB) - sdfSph(V3<T>{pc.x - eps, pc.y, pc.z}, c.parB),
           sdfSph(V3<T>{pc.x, pc.y + eps, pc.z}, c.parB) - sdfSph(V3<T>{pc.x, pc.y - eps, pc.z}, c.parB),
           sdfSph(V3<T>{pc.x, pc.y, pc.z + eps}, c.parB) - sdfSph(V3<T>{pc.x, pc.y, pc.z - eps}, c.parB)};
  const T l = vlen(nl);
  nl = (l > T(1e-9)) ? mul(nl, T(1.0) / l) : V3<T>{T(0.0), T(1.0), T(0.0)};
  const V3<T> nw = rot(qB, nl);
  const V3<T> ps = sub(pw, mul(nw, prad));
  st3(out, 0, nw);
  st3(out, 3, sub(ps, pA));
  st3(out, 6, sub(sub(ps, mul(nw, eff)), pB));
  out[9] = eff;
}

// ---- contact -> manifold contribution (src/contact_preprocessing.hpp:339-374) --------------
// in: n[0..3) rA[3..6) rB[6..9) dist[9]   out: N[0..3) TA[3..6) TB[6..9) rA[9..12) rB[12..15)
constexpr int kManIn = 10, kManOut = 15;
template <class T>
PD void manifoldMap(const T* in, T* out, bool flip) {
  const V3<T> n = ld3(in, 0), rA = ld3(in, 3), rB = ld3(in, 6);
  const T dist = in[9];
  const V3<T> na = flip ? n : neg(n);
  const V3<T> sh{n.x * dist * T(0.5), n.y * dist * T(0.5), n.z * dist * T(0.5)};
  const V3<T> ra = sub(rA, sh);
  const V3<T> rb = add(rB, sh);
  const V3<T> rc = flip ? rb : ra, ro = flip ? ra : rb;
  st3(out, 0, na);
  st3(out, 3, cross(rc, na));
  st3(out, 6, cross(ro, neg(na)));
  st3(out, 9, rc);
  st3(out, 12, ro);
}

// manifold geometry in a flat array: N[0..3) TA[3..6) TB[6..9) rA[9..12) rB[12..15) (sums)
constexpr int kGeo = 15;
struct ManC {
  double invN;        // 1 / number of penetrating contacts
  bool hasB;          // body-body (else a wall manifold)
  V3<double> wv;      // summed wall velocity (wall manifolds)
  double imA, imB;
  V3<double> iIA, iIB;
  double eAvg, muAvg; // summed pair restitution / friction x invN (negative: the globals)
  int sf;             // side flag of the sweep
};

// ---- approach velocity before the solve (src/solver_velocity.hpp:390-453) -----------------
// in: vA[0..3) wA[3..6) vB[6..9) wB[9..12) geo[12..27)   out: vn0[0] vt0[1..4)
constexpr int kVn0In = 27, kVn0Out = 4;
template <class T>
PD void vn0Map(const T* in, T* out, const ManC& m) {
  const V3<T> vA = ld3(in, 0), wA = ld3(in, 3);
  V3<T> vB{T(0.0), T(0.0), T(0.0)}, wB{T(0.0), T(0.0), T(0.0)};
  const T invN(m.invN);
  if (m.hasB) {
    vB = ld3(in, 6);
    wB = ld3(in, 9);
  } else {
    vB = mul(cv3<T>(m.wv), invN);
  }
  const V3<T> N = ld3(in, 12), TA = ld3(in, 15), TB = ld3(in, 18);
  const V3<T> rAa = mul(ld3(in, 21), invN), rBa = mul(ld3(in, 24), invN);
  const V3<T> dc = m.hasB ? sub(rAa, rBa) : rAa;
  const V3<T> vG = mul(dc, T(0.0));  // growth rate 0 (growth is outside the adjoint's scope)
  T vn = dot(vA, N) + dot(wA, TA) + dot(vB, neg(N)) + dot(wB, TB);
  vn += dot(vG, N);
  const T lenN = sqrt(dot(N, N));
  V3<T> vt{T(0.0), T(0.0), T(0.0)};
  if (lenN > T(1e-9)) {
    const V3<T> nh = mul(N, T(1.0) / lenN);
    const V3<T> wBv = m.hasB ? wB : V3<T>{T(0.0), T(0.0), T(0.0)};
    const V3<T> vr = sub(add(vA, cross(wA, rAa)), add(vB, cross(wBv, rBa)));
    vt = sub(vr, mul(nh, dot(vr, nh)));
  }
  out[0] = vn;
  st3(out, 1, vt);
}

// ---- warm start (src/solver_velocity.hpp:498-605) -----------------------------------------
// in: vA[0..3) wA[3..6) vB[6..9) wB[9..12) p[12] lt[13..16) geo[16..31) qA[31..35) qB[35..39)
// out: vA[0..3) wA[3..6) vB[6..9) wB[9..12) lt[12..15)
constexpr int kWarmIn = 39, kWarmOut = 15;
template <class T>
PD void warmMap(const T* in, T* out, const ManC& m) {
  V3<T> vA = ld3(in, 0), wA = ld3(in, 3), vB = ld3(in, 6), wB = ld3(in, 9);
  const T p = in[12];
  V3<T> lt = ld3(in, 13);
  const V3<T> N = ld3(in, 16), TA = ld3(in, 19), TB = ld3(in, 22);
  const Q4<T> qA = ld4(in, 31), qB = ld4(in, 35);
  const T invN(m.invN);
  const bool hasT = lt.x != T(0.0) || lt.y != T(0.0) || lt.z != T(0.0);
  if (p != T(0.0) || hasT) {
    const V3<T> rAa = mul(ld3(in, 25), invN), rBa = mul(ld3(in, 28), invN);
    const V3<T> dc = m.hasB ? sub(rAa, rBa) : rAa;
    const T al = dot(N, dc);
    const T sgn = (al > T(0.0)) ? T(1.0) : T(-1.0);
    const T lam = -sgn * p;
    const V3<T> J = mul(N, lam);
    const T imA(m.imA), imB(m.imB);
    const V3<T> iIA = cv3<T>(m.iIA), iIB = cv3<T>(m.iIB);
    vA = add(vA, mul(J, imA));
    wA = add(wA, angResponse(qA, mul(TA, lam), iIA));
    if (m.hasB) {
      vB = add(vB, mul(neg(J), imB));
      wB = add(wB, angResponse(qB, mul(TB, lam), iIB));
    }
    if (hasT) {
      const T l2 = sqrt(dot(N, N));
      if (l2 > T(1e-9)) {
        const V3<T> nh = mul(N, T(1.0) / l2);
        lt = sub(lt, mul(nh, dot(lt, nh)));
      }
      vA = add(vA, mul(lt, imA));
      wA = add(wA, angResponse(qA, cross(rAa, lt), iIA));
      if (m.hasB) {
        vB = add(vB, mul(neg(lt), imB));
        wB = add(wB, angResponse(qB, cross(rBa, mul(lt, T(-1.0))), iIB));
      }
    }
  }
  st3(out, 0, vA);
  st3(out, 3, wA);
  st3(out, 6, vB);
  st3(out, 9, wB);
  st3(out, 12, lt);
}

// ---- one PGS update of a manifold (src/solver_velocity.hpp:641-858) -----------------------
// in: vA[0..3) wA[3..6) vB[6..9) wB[9..12) p[12] lt[13..16) geo[16..31) qA[31..35) qB[35..39)
//     vn0[39] vt0[40..43) posImp[43] eN[44] eT[45] mu[46]
// out: vA[0..3) wA[3..6) vB[6..9) wB[9..12) p[12] lt[13..16)
constexpr int kPgsIn = 47, kPgsOut = 16;
// `bits` (optional): the update's branch decisions, one bit each (the replay's branch signature)
template <class T>
PD void pgsMap(const T* in, T* out, const ManC& m, double vRest, unsigned* bits = nullptr) {
  const V3<T> vA = ld3(in, 0), wA = ld3(in, 3);
  const T invN(m.invN);
  V3<T> vB{T(0.0), T(0.0), T(0.0)}, wB{T(0.0), T(0.0), T(0.0)};
  if (m.hasB) {
    vB = ld3(in, 6);
    wB = ld3(in, 9);
  } else {
    vB = mul(cv3<T>(m.wv), invN);
  }
  const V3<T> N = ld3(in, 16), TA = ld3(in, 19), TB = ld3(in, 22);
  const V3<T> rAa = mul(ld3(in, 25), invN), rBa = mul(ld3(in, 28), invN);
  const V3<T> dc = m.hasB ? sub(rAa, rBa) : rAa;
  const Q4<T> qA = ld4(in, 31), qB = ld4(in, 35);
  const T vn0 = in[39];
  const T posImp = in[43];
  const T imA(m.imA), imB(m.imB);
  const V3<T> iIA = cv3<T>(m.iIA), iIB = cv3<T>(m.iIB);
  T pOld = in[12];
  V3<T> ltOld = ld3(in, 13);
  // outputs default to the inputs (an early return leaves the entry unchanged)
  for (int k = 0; k < 12; ++k)
    out[k] = in[k];
  out[12] = pOld;
  st3(out, 13, ltOld);
  T e = in[44];
  if (m.eAvg >= 0.0)
    e = T(m.eAvg);
  const T lenN = sqrt(dot(N, N));
  unsigned bb = 0;
  if (lenN < T(1e-9)) {
    if (bits)
      *bits = 1u;
    return;
  }
  const V3<T> vG = mul(dc, T(0.0));
  T vn = dot(vA, N) + dot(wA, TA) + dot(vB, neg(N)) + dot(wB, TB);
  vn += dot(vG, N);
  const T al = dot(N, dc);
  const T sgn = (al > T(0.0)) ? T(1.0) : T(-1.0);
  const T Nsq = dot(N, N);
  T wAn = Nsq * imA + genInvMass(TA, iIA, qA);
  T wBn = Nsq * imB + genInvMass(TB, iIB, qB);
  bool applyA = true, applyB = true;
  if (m.sf == 1) {
    wBn = T(0.0);
    applyB = false;
    e = T(0.0);
  } else if (m.sf == 2) {
    wAn = T(0.0);
    applyA = false;
    e = T(0.0);
  }
  const T wT = wAn + wBn;
  if (wT <= T(0.0)) {
    if (bits)
      *bits = 2u;
    return;
  }
  const T v0 = sgn * vn0;
  if (fabs(vn0) < T(vRest) * lenN) {
    e = T(0.0);
    bb |= 4u;
  }
  if (v0 > T(0.0))
    bb |= 8u;
  if (sgn > T(0.0))
    bb |= 16u;
  const T target = (v0 > T(0.0)) ? -e * v0 : T(0.0);
  const T vt = sgn * vn;
  const T dp = (vt - target) / wT;
  T pNew = pOld + dp;
  if (pNew < T(0.0)) {
    pNew = T(0.0);
    bb |= 32u;
  }
  const T dA = pNew - pOld;
  V3<T> vA2 = vA, wA2 = wA, vB2 = vB, wB2 = wB;
  T pCur = pOld;
  if (dA != T(0.0)) {
    bb |= 64u;
    pCur = pNew;
    const T lam = -sgn * dA;
    const V3<T> J = mul(N, lam), JA = mul(TA, lam), JB = mul(TB, lam);
    if (applyA) {
      vA2 = add(vA2, mul(J, imA));
      wA2 = add(wA2, angResponse(qA, JA, iIA));
    }
    if (m.hasB && applyB) {
      vB2 = add(vB2, mul(neg(J), imB));
      wB2 = add(wB2, angResponse(qB, JB, iIB));
    }
  }
  V3<T> ltCur = ltOld;
  T mu = in[46];
  if (m.muAvg >= 0.0)
    mu = T(m.muAvg);
  const bool haveOld = ltOld.x != T(0.0) || ltOld.y != T(0.0) || ltOld.z != T(0.0);
  if (mu > T(0.0) || haveOld) {
    bb |= 128u;
    const V3<T> nh = mul(N, T(1.0) / lenN);
    const V3<T> vBf = m.hasB ? vB2 : mul(cv3<T>(m.wv), invN);
    const V3<T> wBf = m.hasB ? wB2 : V3<T>{T(0.0), T(0.0), T(0.0)};
    const V3<T> vr = sub(add(vA2, cross(wA2, rAa)), add(vBf, cross(wBf, rBa)));
    const V3<T> vtv = sub(vr, mul(nh, dot(vr, nh)));
    T beta = in[45];
    if (beta != T(0.0) && (m.sf != 0 || fabs(vn0) < T(vRest) * lenN))
      beta = T(0.0);
    V3<T> err = vtv;
    if (beta != T(0.0)) {
      bb |= 256u;
      V3<T> w0 = ld3(in, 40);
      w0 = sub(w0, mul(nh, dot(w0, nh)));
      err = add(vtv, mul(w0, beta));
    }
    const T vl = sqrt(dot(err, err));
    V3<T> ltNew = ltOld;
    T wTt = imA + imB;
    if (vl > T(1e-9)) {
      bb |= 512u;
      const V3<T> th = mul(err, T(1.0) / vl);
      const T wAt = (m.sf == 2) ? T(0.0) : imA + genInvMass(cross(rAa, th), iIA, qA);
      const T wBt = (m.sf == 1 || !m.hasB) ? T(0.0) : imB + genInvMass(cross(rBa, th), iIB, qB);
      wTt = wAt + wBt;
      if (wTt > T(1e-9)) {
        bb |= 1024u;
        ltNew = add(ltOld, mul(th, -vl / wTt));
      }
    }
    ltNew = sub(ltNew, mul(nh, dot(ltNew, nh)));
    T nTot = fmax(pCur, T(0.0)) * lenN;
    if (fabs(vn0) < T(vRest) * lenN)
      nTot += fmax(posImp, T(0.0));
    if (posImp > T(0.0))
      bb |= 2048u;
    const T bound = mu * nTot;
    const T ll = sqrt(dot(ltNew, ltNew));
    if (ll > bound) {
      bb |= 4096u;
      ltNew = (bound > T(0.0)) ? mul(ltNew, bound / ll) : V3<T>{T(0.0), T(0.0), T(0.0)};
    }
    const V3<T> dd = sub(ltNew, ltOld);
    if (dd.x != T(0.0) || dd.y != T(0.0) || dd.z != T(0.0)) {
      bb |= 8192u;
      ltCur = ltNew;
      if (applyA) {
        vA2 = add(vA2, mul(dd, imA));
        wA2 = add(wA2, angResponse(qA, cross(rAa, dd), iIA));
      }
      if (m.hasB && applyB) {
        vB2 = add(vB2, mul(neg(dd), imB));
        wB2 = add(wB2, angResponse(qB, cross(rBa, mul(dd, T(-1.0))), iIB));
      }
    }
  }
  st3(out, 0, vA2);
  st3(out, 3, wA2);
  if (m.hasB) {
    st3(out, 6, vB2);
    st3(out, 9, wB2);
  }
  out[12] = pCur;
  st3(out, 13, ltCur);
  if (bits)
    *bits = bb | 16384u;
}

// ---- one position update of a contact (src/solver_position.hpp:55-99, :266-331) ------------
// in: xA[0..3) xB[3..6) qPA[6..10) qPB[10..14) qA[14..18) qB[18..22) n[22..25) rA[25..28) rB[28..31)
// out: xA[0..3) xB[3..6) dl[6]
constexpr int kPosIn = 31, kPosOut = 7;
struct PosC {
  bool hasB;
  double imA, imB;
  V3<double> iIA, iIB;
};
template <class T>
PD void posMap(const T* in, T* out, const PosC& c, unsigned* bits = nullptr) {
  const V3<T> pA = ld3(in, 0);
  V3<T> pB{T(0.0), T(0.0), T(0.0)};
  Q4<T> qB{T(0.0), T(0.0), T(0.0), T(1.0)};
  if (c.hasB) {
    pB = ld3(in, 3);
    qB = ld4(in, 10);
  }
  const Q4<T> qAd = qmul(ld4(in, 6), qinv(ld4(in, 14)));
  const V3<T> rA = rot(qAd, ld3(in, 25));
  V3<T> rB = ld3(in, 28);
  V3<T> n = ld3(in, 22);
  if (c.hasB) {
    const Q4<T> qBd = qmul(qB, qinv(ld4(in, 18)));
    rB = rot(qBd, rB);
    n = rot(qBd, n);
  }
  T C;
  if (!c.hasB)
    C = dot(sub(add(pA, rA), ld3(in, 28)), n);
  else
    C = dot(sub(add(pA, rA), add(pB, rB)), n);
  for (int k = 0; k < 6; ++k)
    out[k] = in[k];
  out[6] = T(0.0);
  if (bits)
    *bits = 1u;
  if (C >= T(0.0))
    return;
  const T imA(c.imA), imB(c.imB);
  const T wT = computeW(rA, n, imA, cv3<T>(c.iIA)) + computeW(rB, n, imB, cv3<T>(c.iIB));
  if (bits)
    *bits = 2u;
  if (wT < T(1e-6))
    return;
  if (bits)
    *bits = 4u;
  const T dl = -C / wT;
  st3(out, 0, add(pA, V3<T>{n.x * dl * imA, n.y * dl * imA, n.z * dl * imA}));
  if (c.hasB)
    st3(out, 3, add(pB, V3<T>{-n.x * dl * imB, -n.y * dl * imB, -n.z * dl * imB}));
  out[6] = dl;
}

// ---- velocity commit and position prediction (src/integration.hpp:112-148) ----------------
// in: x[0..3) q[3..7) vs[7..10) vf[10..13) w[13..16)   out: xP[0..3) qP[3..7)
constexpr int kIntIn = 16, kIntOut = 7;
template <class T>
PD void integrateMap(const T* in, T* out, double im, double dt) {
  V3<T> x = ld3(in, 0);
  const Q4<T> q = ld4(in, 3);
  const V3<T> w = ld3(in, 13);
  if (im > 0.0)
    x = add(x, mul(add(ld3(in, 7), ld3(in, 10)), T(0.5 * dt)));
  Q4<T> qp = q;
  if (im > 0.0) {
    const T h(0.5 * dt);
    qp.x = qp.x + h * (w.x * q.w + w.y * q.z - w.z * q.y);
    qp.y = qp.y + h * (w.y * q.w + w.z * q.x - w.x * q.z);
    qp.z = qp.z + h * (w.z * q.w + w.x * q.y - w.y * q.x);
    qp.w = qp.w + h * (-w.x * q.x - w.y * q.y - w.z * q.z);
    const T l = sqrt(qp.x * qp.x + qp.y * qp.y + qp.z * qp.z + qp.w * qp.w);
    if (l > T(1e-9)) {
      const T s = T(1.0) / l;
      qp = Q4<T>{qp.x * s, qp.y * s, qp.z * s, qp.w * s};
    }
  }
  st3(out, 0, x);
  st4(out, 3, qp);
}

// ---- hand-written reverse of the PGS update ---------------------------------------------------
// Vector-Jacobian products of the vector pieces (adjoints accumulate with +=):
//   c = a x b:          abar += b x cbar,  bbar += cbar x a
//   y = rot(q, v) = v + w t + qv x t, t = 2 qv x v:
//     vbar += ybar, wbar += t . ybar, tbar = w ybar + ybar x qv, qvbar += t x ybar,
//     then with ubar = 2 tbar (u = qv x v): qvbar += v x ubar, vbar += ubar x qv
//   invrot(q, v) = rot((-qv, w), v)
//   angResponse(q, J, iI) = rot(q, iI * invrot(q, J))
using V3d = V3<double>;
using Q4d = Q4<double>;
PD void acc(V3d& a, V3d b) { a.x += b.x, a.y += b.y, a.z += b.z; }
PD void acc(Q4d& a, Q4d b) { a.x += b.x, a.y += b.y, a.z += b.z, a.w += b.w; }
PD void crossVjp(V3d a, V3d b, V3d cb, V3d& ab, V3d& bb) {
  acc(ab, cross(b, cb));
  acc(bb, cross(cb, a));
}
PD void rotVjp(Q4d q, V3d v, V3d yb, Q4d& qb, V3d& vb) {
  const V3d qv{q.x, q.y, q.z};
  const V3d t = mul(cross(qv, v), 2.0);
  acc(vb, yb);
  qb.w += dot(t, yb);
  const V3d tb = add(mul(yb, q.w), cross(yb, qv));
  V3d qvb = cross(t, yb);
  const V3d ub = mul(tb, 2.0);
  acc(qvb, cross(v, ub));
  acc(vb, cross(ub, qv));
  qb.x += qvb.x, qb.y += qvb.y, qb.z += qvb.z;
}
PD void invrotVjp(Q4d q, V3d v, V3d yb, Q4d& qb, V3d& vb) {
  Q4d c{0.0, 0.0, 0.0, 0.0};
  rotVjp(Q4d{-q.x, -q.y, -q.z, q.w}, v, yb, c, vb);
  qb.x -= c.x, qb.y -= c.y, qb.z -= c.z, qb.w += c.w;
}
PD void angResponseVjp(Q4d q, V3d J, V3d iI, V3d yb, Q4d& qb, V3d& Jb) {
  const V3d u = invrot(q, J);
  const V3d sv{u.x * iI.x, u.y * iI.y, u.z * iI.z};
  V3d sb{0.0, 0.0, 0.0};
  rotVjp(q, sv, yb, qb, sb);
  invrotVjp(q, J, V3d{sb.x * iI.x, sb.y * iI.y, sb.z * iI.z}, qb, Jb);
}
// y = x - n (x . n):  xbar += ybar - n (n . ybar),  nbar += -(x . n) ybar - (n . ybar) x
PD void projVjp(V3d x, V3d n, V3d yb, V3d& xb, V3d& nb) {
  const double ny = dot(n, yb), xn = dot(x, n);
  acc(xb, sub(yb, mul(n, ny)));
  acc(nb, add(mul(yb, -xn), mul(x, -ny)));
}

// Reverse of pgsMap<double> (same inputs, outputs and branches); isotropic inverse inertia (the
// generalised inverse mass |tau|^2 iI does not depend on the orientation), as the adjoint's scope
// requires. xb += J^T yb.
PD void pgsRev(const double* in, const double* yb, double* xb, const ManC& m, double vRest) {
  // ---- forward, keeping what the reverse needs ----
  const V3d vA = ld3(in, 0), wA = ld3(in, 3);
  const double invN = m.invN;
  V3d vB{0.0, 0.0, 0.0}, wB{0.0, 0.0, 0.0};
  if (m.hasB) {
    vB = ld3(in, 6);
    wB = ld3(in, 9);
  } else {
    vB = mul(m.wv, invN);
  }
  const V3d N = ld3(in, 16), TA = ld3(in, 19), TB = ld3(in, 22);
  const V3d rAa = mul(ld3(in, 25), invN), rBa = mul(ld3(in, 28), invN);
  const V3d dc = m.hasB ? sub(rAa, rBa) : rAa;
  const Q4d qA = ld4(in, 31), qB = ld4(in, 35);
  const double vn0 = in[39], posImp = in[43];
  const double imA = m.imA, imB = m.imB;
  const V3d iIA = m.iIA, iIB = m.iIB;
  const double pOld = in[12];
  const V3d ltOld = ld3(in, 13);
  // adjoints of the outputs (identity when the update returns early)
  V3d vAb = ld3(yb, 0), wAb = ld3(yb, 3), vBb = ld3(yb, 6), wBb = ld3(yb, 9);
  double pb = yb[12];
  V3d ltb = ld3(yb, 13);
  auto flush = [&](V3d vab, V3d wab, V3d vbb, V3d wbb, double p0b, V3d lt0b) {
    xb[0] += vab.x, xb[1] += vab.y, xb[2] += vab.z;
    xb[3] += wab.x, xb[4] += wab.y, xb[5] += wab.z;
    if (m.hasB) {
      xb[6] += vbb.x, xb[7] += vbb.y, xb[8] += vbb.z;
      xb[9] += wbb.x, xb[10] += wbb.y, xb[11] += wbb.z;
    }
    xb[12] += p0b;
    xb[13] += lt0b.x, xb[14] += lt0b.y, xb[15] += lt0b.z;
  };
  double e = in[44];
  bool eFromN = true;
  if (m.eAvg >= 0.0) {
    e = m.eAvg;
    eFromN = false;
  }
  const double lenN = ::sqrt(dot(N, N));
  if (lenN < 1e-9) {
    flush(vAb, wAb, vBb, wBb, pb, ltb);
    return;
  }
  const double vn0N = dot(vA, N) + dot(wA, TA) + dot(vB, neg(N)) + dot(wB, TB);
  const double vn = vn0N + dot(mul(dc, 0.0), N);
  const double al = dot(N, dc);
  const double sgn = (al > 0.0) ? 1.0 : -1.0;
  const double Nsq = dot(N, N);
  double wAn = Nsq * imA + genInvMass(TA, iIA, qA);
  double wBn = Nsq * imB + genInvMass(TB, iIB, qB);
  bool applyA = true, applyB = true, useA = true, useB = true;
  if (m.sf == 1) {
    wBn = 0.0;
    applyB = false;
    useB = false;
    e = 0.0;
    eFromN = false;
  } else if (m.sf == 2) {
    wAn = 0.0;
    applyA = false;
    useA = false;
    e = 0.0;
    eFromN = false;
  }
  const double wT = wAn + wBn;
  if (wT <= 0.0) {
    flush(vAb, wAb, vBb, wBb, pb, ltb);
    return;
  }
  const double v0 = sgn * vn0;
  const bool rest = ::fabs(vn0) < vRest * lenN;
  if (rest) {
    e = 0.0;
    eFromN = false;
  }
  const bool tgt = v0 > 0.0;
  const double target = tgt ? -e * v0 : 0.0;
  const double vt = sgn * vn;
  const double dp = (vt - target) / wT;
  double pNew = pOld + dp;
  const bool clampN = pNew < 0.0;
  if (clampN)
    pNew = 0.0;
  const double dA = pNew - pOld;
  const bool act = dA != 0.0;
  V3d vA2 = vA, wA2 = wA, vB2 = vB, wB2 = wB;
  double pCur = pOld;
  const double lam = -sgn * dA;
  const V3d J = mul(N, lam), JA = mul(TA, lam), JB = mul(TB, lam);
  if (act) {
    pCur = pNew;
    if (applyA) {
      vA2 = add(vA2, mul(J, imA));
      wA2 = add(wA2, angResponse(qA, JA, iIA));
    }
    if (m.hasB && applyB) {
      vB2 = add(vB2, mul(neg(J), imB));
      wB2 = add(wB2, angResponse(qB, JB, iIB));
    }
  }
  double mu = in[46];
  bool muFromIn = true;
  if (m.muAvg >= 0.0) {
    mu = m.muAvg;
    muFromIn = false;
  }
  const bool haveOld = ltOld.x != 0.0 || ltOld.y != 0.0 || ltOld.z != 0.0;
  // accumulators of the input adjoints
  V3d vAi{0, 0, 0}, wAi{0, 0, 0}, vBi{0, 0, 0}, wBi{0, 0, 0}, lt0i{0, 0, 0};
  V3d Nb{0, 0, 0}, TAb{0, 0, 0}, TBb{0, 0, 0}, rAab{0, 0, 0}, rBab{0, 0, 0}, vt0b{0, 0, 0};
  Q4d qAb{0, 0, 0, 0}, qBb{0, 0, 0, 0};
  double p0b = 0.0, vn0b = 0.0, posImpb = 0.0, eNb = 0.0, eTb = 0.0, mub = 0.0, lenNb = 0.0;
  // adjoints of the velocities after the normal update and of pCur
  V3d vA2b = vAb, wA2b = wAb, vB2b = vBb, wB2b = wBb;
  double pCurb = pb;
  if (mu > 0.0 || haveOld) {
    const V3d nh = mul(N, 1.0 / lenN);
    const V3d vBf = m.hasB ? vB2 : mul(m.wv, invN);
    const V3d wBf = m.hasB ? wB2 : V3d{0.0, 0.0, 0.0};
    const V3d vr = sub(add(vA2, cross(wA2, rAa)), add(vBf, cross(wBf, rBa)));
    const V3d vtv = sub(vr, mul(nh, dot(vr, nh)));
    double beta = in[45];
    bool betaFromIn = true;
    if (beta != 0.0 && (m.sf != 0 || rest)) {
      beta = 0.0;
      betaFromIn = false;
    }
    V3d err = vtv;
    V3d w0p{0, 0, 0};
    const V3d vt0 = ld3(in, 40);
    if (beta != 0.0) {
      w0p = sub(vt0, mul(nh, dot(vt0, nh)));
      err = add(vtv, mul(w0p, beta));
    }
    const double vl = ::sqrt(dot(err, err));
    V3d ltNew = ltOld;
    double wTt = imA + imB;
    const bool vOn = vl > 1e-9;
    V3d th{0, 0, 0}, uA{0, 0, 0}, uB{0, 0, 0};
    bool wOn = false;
    if (vOn) {
      th = mul(err, 1.0 / vl);
      uA = cross(rAa, th);
      uB = cross(rBa, th);
      const double wAt = (m.sf == 2) ? 0.0 : imA + genInvMass(uA, iIA, qA);
      const double wBt = (m.sf == 1 || !m.hasB) ? 0.0 : imB + genInvMass(uB, iIB, qB);
      wTt = wAt + wBt;
      wOn = wTt > 1e-9;
      if (wOn)
        ltNew = add(ltOld, mul(th, -vl / wTt));
    }
    const V3d ltP = sub(ltNew, mul(nh, dot(ltNew, nh)));
    const bool pPos = !(0.0 > pCur);  // fmax(pCur, 0) takes pCur (also at 0)
    double nTot = (pPos ? pCur : 0.0) * lenN;
    const bool posOn = rest && !(0.0 > posImp);
    if (rest)
      nTot += (!(0.0 > posImp)) ? posImp : 0.0;
    const double bound = mu * nTot;
    const double ll = ::sqrt(dot(ltP, ltP));
    const bool cone = ll > bound;
    V3d ltC = ltP;
    if (cone)
      ltC = (bound > 0.0) ? mul(ltP, bound / ll) : V3d{0.0, 0.0, 0.0};
    const V3d dd = sub(ltC, ltOld);
    if (dd.x != 0.0 || dd.y != 0.0 || dd.z != 0.0) {
      // ---- reverse of the friction update ----
      V3d ddb = ltb;  // ltCur = ltC
      V3d ltCb{0, 0, 0};
      acc(ltCb, ltb);
      ddb = V3d{0, 0, 0};
      if (applyA) {
        acc(ddb, mul(vAb, imA));
        const V3d c = cross(rAa, dd);
        V3d cb{0, 0, 0};
        angResponseVjp(qA, c, iIA, wAb, qAb, cb);
        crossVjp(rAa, dd, cb, rAab, ddb);
      }
      if (m.hasB && applyB) {
        acc(ddb, mul(vBb, -imB));
        const V3d nd = mul(dd, -1.0);
        const V3d c = cross(rBa, nd);
        V3d cb{0, 0, 0}, ndb{0, 0, 0};
        angResponseVjp(qB, c, iIB, wBb, qBb, cb);
        crossVjp(rBa, nd, cb, rBab, ndb);
        acc(ddb, mul(ndb, -1.0));
      }
      acc(ltCb, ddb);
      acc(lt0i, mul(ddb, -1.0));
      // cone
      V3d ltPb{0, 0, 0};
      double boundb = 0.0;
      if (cone) {
        if (bound > 0.0) {
          const double sc = bound / ll;
          acc(ltPb, mul(ltCb, sc));
          const double scb = dot(ltCb, ltP);
          boundb += scb / ll;
          const double llb = -scb * bound / (ll * ll);
          if (ll > 0.0)
            acc(ltPb, mul(ltP, llb / ll));
        }
      } else {
        acc(ltPb, ltCb);
      }
      if (muFromIn)
        mub += boundb * nTot;
      const double nTotb = boundb * mu;
      if (pPos) {
        pCurb += nTotb * lenN;
        lenNb += nTotb * pCur;
      }
      if (posOn)
        posImpb += nTotb;
      // projection onto the tangent plane
      V3d ltNewb{0, 0, 0}, nhb{0, 0, 0};
      projVjp(ltNew, nh, ltPb, ltNewb, nhb);
      V3d errb{0, 0, 0};
      if (vOn && wOn) {
        const double k = -vl / wTt;
        acc(lt0i, ltNewb);
        V3d thb = mul(ltNewb, k);
        const double kb = dot(ltNewb, th);
        double vlb = -kb / wTt;
        const double wTtb = kb * vl / (wTt * wTt);
        if (m.sf != 2) {  // wAt = imA + |rAa x th|^2 iIA
          const V3d ub = mul(uA, 2.0 * iIA.x * wTtb);
          crossVjp(rAa, th, ub, rAab, thb);
        }
        if (!(m.sf == 1 || !m.hasB)) {
          const V3d ub = mul(uB, 2.0 * iIB.x * wTtb);
          crossVjp(rBa, th, ub, rBab, thb);
        }
        // th = err / vl
        acc(errb, mul(thb, 1.0 / vl));
        vlb += -dot(thb, err) / (vl * vl);
        acc(errb, mul(err, vlb / vl));
      } else {
        acc(lt0i, ltNewb);
      }
      V3d vtvb = errb;
      if (beta != 0.0) {
        const V3d w0pb = mul(errb, beta);
        const double betab = dot(errb, w0p);
        if (betaFromIn)
          eTb += betab;
        projVjp(vt0, nh, w0pb, vt0b, nhb);
      }
      V3d vrb{0, 0, 0};
      projVjp(vr, nh, vtvb, vrb, nhb);
      acc(vA2b, vrb);
      crossVjp(wA2, rAa, vrb, wA2b, rAab);
      if (m.hasB) {
        const V3d nvrb = mul(vrb, -1.0);
        acc(vB2b, nvrb);
        crossVjp(wB2, rBa, nvrb, wB2b, rBab);
      }
      // nh = N / lenN
      acc(Nb, mul(nhb, 1.0 / lenN));
      lenNb += -dot(nhb, N) / (lenN * lenN);
    } else {
      acc(lt0i, ltb);  // ltCur = ltOld
    }
  } else {
    acc(lt0i, ltb);
  }
  // ---- reverse of the normal update ----
  double dpb = 0.0;
  if (act) {
    double lamb = 0.0;
    if (applyA) {
      acc(vAi, vA2b);
      acc(Nb, mul(vA2b, lam * imA));  // J = N lam: Jbar = vA2b imA
      lamb += dot(vA2b, N) * imA;
      acc(wAi, wA2b);
      V3d JAb{0, 0, 0};
      angResponseVjp(qA, JA, iIA, wA2b, qAb, JAb);
      acc(TAb, mul(JAb, lam));
      lamb += dot(JAb, TA);
    } else {
      acc(vAi, vA2b);
      acc(wAi, wA2b);
    }
    if (m.hasB) {
      acc(vBi, vB2b);
      acc(wBi, wB2b);
      if (applyB) {
        acc(Nb, mul(vB2b, -lam * imB));
        lamb += -dot(vB2b, N) * imB;
        V3d JBb{0, 0, 0};
        angResponseVjp(qB, JB, iIB, wB2b, qBb, JBb);
        acc(TBb, mul(JBb, lam));
        lamb += dot(JBb, TB);
      }
    }
    const double dAb = -sgn * lamb;
    double pNewb = pCurb + dAb;
    p0b -= dAb;
    if (!clampN) {
      p0b += pNewb;
      dpb = pNewb;
    }
  } else {
    acc(vAi, vA2b);
    acc(wAi, wA2b);
    if (m.hasB) {
      acc(vBi, vB2b);
      acc(wBi, wB2b);
    }
    p0b += pCurb;
  }
  // dp = (vt - target) / wT
  const double vtb = dpb / wT;
  const double targetb = -dpb / wT;
  const double wTb = -dpb * dp / wT;
  const double vnb = sgn * vtb;
  if (tgt) {
    const double eb = -targetb * v0;
    if (eFromN)
      eNb += eb;
    vn0b += sgn * (-targetb * e);
  }
  double Nsqb = 0.0;
  if (useA) {
    Nsqb += wTb * imA;
    acc(TAb, mul(TA, 2.0 * iIA.x * wTb));
  }
  if (useB) {
    Nsqb += wTb * imB;
    acc(TBb, mul(TB, 2.0 * iIB.x * wTb));
  }
  acc(Nb, mul(N, 2.0 * Nsqb));
  // vn = vA . N + wA . TA - vB . N + wB . TB
  acc(vAi, mul(N, vnb));
  acc(wAi, mul(TA, vnb));
  acc(Nb, mul(sub(vA, vB), vnb));
  acc(TAb, mul(wA, vnb));
  if (m.hasB) {
    acc(vBi, mul(N, -vnb));
    acc(wBi, mul(TB, vnb));
    acc(TBb, mul(wB, vnb));
  }
  // lenN = |N|
  acc(Nb, mul(N, lenNb / lenN));
  // store
  flush(vAi, wAi, vBi, wBi, p0b, lt0i);
  xb[16] += Nb.x, xb[17] += Nb.y, xb[18] += Nb.z;
  xb[19] += TAb.x, xb[20] += TAb.y, xb[21] += TAb.z;
  xb[22] += TBb.x, xb[23] += TBb.y, xb[24] += TBb.z;
  xb[25] += rAab.x * invN, xb[26] += rAab.y * invN, xb[27] += rAab.z * invN;
  xb[28] += rBab.x * invN, xb[29] += rBab.y * invN, xb[30] += rBab.z * invN;
  xb[31] += qAb.x, xb[32] += qAb.y, xb[33] += qAb.z, xb[34] += qAb.w;
  xb[35] += qBb.x, xb[36] += qBb.y, xb[37] += qBb.z, xb[38] += qBb.w;
  xb[39] += vn0b;
  xb[40] += vt0b.x, xb[41] += vt0b.y, xb[42] += vt0b.z;
  xb[43] += posImpb;
  xb[44] += eNb;
  xb[45] += eTb;
  xb[46] += mub;
}

// ---- hand-written reverses of the approach velocity, the warm start and the position update -----
// Reverse of vn0Map<double>: xb += J^T yb (inputs and outputs as vn0Map's)
PD void vn0Rev(const double* in, const double* yb, double* xb, const ManC& m) {
  const V3d vA = ld3(in, 0), wA = ld3(in, 3);
  const double invN = m.invN;
  const V3d vB = m.hasB ? ld3(in, 6) : mul(m.wv, invN);
  const V3d wB = m.hasB ? ld3(in, 9) : V3d{0.0, 0.0, 0.0};
  const V3d N = ld3(in, 12), TA = ld3(in, 15), TB = ld3(in, 18);
  const V3d rAa = mul(ld3(in, 21), invN), rBa = mul(ld3(in, 24), invN);
  const double vnb = yb[0];
  const V3d vtb = ld3(yb, 1);
  V3d vAb = mul(N, vnb), wAb = mul(TA, vnb), vBb = mul(N, -vnb), wBb = mul(TB, vnb);
  V3d Nb = mul(sub(vA, vB), vnb), TAb = mul(wA, vnb), TBb = mul(wB, vnb), rAab{0, 0, 0}, rBab{0, 0, 0};
  const double lenN = ::sqrt(dot(N, N));
  if (lenN > 1e-9) {
    const V3d nh = mul(N, 1.0 / lenN);
    const V3d vr = sub(add(vA, cross(wA, rAa)), add(vB, cross(wB, rBa)));
    V3d vrb{0, 0, 0}, nhb{0, 0, 0};
    projVjp(vr, nh, vtb, vrb, nhb);
    acc(vAb, vrb);
    crossVjp(wA, rAa, vrb, wAb, rAab);
    const V3d nvrb = mul(vrb, -1.0);
    acc(vBb, nvrb);
    crossVjp(wB, rBa, nvrb, wBb, rBab);
    acc(Nb, mul(nhb, 1.0 / lenN));
    acc(Nb, mul(N, -dot(nhb, N) / (lenN * lenN * lenN)));
  }
  for (int k = 0; k < 3; ++k) {
    xb[k] += (&vAb.x)[k];
    xb[3 + k] += (&wAb.x)[k];
    if (m.hasB) {
      xb[6 + k] += (&vBb.x)[k];
      xb[9 + k] += (&wBb.x)[k];
    }
    xb[12 + k] += (&Nb.x)[k];
    xb[15 + k] += (&TAb.x)[k];
    xb[18 + k] += (&TBb.x)[k];
    xb[21 + k] += (&rAab.x)[k] * invN;
    xb[24 + k] += (&rBab.x)[k] * invN;
  }
}

// Reverse of warmMap<double> with respect to its non-velocity inputs (the velocities pass through
// with the identity, which the caller keeps): xb[12..39) += J^T yb
PD void warmRev(const double* in, const double* yb, double* xb, const ManC& m) {
  const double p = in[12];
  const V3d lt0 = ld3(in, 13);
  const V3d N = ld3(in, 16), TA = ld3(in, 19), TB = ld3(in, 22);
  const Q4d qA = ld4(in, 31), qB = ld4(in, 35);
  const double invN = m.invN;
  const V3d vAb = ld3(yb, 0), wAb = ld3(yb, 3), vBb = ld3(yb, 6), wBb = ld3(yb, 9);
  const V3d ltOutb = ld3(yb, 12);
  const bool hasT = lt0.x != 0.0 || lt0.y != 0.0 || lt0.z != 0.0;
  if (!(p != 0.0 || hasT)) {
    xb[13] += ltOutb.x, xb[14] += ltOutb.y, xb[15] += ltOutb.z;
    return;
  }
  const V3d rAa = mul(ld3(in, 25), invN), rBa = mul(ld3(in, 28), invN);
  const V3d dc = m.hasB ? sub(rAa, rBa) : rAa;
  const double sgn = (dot(N, dc) > 0.0) ? 1.0 : -1.0;
  const double lam = -sgn * p;
  const V3d JA = mul(TA, lam), JB = mul(TB, lam);
  V3d Nb{0, 0, 0}, TAb{0, 0, 0}, TBb{0, 0, 0}, rAab{0, 0, 0}, rBab{0, 0, 0}, lt0b{0, 0, 0};
  Q4d qAb{0, 0, 0, 0}, qBb{0, 0, 0, 0};
  double lamb = 0.0;
  // normal impulse
  {
    const V3d Jb = m.hasB ? sub(mul(vAb, m.imA), mul(vBb, m.imB)) : mul(vAb, m.imA);
    acc(Nb, mul(Jb, lam));
    lamb += dot(Jb, N);
    V3d JAb{0, 0, 0};
    angResponseVjp(qA, JA, m.iIA, wAb, qAb, JAb);
    acc(TAb, mul(JAb, lam));
    lamb += dot(JAb, TA);
    if (m.hasB) {
      V3d JBb{0, 0, 0};
      angResponseVjp(qB, JB, m.iIB, wBb, qBb, JBb);
      acc(TBb, mul(JBb, lam));
      lamb += dot(JBb, TB);
    }
  }
  if (hasT) {
    const double l2 = ::sqrt(dot(N, N));
    V3d lt1 = lt0, nh{0, 0, 0};
    if (l2 > 1e-9) {
      nh = mul(N, 1.0 / l2);
      lt1 = sub(lt0, mul(nh, dot(lt0, nh)));
    }
    V3d lt1b = ltOutb;
    acc(lt1b, mul(vAb, m.imA));
    {
      const V3d c = cross(rAa, lt1);
      V3d cb{0, 0, 0};
      angResponseVjp(qA, c, m.iIA, wAb, qAb, cb);
      crossVjp(rAa, lt1, cb, rAab, lt1b);
    }
    if (m.hasB) {
      acc(lt1b, mul(vBb, -m.imB));
      const V3d nd = mul(lt1, -1.0);
      const V3d c = cross(rBa, nd);
      V3d cb{0, 0, 0}, ndb{0, 0, 0};
      angResponseVjp(qB, c, m.iIB, wBb, qBb, cb);
      crossVjp(rBa, nd, cb, rBab, ndb);
      acc(lt1b, mul(ndb, -1.0));
    }
    if (l2 > 1e-9) {
      V3d nhb{0, 0, 0};
      projVjp(lt0, nh, lt1b, lt0b, nhb);
      acc(Nb, mul(nhb, 1.0 / l2));
      acc(Nb, mul(N, -dot(nhb, N) / (l2 * l2 * l2)));
    } else {
      acc(lt0b, lt1b);
    }
  } else {
    acc(lt0b, ltOutb);
  }
  xb[12] += -sgn * lamb;
  for (int k = 0; k < 3; ++k) {
    xb[13 + k] += (&lt0b.x)[k];
    xb[16 + k] += (&Nb.x)[k];
    xb[19 + k] += (&TAb.x)[k];
    xb[22 + k] += (&TBb.x)[k];
    xb[25 + k] += (&rAab.x)[k] * invN;
    xb[28 + k] += (&rBab.x)[k] * invN;
  }
  xb[31] += qAb.x, xb[32] += qAb.y, xb[33] += qAb.z, xb[34] += qAb.w;
  xb[35] += qBb.x, xb[36] += qBb.y, xb[37] += qBb.z, xb[38] += qBb.w;
}

// y = qmul(a, b): abar, bbar += (the transposed product)
PD void qmulVjp(Q4d a, Q4d b, Q4d y, Q4d& ab, Q4d& bb) {
  ab.x += y.x * b.w - y.y * b.z + y.z * b.y - y.w * b.x;
  ab.y += y.x * b.z + y.y * b.w - y.z * b.x - y.w * b.y;
  ab.z += -y.x * b.y + y.y * b.x + y.z * b.w - y.w * b.z;
  ab.w += y.x * b.x + y.y * b.y + y.z * b.z + y.w * b.w;
  bb.x += y.x * a.w + y.y * a.z - y.z * a.y - y.w * a.x;
  bb.y += -y.x * a.z + y.y * a.w + y.z * a.x - y.w * a.y;
  bb.z += y.x * a.y - y.y * a.x + y.z * a.w - y.w * a.z;
  bb.w += y.x * a.x + y.y * a.y + y.z * a.z + y.w * a.w;
}
// W = im + sum_k (r x d)_k^2 iI_k:  rbar, dbar += ...
PD void computeWVjp(V3d r, V3d d, V3d iI, double Wb, V3d& rb, V3d& db) {
  const V3d rn = cross(r, d);
  crossVjp(r, d, V3d{2.0 * rn.x * iI.x * Wb, 2.0 * rn.y * iI.y * Wb, 2.0 * rn.z * iI.z * Wb}, rb, db);
}

// Reverse of posMap<double>: xb += J^T yb
PD void posRev(const double* in, const double* yb, double* xb, const PosC& c) {
  const V3d pA = ld3(in, 0);
  const V3d pB = c.hasB ? ld3(in, 3) : V3d{0.0, 0.0, 0.0};
  const Q4d qPA = ld4(in, 6), qA0 = ld4(in, 14);
  const Q4d qPB = c.hasB ? ld4(in, 10) : Q4d{0.0, 0.0, 0.0, 1.0};
  const V3d nc = ld3(in, 22), rAc = ld3(in, 25), rBc = ld3(in, 28);
  const Q4d qAd = qmul(qPA, qinv(qA0));
  const V3d rA = rot(qAd, rAc);
  V3d rB = rBc, n = nc;
  Q4d qBd{0.0, 0.0, 0.0, 1.0};
  if (c.hasB) {
    qBd = qmul(qPB, qinv(ld4(in, 18)));
    rB = rot(qBd, rBc);
    n = rot(qBd, nc);
  }
  const V3d d = c.hasB ? sub(add(pA, rA), add(pB, rB)) : sub(add(pA, rA), rBc);
  const double C = dot(d, n);
  // the positions pass through (identity); dl and the updates only on the active branch
  xb[0] += yb[0], xb[1] += yb[1], xb[2] += yb[2];
  if (c.hasB)
    xb[3] += yb[3], xb[4] += yb[4], xb[5] += yb[5];
  if (C >= 0.0)
    return;
  const double wT = computeW(rA, n, c.imA, c.iIA) + computeW(rB, n, c.imB, c.iIB);
  if (wT < 1e-6)
    return;
  const double dl = -C / wT;
  const V3d pAb = ld3(yb, 0), pBb = c.hasB ? ld3(yb, 3) : V3d{0.0, 0.0, 0.0};
  double dlb = yb[6] + dot(pAb, n) * c.imA;
  V3d nb = mul(pAb, dl * c.imA);
  if (c.hasB) {
    dlb -= dot(pBb, n) * c.imB;
    acc(nb, mul(pBb, -dl * c.imB));
  }
  const double Cb = -dlb / wT;
  const double wTb = dlb * C / (wT * wT);
  V3d rAb{0, 0, 0}, rBb{0, 0, 0};
  computeWVjp(rA, n, c.iIA, wTb, rAb, nb);
  computeWVjp(rB, n, c.iIB, wTb, rBb, nb);
  // C = d . n
  acc(nb, mul(d, Cb));
  const V3d dn = mul(n, Cb);
  xb[0] += dn.x, xb[1] += dn.y, xb[2] += dn.z;
  acc(rAb, dn);
  V3d rBcb{0, 0, 0}, ncb{0, 0, 0};
  if (c.hasB) {
    xb[3] -= dn.x, xb[4] -= dn.y, xb[5] -= dn.z;
    acc(rBb, mul(dn, -1.0));
    Q4d qBdb{0, 0, 0, 0};
    rotVjp(qBd, nc, nb, qBdb, ncb);
    rotVjp(qBd, rBc, rBb, qBdb, rBcb);
    Q4d qPBb{0, 0, 0, 0}, qiBb{0, 0, 0, 0};
    const Q4d qB0 = ld4(in, 18);
    qmulVjp(qPB, qinv(qB0), qBdb, qPBb, qiBb);
    xb[10] += qPBb.x, xb[11] += qPBb.y, xb[12] += qPBb.z, xb[13] += qPBb.w;
    xb[18] -= qiBb.x, xb[19] -= qiBb.y, xb[20] -= qiBb.z, xb[21] += qiBb.w;
  } else {
    acc(rBcb, mul(dn, -1.0));
    acc(ncb, nb);
  }
  Q4d qAdb{0, 0, 0, 0};
  V3d rAcb{0, 0, 0};
  rotVjp(qAd, rAc, rAb, qAdb, rAcb);
  Q4d qPAb{0, 0, 0, 0}, qiAb{0, 0, 0, 0};
  qmulVjp(qPA, qinv(qA0), qAdb, qPAb, qiAb);
  xb[6] += qPAb.x, xb[7] += qPAb.y, xb[8] += qPAb.z, xb[9] += qPAb.w;
  xb[14] -= qiAb.x, xb[15] -= qiAb.y, xb[16] -= qiAb.z, xb[17] += qiAb.w;
  xb[22] += ncb.x, xb[23] += ncb.y, xb[24] += ncb.z;
  xb[25] += rAcb.x, xb[26] += rAcb.y, xb[27] += rAcb.z;
  xb[28] += rBcb.x, xb[29] += rBcb.y, xb[30] += rBcb.z;
}

// ---- one chunk of a vector-Jacobian product -------------------------------------------------
// part[l] = sum_o ybar[o] d out[o] / d in[chunk kLanes + l]: the threads of a group each take one
// chunk of the inputs, so the chunks of one entry run side by side
constexpr int kGroup = 8;  // 8 chunks of kLanes cover up to 56 inputs
template <int NI, int NO, class F>
__device__ __forceinline__ void vjpChunk(const double* in, const double* ybar, double* part, int chunk, F f) {
  using D = Dd<kLanes>;
  const int c0 = chunk * kLanes;
  D x[NI];
  D y[NO];
  for (int i = 0; i < NI; ++i) {
    x[i] = D(in[i]);
    const int l = i - c0;
    if (l >= 0 && l < kLanes)
      x[i].d[l] = 1.0;
  }
  f(x, y);
  for (int l = 0; l < kLanes; ++l) {
    double s = 0.0;
    for (int o = 0; o < NO; ++o)
      s += ybar[o] * y[o].d[l];
    part[l] = s;
  }
}

// ---- vector-Jacobian product of a local map by forward-mode chunks ------------------------
// xbar[i] += sum_o ybar[o] d out[o] / d in[i]; `f(in, out)` is the map on Dd<kLanes> scalars.
template <int NI, int NO, class F>
__device__ __forceinline__ void vjp(const double* in, const double* ybar, double* xbar, F f) {
  using D = Dd<kLanes>;
  for (int c0 = 0; c0 < NI; c0 += kLanes) {
    D x[NI];
    D y[NO];
    for (int i = 0; i < NI; ++i) {
      x[i] = D(in[i]);
      const int l = i - c0;
      if (l >= 0 && l < kLanes)
        x[i].d[l] = 1.0;
    }
    f(x, y);
    for (int l = 0; l < kLanes && c0 + l < NI; ++l) {
      double s = 0.0;
      for (int o = 0; o < NO; ++o)
        s += ybar[o] * y[o].d[l];
      xbar[c0 + l] += s;
    }
  }
}

}  // namespace xadj
}  // namespace pdem
