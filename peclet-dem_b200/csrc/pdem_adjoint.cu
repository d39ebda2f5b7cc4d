// Forward and hand-written adjoint of the explicit Hertz-Mindlin substep for spheres, for
// differentiable calibration: gradients of a loss on the final state with respect to Young's
// modulus E, the restitution e, the friction mu and the initial state.
//
// The force law is the Hertz engine's (src/solver_hertz.hpp:88-144 for sphere pairs, the same law
// against a wall at rest for the planes, src/solver_hertz.hpp:300-372), the integration its
// symplectic kick-drift (src/solver_hertz.hpp:374-425) without orientation update:
//   per pair (i, j) with overlap d = r_i + r_j - |x_i - x_j| > 0: force f(d, n, v_rel, xi; E, e, mu)
//   and the new Mindlin history xi' (hertzForce, shared with the engine), torques r_A x f on i and
//   r_B x (-f) on j; per sphere and plane the same law with the plane at rest; then
//   v' = v + (F / m + g) dt, w' = w + T / I dt, x' = x + v' dt.
// The pair list is fixed over a window of substeps (the caller builds it with a skin at each window
// start); plane contacts are evaluated for every (sphere, plane).
//
// State of a substep (one contiguous block): x, v, w (3 n each), pair histories (3 per pair),
// plane histories (3 per sphere and plane). The forward stores every substep of a window (or
// ping-pongs two states); the backward walks the stored window in reverse.
//
// Adjoint of one substep, given the adjoint of S_{k+1}: the integration is linear and reversed by
// hand; each contact's local Jacobian (outputs: force, torques, new history; inputs: relative
// position, relative velocity, both spins, history, E, e, mu) is taken in forward mode with dual
// numbers through the same hertzForce the forward runs (so the recorded active set and friction
// branch are exactly the forward's), and its transpose is applied to the outputs' adjoints.
// Accumulation into bodies and parameters uses atomics, so gradients are summed in an unspecified
// order (forward forces too: the forward is deterministic only up to that summation order).
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "../../include/pdem.h"
#include "pdem_hertz.cuh"

namespace pdem {
void setLastError(const std::string& msg);  // pdem_capi.cu
}

namespace {

using pdem::V3;
using std::fabs;  // the plain overloads stay visible beside the dual-number ones below
using std::log;
using std::sqrt;

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

// material stars of one material against itself (hertzStars with E_i = E_j, nu_i = nu_j)
template <class T>
__device__ void stars(T E, double nu, T& eS, T& gS) {
  const T one(1.0), two(2.0), a(1.0 - nu * nu), b((2.0 - nu) * (1.0 + nu));
  eS = one / (a / E + a / E);
  gS = one / (two * b / E + two * b / E);
}

// sphere pair: in = dx(3) dv(3) wi(3) wj(3) xi(3) E e mu; out = f(3) Ti(3) Tj(3) xi'(3).
// Returns false (no force, history cleared) when the spheres do not overlap.
constexpr int kPairIn = 18, kPairOut = 12, kPlaneIn = 15, kPlaneOut = 9;
template <class T, class S>
__device__ bool pairLaw(const T* in, S ri, S rj, S mS, double nu, S dt, T* out) {
  const V3<T> dx{in[0], in[1], in[2]}, dv{in[3], in[4], in[5]}, wi{in[6], in[7], in[8]}, wj{in[9], in[10], in[11]};
  V3<T> xi{in[12], in[13], in[14]};
  const T dd = sqrt(pdem::dot(dx, dx));
  const T delta = T(ri + rj) - dd;
  if (delta <= T(0.0) || dd < T(1e-12))
    return false;
  const V3<T> nh = pdem::mul(dx, T(1.0) / dd);
  const V3<T> rA = pdem::mul(nh, -(T(ri) - T(0.5) * delta));
  const V3<T> rB = pdem::mul(nh, T(rj) - T(0.5) * delta);
  const V3<T> vr = pdem::sub(pdem::add(dv, pdem::cross(wi, rA)), pdem::cross(wj, rB));
  T eS, gS;
  stars(in[15], nu, eS, gS);
  const V3<T> f = pdem::hertzForce(delta, nh, vr, T(ri * rj / (ri + rj)), T(mS), eS, gS, in[16], in[17], T(dt), xi);
  const V3<T> ti = pdem::cross(rA, f), tj = pdem::cross(rB, pdem::mul(f, T(-1.0)));
  out[0] = f.x, out[1] = f.y, out[2] = f.z;
  out[3] = ti.x, out[4] = ti.y, out[5] = ti.z;
  out[6] = tj.x, out[7] = tj.y, out[8] = tj.z;
  out[9] = xi.x, out[10] = xi.y, out[11] = xi.z;
  return true;
}
// sphere on plane (point p0, unit normal n into the domain): in = x(3) v(3) w(3) xi(3) E e mu;
// out = f(3) T(3) xi'(3)
template <class T, class S>
__device__ bool planeLaw(const T* in, const S* pl, S ri, S mi, double nu, S dt, T* out) {
  const V3<T> x{in[0], in[1], in[2]}, v{in[3], in[4], in[5]}, w{in[6], in[7], in[8]};
  V3<T> xi{in[9], in[10], in[11]};
  const V3<T> p0{T(pl[0]), T(pl[1]), T(pl[2])}, n{T(pl[3]), T(pl[4]), T(pl[5])};
  const T delta = T(ri) - pdem::dot(pdem::sub(x, p0), n);
  if (delta <= T(0.0))
    return false;
  const V3<T> rA = pdem::mul(n, -(T(ri) - T(0.5) * delta));
  const V3<T> vr = pdem::add(v, pdem::cross(w, rA));
  T eS, gS;
  stars(in[12], nu, eS, gS);
  const V3<T> f = pdem::hertzForce(delta, n, vr, T(ri), T(mi), eS, gS, in[13], in[14], T(dt), xi);
  const V3<T> t = pdem::cross(rA, f);
  out[0] = f.x, out[1] = f.y, out[2] = f.z;
  out[3] = t.x, out[4] = t.y, out[5] = t.z;
  out[6] = xi.x, out[7] = xi.y, out[8] = xi.z;
  return true;
}

template <class R>
struct StateView {
  R *x, *v, *w, *xiP, *xiW;  // xiP: 3 per pair, xiW: 3 per (sphere, plane), sphere-major
};
inline size_t stateSize(long n, long npair, long nplane) { return (size_t)(9 * n + 3 * npair + 3 * n * nplane); }
template <class R>
StateView<R> view(R* base, long n, long npair) {
  StateView<R> s;
  s.x = base;
  s.v = base + 3 * n;
  s.w = base + 6 * n;
  s.xiP = base + 9 * n;
  s.xiW = s.xiP + 3 * npair;
  return s;
}

template <class R>
struct Model {
  int n, npair, nplane;
  const int* pairs;  // [npair] (i, j), i < j
  const R *planes, *r, *m, *I;
  R E, e, mu, dt, g[3];
  double nu;
};

// ---- forward ----
template <class R>
__global__ void kPairForces(Model<R> M, StateView<R> s, StateView<R> t, R* F, R* T) {
  GRID_STRIDE(p, M.npair) {
    const int i = M.pairs[2 * p], j = M.pairs[2 * p + 1];
    R in[kPairIn], out[kPairOut];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      in[a] = s.x[3 * i + a] - s.x[3 * j + a];
      in[3 + a] = s.v[3 * i + a] - s.v[3 * j + a];
      in[6 + a] = s.w[3 * i + a];
      in[9 + a] = s.w[3 * j + a];
      in[12 + a] = s.xiP[3 * p + a];
    }
    in[15] = M.E, in[16] = M.e, in[17] = M.mu;
    const R mS = R(1) / (R(1) / M.m[i] + R(1) / M.m[j]);
    if (!pairLaw<R, R>(in, M.r[i], M.r[j], mS, M.nu, M.dt, out)) {
      t.xiP[3 * p] = t.xiP[3 * p + 1] = t.xiP[3 * p + 2] = R(0);
      continue;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      atomicAdd(&F[3 * i + a], out[a]);
      atomicAdd(&F[3 * j + a], -out[a]);
      atomicAdd(&T[3 * i + a], out[3 + a]);
      atomicAdd(&T[3 * j + a], out[6 + a]);
      t.xiP[3 * p + a] = out[9 + a];
    }
  }
}
// plane contacts and the kick-drift of each sphere (one thread per sphere, planes in order)
template <class R>
__global__ void kPlanesIntegrate(Model<R> M, StateView<R> s, StateView<R> t, const R* F, const R* T) {
  GRID_STRIDE(i, M.n) {
    R f[3] = {F[3 * i], F[3 * i + 1], F[3 * i + 2]}, tq[3] = {T[3 * i], T[3 * i + 1], T[3 * i + 2]};
    const R ri = M.r[i], mi = M.m[i];
    for (int k = 0; k < M.nplane; ++k) {
      const long q = i * M.nplane + k;
      R in[kPlaneIn], out[kPlaneOut];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        in[a] = s.x[3 * i + a];
        in[3 + a] = s.v[3 * i + a];
        in[6 + a] = s.w[3 * i + a];
        in[9 + a] = s.xiW[3 * q + a];
      }
      in[12] = M.E, in[13] = M.e, in[14] = M.mu;
      if (!planeLaw<R, R>(in, M.planes + 6 * k, ri, mi, M.nu, M.dt, out)) {
        t.xiW[3 * q] = t.xiW[3 * q + 1] = t.xiW[3 * q + 2] = R(0);
        continue;
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        f[a] += out[a];
        tq[a] += out[3 + a];
        t.xiW[3 * q + a] = out[6 + a];
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const R v = s.v[3 * i + a] + (f[a] / mi + M.g[a]) * M.dt;
      t.v[3 * i + a] = v;
      t.w[3 * i + a] = s.w[3 * i + a] + tq[a] / M.I[i] * M.dt;
      t.x[3 * i + a] = s.x[3 * i + a] + v * M.dt;
    }
  }
}

// ---- adjoint ----
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
// Integration: b0.{x,v,w} = b1 carried back through x' = x + v' dt, v' = v + ..., w' = w + ...;
// Fb, Tb = adjoints of the substep's force and torque sums. Plane contacts are reversed here too
// (one thread per sphere) into b0 and the plane history adjoints. Warps iterate in lockstep so the
// parameter sums can be reduced with shuffles.
template <class R, class S>
__global__ void kIntegratePlanesAdj(Model<R> M, StateView<R> s, StateView<R> b1, StateView<R> b0, R* Fb, R* Tb,
                                    double* thetaB) {
  double gE = 0, ge = 0, gmu = 0;
  const long n = M.n;
  for (long i0 = (long)blockIdx.x * blockDim.x + threadIdx.x - (threadIdx.x & 31); i0 < n;
       i0 += (long)gridDim.x * blockDim.x) {
    const long i = i0 + (threadIdx.x & 31);
    if (i < n) {
      R xb[3], vb[3], wb[3], fb[3], tb[3];
      const R mi = M.m[i], ri = M.r[i];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const R vbt = b1.v[3 * i + a] + M.dt * b1.x[3 * i + a];  // v' feeds x' = x + v' dt
        xb[a] = b1.x[3 * i + a];
        vb[a] = vbt;
        wb[a] = b1.w[3 * i + a];
        fb[a] = vbt * M.dt / mi;
        tb[a] = b1.w[3 * i + a] * M.dt / M.I[i];
        Fb[3 * i + a] = fb[a];
        Tb[3 * i + a] = tb[a];
      }
      for (int k = 0; k < M.nplane; ++k) {
        const long q = i * M.nplane + k;
        // contact test on plain values first: an inactive contact has a zero Jacobian apart from
        // the cleared history, whose adjoint is zero
        const R* pl = M.planes + 6 * k;
        const R dist =
            (s.x[3 * i] - pl[0]) * pl[3] + (s.x[3 * i + 1] - pl[1]) * pl[4] + (s.x[3 * i + 2] - pl[2]) * pl[5];
        if (!(ri - dist > R(0))) {
          b0.xiW[3 * q] = b0.xiW[3 * q + 1] = b0.xiW[3 * q + 2] = R(0);
          continue;
        }
        Dn<S, kPlaneIn> in[kPlaneIn], out[kPlaneOut];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          in[a] = Dn<S, kPlaneIn>(s.x[3 * i + a]);
          in[3 + a] = Dn<S, kPlaneIn>(s.v[3 * i + a]);
          in[6 + a] = Dn<S, kPlaneIn>(s.w[3 * i + a]);
          in[9 + a] = Dn<S, kPlaneIn>(s.xiW[3 * q + a]);
        }
        in[12] = Dn<S, kPlaneIn>(M.E), in[13] = Dn<S, kPlaneIn>(M.e), in[14] = Dn<S, kPlaneIn>(M.mu);
#pragma unroll
        for (int c = 0; c < kPlaneIn; ++c)
          in[c].d[c] = S(1);
        if (!planeLaw<Dn<S, kPlaneIn>, R>(in, pl, ri, mi, M.nu, M.dt, out)) {
          b0.xiW[3 * q] = b0.xiW[3 * q + 1] = b0.xiW[3 * q + 2] = R(0);
          continue;
        }
        S yb[kPlaneOut];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          yb[a] = fb[a];
          yb[3 + a] = tb[a];
          yb[6 + a] = b1.xiW[3 * q + a];
        }
        S cb[kPlaneIn];
#pragma unroll
        for (int c = 0; c < kPlaneIn; ++c) {
          S acc = 0;
#pragma unroll
          for (int o = 0; o < kPlaneOut; ++o)
            acc += out[o].d[c] * yb[o];
          cb[c] = acc;
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          xb[a] += R(cb[a]);
          vb[a] += R(cb[3 + a]);
          wb[a] += R(cb[6 + a]);
          b0.xiW[3 * q + a] = R(cb[9 + a]);
        }
        gE += cb[12], ge += cb[13], gmu += cb[14];
      }
      // pair contributions are added to b0.{x,v,w} with atomics by kPairAdj, which runs after this
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        b0.x[3 * i + a] = xb[a];
        b0.v[3 * i + a] = vb[a];
        b0.w[3 * i + a] = wb[a];
      }
    }
  }
  flushParams(thetaB, gE, ge, gmu);
}
template <class R, class S>
__global__ void kPairAdj(Model<R> M, StateView<R> s, StateView<R> b1, StateView<R> b0, const R* Fb, const R* Tb,
                         double* thetaB) {
  double gE = 0, ge = 0, gmu = 0;
  for (long p0 = (long)blockIdx.x * blockDim.x + threadIdx.x - (threadIdx.x & 31); p0 < M.npair;
       p0 += (long)gridDim.x * blockDim.x) {
    const long p = p0 + (threadIdx.x & 31);
    if (p < M.npair) {
      const int i = M.pairs[2 * p], j = M.pairs[2 * p + 1];
      const R ri = M.r[i], rj = M.r[j];
      R dx[3];
#pragma unroll
      for (int a = 0; a < 3; ++a)
        dx[a] = s.x[3 * i + a] - s.x[3 * j + a];
      const R dd = ::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      if (!(ri + rj - dd > R(0)) || dd < R(1e-12)) {
        b0.xiP[3 * p] = b0.xiP[3 * p + 1] = b0.xiP[3 * p + 2] = R(0);
        continue;
      }
      Dn<S, kPairIn> in[kPairIn], out[kPairOut];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        in[a] = Dn<S, kPairIn>(dx[a]);
        in[3 + a] = Dn<S, kPairIn>(s.v[3 * i + a] - s.v[3 * j + a]);
        in[6 + a] = Dn<S, kPairIn>(s.w[3 * i + a]);
        in[9 + a] = Dn<S, kPairIn>(s.w[3 * j + a]);
        in[12 + a] = Dn<S, kPairIn>(s.xiP[3 * p + a]);
      }
      in[15] = Dn<S, kPairIn>(M.E), in[16] = Dn<S, kPairIn>(M.e), in[17] = Dn<S, kPairIn>(M.mu);
#pragma unroll
      for (int k = 0; k < kPairIn; ++k)
        in[k].d[k] = S(1);
      const R mS = R(1) / (R(1) / M.m[i] + R(1) / M.m[j]);
      if (!pairLaw<Dn<S, kPairIn>, R>(in, ri, rj, mS, M.nu, M.dt, out)) {
        b0.xiP[3 * p] = b0.xiP[3 * p + 1] = b0.xiP[3 * p + 2] = R(0);
        continue;
      }
      S yb[kPairOut];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        yb[a] = Fb[3 * i + a] - Fb[3 * j + a];  // f acts on i, -f on j
        yb[3 + a] = Tb[3 * i + a];
        yb[6 + a] = Tb[3 * j + a];
        yb[9 + a] = b1.xiP[3 * p + a];
      }
      S cb[kPairIn];
#pragma unroll
      for (int k = 0; k < kPairIn; ++k) {
        S acc = 0;
#pragma unroll
        for (int o = 0; o < kPairOut; ++o)
          acc += out[o].d[k] * yb[o];
        cb[k] = acc;
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        atomicAdd(&b0.x[3 * i + a], R(cb[a]));
        atomicAdd(&b0.x[3 * j + a], R(-cb[a]));
        atomicAdd(&b0.v[3 * i + a], R(cb[3 + a]));
        atomicAdd(&b0.v[3 * j + a], R(-cb[3 + a]));
        atomicAdd(&b0.w[3 * i + a], R(cb[6 + a]));
        atomicAdd(&b0.w[3 * j + a], R(cb[9 + a]));
        b0.xiP[3 * p + a] = R(cb[12 + a]);
      }
      gE += cb[15], ge += cb[16], gmu += cb[17];
    }
  }
  flushParams(thetaB, gE, ge, gmu);
}

// candidate pairs within scenes: i < j < end[i] (end = exclusive end of i's scene range),
// |x_i - x_j| < r_i + r_j + skin; pass 1 counts per sphere, pass 2 writes at off[i]
template <class R>
__global__ void kCandPairs(const R* x, const R* r, const int* end, int n, R skin, int* cnt, const int* off,
                           int* out) {
  GRID_STRIDE(i, n) {
    int c = 0;
    const int base = off ? off[i] : 0;
    const int last = end ? end[i] : n;
    const R xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2], ri = r[i];
    for (int j = (int)i + 1; j < last; ++j) {
      const R dx = xi - x[3 * j], dy = yi - x[3 * j + 1], dz = zi - x[3 * j + 2];
      const R lim = ri + r[j] + skin;
      if (dx * dx + dy * dy + dz * dz < lim * lim) {
        if (off) {
          out[2 * (base + c)] = (int)i;
          out[2 * (base + c) + 1] = j;
        }
        ++c;
      }
    }
    if (!off)
      cnt[i] = c;
  }
}

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
  if (!h || h->n < 0 || h->npair < 0 || h->nplane < 0)
    throw Fail{PDEM_ERR_INVALID, "hz model: negative sizes"};
  if (h->n > 0 && (!h->radius || !h->mass || !h->inertia))
    throw Fail{PDEM_ERR_INVALID, "hz model: radius, mass and inertia are required"};
  if ((h->npair > 0 && !h->pairs) || (h->nplane > 0 && !h->planes))
    throw Fail{PDEM_ERR_INVALID, "hz model: pair list or planes missing"};
  if (!(h->youngs > 0) || !(h->dt > 0))
    throw Fail{PDEM_ERR_INVALID, "hz model: Young's modulus and dt must be positive"};
  Model<R> M;
  M.n = h->n, M.npair = h->npair, M.nplane = h->nplane, M.pairs = h->pairs;
  M.planes = static_cast<const R*>(h->planes);
  M.r = static_cast<const R*>(h->radius);
  M.m = static_cast<const R*>(h->mass);
  M.I = static_cast<const R*>(h->inertia);
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
  const size_t S = stateSize(M.n, M.npair, M.nplane);
  R* F = work;
  R* T = work + 3 * (size_t)M.n;
  for (int k = 0; k < steps; ++k) {
    const size_t a = store ? k : (k & 1), b = store ? k + 1 : ((k + 1) & 1);
    const StateView<R> s = view(traj + S * a, M.n, M.npair), t = view(traj + S * b, M.n, M.npair);
    check(cudaMemsetAsync(F, 0, 6 * (size_t)M.n * sizeof(R), st), "memset");
    if (M.npair > 0)
      kPairForces<R><<<pdem::gridFor(M.npair), pdem::kBlock, 0, st>>>(M, s, t, F, T);
    kPlanesIntegrate<R><<<pdem::gridFor(M.n), pdem::kBlock, 0, st>>>(M, s, t, F, T);
  }
  if (!store && (steps & 1) == 0)  // the final state of a ping-pong run always ends in slot 1
    check(cudaMemcpyAsync(traj + S, traj, S * sizeof(R), cudaMemcpyDeviceToDevice, st), "D2D");
  check(cudaGetLastError(), "hz forward");
}

template <class R, class S>
void backward(const pdem_hz_model* h, int steps, const R* traj, R* adj, double* thetaB, R* work, cudaStream_t st) {
  const Model<R> M = makeModel<R>(h);
  if (steps <= 0 || M.n == 0)
    return;
  if (!traj || !adj || !work)
    throw Fail{PDEM_ERR_INVALID, "hz backward: trajectory, adjoint or work buffer missing"};
  const size_t SZ = stateSize(M.n, M.npair, M.nplane);
  R* Fb = work;
  R* Tb = work + 3 * (size_t)M.n;
  R* other = work + 6 * (size_t)M.n;  // second adjoint state, ping-pong with adj
  R* cur = adj;
  for (int k = steps - 1; k >= 0; --k) {
    const StateView<R> s = view(const_cast<R*>(traj) + SZ * k, M.n, M.npair);
    const StateView<R> b1 = view(cur, M.n, M.npair), b0 = view(other, M.n, M.npair);
    kIntegratePlanesAdj<R, S><<<pdem::gridFor(M.n), pdem::kBlock, 0, st>>>(M, s, b1, b0, Fb, Tb, thetaB);
    if (M.npair > 0)
      kPairAdj<R, S><<<pdem::gridFor(M.npair), pdem::kBlock, 0, st>>>(M, s, b1, b0, Fb, Tb, thetaB);
    std::swap(cur, other);
  }
  if (cur != adj)
    check(cudaMemcpyAsync(adj, cur, SZ * sizeof(R), cudaMemcpyDeviceToDevice, st), "D2D");
  check(cudaGetLastError(), "hz backward");
}

template <class R>
void pairs(const R* x, const R* r, const int* end, int n, double skin, int* cnt, int* off, int* out, long cap,
           long* count, cudaStream_t st) {
  *count = 0;
  if (n < 2)
    return;
  kCandPairs<R><<<pdem::gridFor(n), pdem::kBlock, 0, st>>>(x, r, end, n, R(skin), cnt, nullptr, nullptr);
  check(cudaGetLastError(), "hz pair count");
  std::vector<int> c(n), o(n + 1, 0);
  check(cudaMemcpyAsync(c.data(), cnt, n * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  check(cudaStreamSynchronize(st), "sync");
  for (int i = 0; i < n; ++i)
    o[i + 1] = o[i] + c[i];
  *count = o[n];
  if (o[n] > cap || o[n] == 0)
    return;
  check(cudaMemcpyAsync(off, o.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
  kCandPairs<R><<<pdem::gridFor(n), pdem::kBlock, 0, st>>>(x, r, end, n, R(skin), nullptr, off, out);
  check(cudaGetLastError(), "hz pair write");
  check(cudaStreamSynchronize(st), "sync");  // o is released on return
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

long pdem_hz_state_size(int n, int npair, int nplane) {
  return (n < 0 || npair < 0 || nplane < 0) ? -1 : (long)stateSize(n, npair, nplane);
}
long pdem_hz_work_size(int n, int npair, int nplane) {
  return (n < 0 || npair < 0 || nplane < 0) ? -1 : (long)(6 * (size_t)n + stateSize(n, npair, nplane));
}

int pdem_hz_pairs(int precision, const void* d_x, const void* d_radius, const int* d_end, int n, double skin,
                  int* d_cnt, int* d_off, int* d_pairs, long cap, long* count, void* stream) {
  return guarded([&] {
    if (!count || n < 0)
      throw Fail{PDEM_ERR_INVALID, "hz pairs: bad arguments"};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precisionOf(precision) == 64)
      pairs<double>(static_cast<const double*>(d_x), static_cast<const double*>(d_radius), d_end, n, skin, d_cnt, d_off,
                    d_pairs, cap, count, st);
    else
      pairs<float>(static_cast<const float*>(d_x), static_cast<const float*>(d_radius), d_end, n, skin, d_cnt, d_off,
                   d_pairs, cap, count, st);
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
                     double* d_grad, void* d_work, void* stream) {
  return guarded([&] {
    if (!d_grad)
      throw Fail{PDEM_ERR_INVALID, "hz backward: parameter gradient buffer missing"};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precisionOf(precision) == 64)
      backward<double, double>(model, steps, static_cast<const double*>(d_traj), static_cast<double*>(d_adj), d_grad,
                               static_cast<double*>(d_work), st);
    else
      backward<float, float>(model, steps, static_cast<const float*>(d_traj), static_cast<float*>(d_adj), d_grad,
                             static_cast<float*>(d_work), st);
  });
}

}  // extern "C"
