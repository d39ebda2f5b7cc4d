// Multilevel stabilization pass (the reference's "multilevel" stabilization mode: src/sim.hpp:303-356,
// src/solver_multilevel.hpp). Greedy pairwise aggregation of the quasi-static contact graph into
// super-bodies over up to 10 levels, per level a colouring of the manifolds that cross aggregate
// boundaries (one 6-bit slot per level in a packed word, 63 = skipped), then per iteration one fine
// projected GS sweep and, on every level, restriction to momentum-weighted group velocities, two
// translation-only coarse PGS sweeps at the aggregate masses on the shared normal accumulator, and
// prolongation; the loop ends on the quasi-static residual.
//
// Every decision of the build is order-free (maxima of the manifolds' colour keys, as in the
// colouring), so it runs in parallel. The sums of the reference (group masses and momenta, float
// atomics there, ascending body order on its serial build) run in that order in one thread: this is
// a diagnostic mode of the reference and the sums are a few passes over the bodies. The host drives
// the build and the loop (the level count and the colouring rounds decide the launches).
#pragma once
#include "pdem_solve.cuh"

namespace pdem {

constexpr int kMlMaxLevels = 10;
constexpr int kMlSkip = 63;

template <class R>
__device__ __forceinline__ R mlEffMass(R im) {  // solver_multilevel.hpp:79-81
  return R(1) / fmax(im, R(1e-30));
}
// coarse eligibility with the reference's default gate (slip): active, coloured, quasi-static
// approach and slip (solver_multilevel.hpp:97-128)
template <class R>
__device__ __forceinline__ bool mlEligible(const Dev<R>& d, int idx, R qsThr) {
  if (d.mnp[idx] <= 0 || d.mColor[idx] < 0)
    return false;
  if (fabs(d.vn0[idx]) > qsThr)
    return false;
  const V3<R> vt = v3(d.vt0[idx]);
  return !(dot(vt, vt) > qsThr * qsThr);
}
template <class R>
__device__ __forceinline__ void mlEnds(const Dev<R>& d, const int* grp, int idx, int& gA, int& gB) {
  const int2 ab = d.mab[idx];
  gA = grp[d.realIdx[ab.x]];
  gB = ab.y >= 0 ? grp[d.realIdx[ab.y]] : -1;
}

__global__ void kMlIota(int* p, int n) {
  GRID_STRIDE(i, n) { p[i] = (int)i; }
}
// matching: every eligible body-body manifold between two groups bids its colour key at both ends;
// a manifold that wins both ends pairs them (solver_multilevel.hpp:157-193)
template <class R>
__global__ void kMlMatchContend(Dev<R> d, int nm, R qsThr, const int* grp, long long* winner) {
  GRID_STRIDE(idx, nm) {
    if (d.mab[idx].y < 0 || !mlEligible(d, (int)idx, qsThr))
      continue;
    int gA, gB;
    mlEnds(d, grp, (int)idx, gA, gB);
    if (gA == gB)
      continue;
    const long long key = colorKey((int)idx);
    atomicMax(&winner[gA], key);
    atomicMax(&winner[gB], key);
  }
}
template <class R>
__global__ void kMlMatchCommit(Dev<R> d, int nm, R qsThr, const int* grp, const long long* winner, int* mate) {
  GRID_STRIDE(idx, nm) {
    if (d.mab[idx].y < 0 || !mlEligible(d, (int)idx, qsThr))
      continue;
    int gA, gB;
    mlEnds(d, grp, (int)idx, gA, gB);
    if (gA == gB)
      continue;
    const long long key = colorKey((int)idx);
    if (winner[gA] == key && winner[gB] == key) {
      mate[gA] = gB;
      mate[gB] = gA;
    }
  }
}
// compaction: a matched pair becomes one group whose id is its smaller member's rank among the
// leaders (solver_multilevel.hpp:195-215): flags, an exclusive scan, then the parent map
__global__ void kMlLeader(const int* mate, int n, int* flag) {
  GRID_STRIDE(g, n) { flag[g] = mate[g] >= g ? 1 : 0; }
}
__global__ void kMlParent(const int* mate, const int* flag, const int* pos, int n, int* parent) {
  GRID_STRIDE(g, n) { parent[g] = pos[flag[g] ? (int)g : mate[g]]; }
}
__global__ void kMlCompose(int* grp, int n, const int* parent) {
  GRID_STRIDE(i, n) { grp[i] = parent[grp[i]]; }
}
// group masses and inverse masses, summed in ascending body order (solver_multilevel.hpp:226-243)
template <class R>
__global__ void kMlGroupMass(Dev<R> d, int n, const int* grp, R* massG, R* invMassG, int ng) {
  if (blockIdx.x | threadIdx.x)
    return;
  for (int g = 0; g < ng; ++g)
    massG[g] = R(0);
  for (int i = 0; i < n; ++i)
    massG[grp[i]] += mlEffMass(d.invMass[i]);
  for (int g = 0; g < ng; ++g)
    invMassG[g] = R(1) / massG[g];
}
// colouring of the crossing manifolds on the group graph, one round (solver_multilevel.hpp:244-306):
// pending = eligible, this level's slot still 63 and ends in different groups; winners (the largest
// key at both ends: a group has at most one) take the lowest colour free at both ends
template <class R>
__device__ __forceinline__ bool mlPending(const Dev<R>& d, const int* grp, const long long* packed, int shift,
                                          R qsThr, int idx, int& gA, int& gB) {
  if (!mlEligible(d, idx, qsThr) || ((packed[idx] >> shift) & 63) != kMlSkip)
    return false;
  mlEnds(d, grp, idx, gA, gB);
  return gB != gA;
}
template <class R>
__global__ void kMlColorContend(Dev<R> d, int nm, R qsThr, const int* grp, const long long* packed, int shift,
                                long long* winner) {
  GRID_STRIDE(idx, nm) {
    int gA, gB;
    if (!mlPending(d, grp, packed, shift, qsThr, (int)idx, gA, gB))
      continue;
    const long long key = colorKey((int)idx);
    atomicMax(&winner[gA], key);
    if (gB >= 0)
      atomicMax(&winner[gB], key);
  }
}
template <class R>
__global__ void kMlColorCommit(Dev<R> d, int nm, R qsThr, const int* grp, long long* packed, int shift,
                               const long long* winner, u64* mask, int* rem) {
  GRID_STRIDE(idx, nm) {
    int gA, gB;
    if (!mlPending(d, grp, packed, shift, qsThr, (int)idx, gA, gB))
      continue;
    const long long key = colorKey((int)idx);
    if (winner[gA] != key || (gB >= 0 && winner[gB] != key)) {
      atomicAdd(rem, 1);
      continue;
    }
    const u64 forb = mask[gA] | (gB >= 0 ? mask[gB] : 0ull);
    int c = 0;
    while (c < kMlSkip - 1 && (forb & (1ull << c)))
      ++c;
    packed[idx] = (packed[idx] & ~(63ll << shift)) | ((long long)c << shift);
    mask[gA] |= 1ull << c;
    if (gB >= 0)
      mask[gB] |= 1ull << c;
  }
}
__global__ void kMlMaxColor(const long long* packed, int nm, int shift, int* mx) {
  GRID_STRIDE(idx, nm) {
    const int c = (int)((packed[idx] >> shift) & 63);
    if (c != kMlSkip)
      atomicMax(mx, c);
  }
}
// restriction: V_g = sum(m v) / sum(m), in ascending body order, and its snapshot
// (solver_multilevel.hpp:354-380)
template <class R>
__global__ void kMlRestrict(Dev<R> d, int n, const int* grp, Q4<R>* velG, Q4<R>* velG0, const R* massG, int ng) {
  if (blockIdx.x | threadIdx.x)
    return;
  for (int g = 0; g < ng; ++g)
    velG[g] = Q4<R>{0, 0, 0, 0};
  for (int i = 0; i < n; ++i) {
    const R m = mlEffMass(d.invMass[i]);
    const Q4<R> v = d.velPred[i];
    Q4<R>& G = velG[grp[i]];
    G.x += m * v.x;
    G.y += m * v.y;
    G.z += m * v.z;
  }
  for (int g = 0; g < ng; ++g) {
    const R invM = R(1) / massG[g];
    velG[g].x *= invM;
    velG[g].y *= invM;
    velG[g].z *= invM;
    velG0[g] = velG[g];
  }
}
// one colour of a coarse sweep: translation-only inelastic PGS at the aggregate masses on the fine
// normal accumulator (solver_multilevel.hpp:382-454); the colour's manifolds share no group
template <class R>
__global__ void kMlCoarsePGS(Dev<R> d, int nm, const int* grp, const long long* packed, int shift, int color,
                             Q4<R>* velG, const R* invMassG, R* qs) {
  R mx = R(0);
  GRID_STRIDE(idx, nm) {
    if ((int)((packed[idx] >> shift) & 63) != color)
      continue;
    int gA, gB;
    mlEnds(d, grp, (int)idx, gA, gB);
    const R invN = R(1) / static_cast<R>(d.mnp[idx]);
    const V3<R> N = v3(d.mN[idx]);
    const R lenN = sqrt(dot(N, N));
    if (lenN < R(1e-9))
      continue;
    const V3<R> rAa = mul(v3(d.mrA[idx]), invN), rBa = mul(v3(d.mrB[idx]), invN);
    const V3<R> dc = gB < 0 ? rAa : sub(rAa, rBa);
    const V3<R> vA = v3(velG[gA]);
    const V3<R> vB = gB >= 0 ? v3(velG[gB]) : mul(v3(d.mwv[idx]), invN);
    const R vn = dot(sub(vA, vB), N);
    const R al = dot(N, dc);
    const R sgn = al > R(0) ? R(1) : R(-1);
    const R iA = invMassG[gA];
    const R iB = gB >= 0 ? invMassG[gB] : R(0);
    const R w = dot(N, N) * (iA + iB);
    if (w <= R(0))
      continue;
    const R dp = (sgn * vn) / w;
    const R pOld = d.lambda[idx];
    R pNew = pOld + dp;
    if (pNew < R(0))
      pNew = R(0);
    const R dd = pNew - pOld;
    if (dd == R(0))
      continue;
    d.lambda[idx] = pNew;
    runMax(mx, fabs(dd) * w / lenN);
    const V3<R> J = mul(N, -sgn * dd);
    Q4<R>& a = velG[gA];
    a.x += J.x * iA;
    a.y += J.y * iA;
    a.z += J.z * iA;
    if (gB >= 0) {
      Q4<R>& b = velG[gB];
      b.x -= J.x * iB;
      b.y -= J.y * iB;
      b.z -= J.z * iB;
    }
  }
  warpMaxAtomic(qs, mx);
}
// prolongation: every member takes its group's velocity change (solver_multilevel.hpp:456-467)
template <class R>
__global__ void kMlProlong(Dev<R> d, int n, const int* grp, const Q4<R>* velG, const Q4<R>* velG0) {
  GRID_STRIDE(i, n) {
    const Q4<R> g = velG[grp[i]], g0 = velG0[grp[i]];
    Q4<R>& v = d.velPred[i];
    v.x += g.x - g0.x;
    v.y += g.y - g0.y;
    v.z += g.z - g0.z;
  }
}
// one colour of the fine sweep of the multilevel loop: the PGS update of the main loop, which also
// raises the quasi-static residual qs on contacts with |vn0| <= 4 vRest |N|
template <class R>
__global__ void kPGSColorQS(Dev<R> d, const int* order, const int* coff, int color, SolveP<R> P, R* qs) {
  const int b = coff[color], n = coff[color + 1] - b;
  const bool serial = color >= kSaturatedColor;  // the saturated colour runs in manifold order
  if (serial && (blockIdx.x | threadIdx.x))
    return;
  R mx = R(0), mq = R(0);
  for (long t = serial ? 0 : (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += serial ? 1 : (long)gridDim.x * blockDim.x) {
    const int idx = order[b + t];
    pgsCore<R, false, true>(d, idx, pgsStatic(d, idx), P.eN, P.mu, 0, P, mx, &mq);
  }
  if (serial) {
    atomicMaxNonNeg(&d.ctr->maxApproach, mx);
    atomicMaxNonNeg(qs, mq);
  } else {
    warpMaxAtomic(&d.ctr->maxApproach, mx);
    warpMaxAtomic(qs, mq);
  }
}

}  // namespace pdem
