// Velocity and position solves of the substep (src/solver_velocity.hpp, src/solver_position.hpp,
// src/solver_friction.hpp).
//
// Colour classes are body-disjoint, so each per-colour kernel updates velocities / positions in
// place with no atomics (the reference's colored Gauss-Seidel). Accumulations the reference does
// with atomics (warm-start impulses, Jacobi deltas, friction deltas) are owner-computes gathers over
// per-body incidence lists sorted by source index — the serial reference's order. Loop control
// (adaptive stops, the stabilization trigger) lives in device flags so the host never waits.
#pragma once
#include "pdem_common.cuh"

namespace pdem {

// colours are capped at 62 (src/solver_velocity.hpp:341-342): bodies of degree > 62 can leave
// several manifolds sharing a body in colour 62
constexpr int kSaturatedColor = 62;

// incidence list entry: source index << 1 | side (0 = body A, 1 = body B)
struct Incidence {
  const int* off;  // [nbodies + 1]
  const int* ent;  // entries sorted by (body, source index, side)
};

template <class R>
struct ManifoldView {
  int ra, rb;
  R imA, imB;
  V3<R> iIA, iIB;
  Q4<R> qA, qB;
  R invN;
  V3<R> N, TA, TB, rAa, rBa, dc, wv;
  R eSum, muSum;
};
template <class R>
__device__ __forceinline__ ManifoldView<R> loadManifold(const Dev<R>& d, int idx) {
  ManifoldView<R> v;
  const int2 ab = d.mab[idx];
  v.ra = d.realIdx[ab.x];
  v.rb = ab.y >= 0 ? d.realIdx[ab.y] : ab.y;
  v.imA = d.invMass[v.ra];
  v.imB = ab.y >= 0 ? d.invMass[v.rb] : R(0);
  v.iIA = v3(d.invI[v.ra]);
  v.iIB = ab.y >= 0 ? v3(d.invI[v.rb]) : V3<R>{0, 0, 0};
  v.qA = d.quat[v.ra];
  v.qB = ab.y >= 0 ? d.quat[v.rb] : Q4<R>{0, 0, 0, 1};
  v.invN = R(1) / static_cast<R>(d.mnp[idx]);
  const Q4<R> N = d.mN[idx], TA = d.mTA[idx];
  v.N = v3(N);
  v.eSum = N.w;
  v.TA = v3(TA);
  v.muSum = TA.w;
  v.TB = v3(d.mTB[idx]);
  v.rAa = mul(v3(d.mrA[idx]), v.invN);
  v.rBa = mul(v3(d.mrB[idx]), v.invN);
  v.dc = (ab.y < 0) ? v.rAa : sub(v.rAa, v.rBa);
  v.wv = v3(d.mwv[idx]);
  return v;
}

template <class R>
struct SolveP {
  R growthRate, eN, eT, mu, vRest, dt;
  int ncol;
};

// ---------------------------------------------------------------------------------------------
// loop control
enum CtlOp : int {
  CTL_VEL_BEGIN = 0,   // main velocity sweep start: maxApproach = 0 unless done
  CTL_VEL_END = 1,     // main velocity sweep end: done if maxApproach <= thr
  CTL_STAB_DECIDE = 2, // stabilization runs iff mode != 0 && maxApproach > thr
  CTL_STAB_BEGIN = 3,
  CTL_STAB_END = 4,
  CTL_POS_BEGIN = 5,   // position sweep start: maxOverlap = 0 unless done
  CTL_POS_END = 6,     // position sweep end: done if maxOverlap < thr
};
template <class R>
__global__ void kCtl(Counters<R>* c, int op, R thr, int mode) {
  if (threadIdx.x | blockIdx.x)
    return;
  switch (op) {
    case CTL_VEL_BEGIN:
      if (!c->velDone) {
        c->maxApproach = R(0);
        c->velSweeps += 1;
      }
      break;
    case CTL_VEL_END:
      if (!c->velDone && c->maxApproach <= thr)
        c->velDone = 1;
      break;
    case CTL_STAB_DECIDE:
      c->stabRun = (mode != 0 && c->maxApproach > thr) ? 1 : 0;
      c->stabDone = c->stabRun ? 0 : 1;
      break;
    case CTL_STAB_BEGIN:
      if (!c->stabDone) {
        c->maxApproach = R(0);
        c->stabSweeps += 1;
      }
      break;
    case CTL_STAB_END:
      if (!c->stabDone && c->maxApproach <= thr)
        c->stabDone = 1;
      break;
    case CTL_POS_BEGIN:
      if (!c->posDone) {
        c->maxOverlap = R(0);
        c->posSweeps += 1;
      }
      break;
    case CTL_POS_END:
      if (!c->posDone && c->maxOverlap < thr)
        c->posDone = 1;
      break;
  }
}
// batched form: the same control for every scene (one block); the global flags become "every
// scene done" and "some scene runs the stabilization pass", so whole launches still skip
template <class R>
__global__ void kCtlScenes(Counters<R>* c, SceneCtl<R>* scn, int S, int op, R thr, int mode) {
  int notDone = 0, anyStab = 0;
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    SceneCtl<R>& q = scn[s];
    switch (op) {
      case CTL_VEL_BEGIN:
        if (!q.velDone) {
          q.maxApproach = R(0);
          q.velSweeps += 1;
        }
        break;
      case CTL_VEL_END:
        if (!q.velDone && q.maxApproach <= thr)
          q.velDone = 1;
        break;
      case CTL_STAB_DECIDE:
        q.stabRun = (mode != 0 && q.maxApproach > thr) ? 1 : 0;
        q.stabDone = q.stabRun ? 0 : 1;
        break;
      case CTL_STAB_BEGIN:
        if (!q.stabDone) {
          q.maxApproach = R(0);
          q.stabSweeps += 1;
        }
        break;
      case CTL_STAB_END:
        if (!q.stabDone && q.maxApproach <= thr)
          q.stabDone = 1;
        break;
      case CTL_POS_BEGIN:
        if (!q.posDone) {
          q.maxOverlap = R(0);
          q.posSweeps += 1;
        }
        break;
      case CTL_POS_END:
        if (!q.posDone && q.maxOverlap < thr)
          q.posDone = 1;
        break;
    }
    notDone |= (op <= CTL_VEL_END) ? !q.velDone : (op <= CTL_STAB_END) ? !q.stabDone : !q.posDone;
    anyStab |= q.stabRun;
  }
  notDone = __syncthreads_or(notDone);
  anyStab = __syncthreads_or(anyStab);
  if (threadIdx.x == 0) {
    if (op <= CTL_VEL_END) {
      c->velDone = !notDone;
    } else if (op == CTL_STAB_DECIDE) {
      c->stabRun = anyStab;
      c->stabDone = !anyStab;
    } else if (op <= CTL_STAB_END) {
      c->stabDone = !notDone;
    } else {
      c->posDone = !notDone;
    }
  }
}
template <class R>
__device__ __forceinline__ bool gateOpen(const Counters<R>* c, int gate) {
  // gate: 0 always, 1 main velocity loop, 2 stabilization loop, 3 position loop
  if (gate == 1)
    return !c->velDone;
  if (gate == 2)
    return !c->stabDone;
  if (gate == 3)
    return !c->posDone;
  return true;
}

// ---------------------------------------------------------------------------------------------
// pre-solve approach velocity (src/solver_velocity.hpp:390-447)
template <class R>
__global__ void kVn0(Dev<R> d, int nm, R growthRate) {
  GRID_STRIDE(idx, nm) {
    if (d.mnp[idx] <= 0)
      continue;
    const int2 ab = d.mab[idx];
    const int ra = d.realIdx[ab.x];
    if (ab.y >= 0 && ra > d.realIdx[ab.y])
      continue;
    const ManifoldView<R> v = loadManifold(d, (int)idx);
    const V3<R> vA = v3(d.velPred[ra]), wA = v3(d.angVelPred[ra]);
    V3<R> vB{0, 0, 0}, wB{0, 0, 0};
    if (ab.y >= 0) {
      vB = v3(d.velPred[v.rb]);
      wB = v3(d.angVelPred[v.rb]);
    } else {
      vB = mul(v.wv, v.invN);
    }
    const V3<R> vG = mul(v.dc, growthRate);
    R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
    vn += dot(vG, v.N);
    d.vn0[idx] = vn;
    const R lenN = sqrt(dot(v.N, v.N));
    V3<R> vt{0, 0, 0};
    if (lenN > R(1e-9)) {
      const V3<R> nh = mul(v.N, R(1) / lenN);
      const V3<R> wBv = ab.y >= 0 ? v3(d.angVelPred[v.rb]) : V3<R>{0, 0, 0};
      const V3<R> vr = sub(add(vA, cross(wA, v.rAa)), add(vB, cross(wBv, v.rBa)));
      vt = sub(vr, mul(nh, dot(vr, nh)));
    }
    d.vt0[idx] = q4(vt);
  }
}

// one-sided stabilization flags (src/solver_velocity.hpp:456-495)
template <class R>
__global__ void kSideFlags(Dev<R> d, int nm, V3<R> gHat, R riseThr, R approachThr) {
  if (!d.ctr->stabRun)
    return;
  GRID_STRIDE(idx, nm) {
    const uint8_t was = d.persistent[idx];
    d.sideFlags[idx] = 0;
    const int2 ab = d.mab[idx];
    if (d.mnp[idx] <= 0 || ab.y < 0 || was == 0)
      continue;
    if (fabs(d.vn0[idx]) > approachThr)
      continue;
    const int ra = d.realIdx[ab.x], rb = d.realIdx[ab.y];
    if (ra > rb)
      continue;
    const V3<R> dx = sub(v3(d.posPred[ab.x]), v3(d.posPred[ab.y]));
    const R up = -(dx.x * gHat.x + dx.y * gHat.y + dx.z * gHat.z);
    const R thr = R(0.3) * sqrt(dot(dx, dx));
    if (up > thr && -dot(v3(d.velPred[rb]), gHat) <= riseThr && d.grounded[rb] > 0)
      d.sideFlags[idx] = 1;
    else if (up < -thr && -dot(v3(d.velPred[ra]), gHat) <= riseThr && d.grounded[ra] > 0)
      d.sideFlags[idx] = 2;
  }
}

// warm-start impulses (src/solver_velocity.hpp:498-605), gathered per real body in manifold order.
// Per manifold the reference applies: normal on A, normal on B, tangential on A, tangential on B.
template <class R>
__device__ __forceinline__ bool warmParts(const Dev<R>& d, int idx, R& lam, V3<R>& lt, bool& hasT) {
  const R p = d.lambda[idx];
  lt = v3(d.lambdaT[idx]);
  hasT = nonzero(lt);
  if (p == R(0) && !hasT)
    return false;
  if (d.mnp[idx] <= 0)
    return false;
  const int2 ab = d.mab[idx];
  if (ab.y >= 0 && d.realIdx[ab.x] > d.realIdx[ab.y])
    return false;
  const R invN = R(1) / static_cast<R>(d.mnp[idx]);
  const V3<R> N = v3(d.mN[idx]);
  const V3<R> rAa = mul(v3(d.mrA[idx]), invN), rBa = mul(v3(d.mrB[idx]), invN);
  const V3<R> dc = (ab.y < 0) ? rAa : sub(rAa, rBa);
  const R al = dot(N, dc);
  const R sgn = (al > R(0)) ? R(1) : R(-1);
  lam = -sgn * p;
  if (hasT) {
    const R l2 = sqrt(dot(N, N));
    if (l2 > R(1e-9)) {
      const V3<R> nh = mul(N, R(1) / l2);
      lt = sub(lt, mul(nh, dot(lt, nh)));
    }
  }
  return true;
}
// the projected tangential accumulator is written back once per manifold
template <class R>
__global__ void kWarmProject(Dev<R> d, int nm) {
  GRID_STRIDE(idx, nm) {
    R lam;
    V3<R> lt;
    bool hasT;
    if (warmParts(d, (int)idx, lam, lt, hasT) && hasT)
      d.lambdaT[idx] = q4(lt);
  }
}
template <class R>
__global__ void kWarmApply(Dev<R> d, int numReal, Incidence inc) {
  GRID_STRIDE(b, numReal) {
    const int s = inc.off[b], e = inc.off[b + 1];
    if (s == e)
      continue;
    V3<R> v = v3(d.velPred[b]), w = v3(d.angVelPred[b]);
    const R im = d.invMass[b];
    const V3<R> iI = v3(d.invI[b]);
    const Q4<R> q = d.quat[b];
    for (int t = s; t < e; ++t) {
      const int idx = inc.ent[t] >> 1, side = inc.ent[t] & 1;
      const bool both = (side == 0 && t + 1 < e && (inc.ent[t + 1] >> 1) == idx);
      R lam;
      V3<R> lt;
      bool hasT;
      if (!warmParts(d, idx, lam, lt, hasT)) {
        if (both)
          ++t;
        continue;
      }
      const V3<R> N = v3(d.mN[idx]);
      const R invN = R(1) / static_cast<R>(d.mnp[idx]);
      const V3<R> J = mul(N, lam);
      // normal part(s)
      for (int sd = side; sd <= (both ? 1 : side); ++sd) {
        if (sd == 0) {
          v = add(v, mul(J, im));
          w = add(w, angResponse(q, mul(v3(d.mTA[idx]), lam), iI));
        } else {
          v = add(v, mul(neg(J), im));
          w = add(w, angResponse(q, mul(v3(d.mTB[idx]), lam), iI));
        }
      }
      if (hasT)
        for (int sd = side; sd <= (both ? 1 : side); ++sd) {
          if (sd == 0) {
            v = add(v, mul(lt, im));
            w = add(w, angResponse(q, cross(mul(v3(d.mrA[idx]), invN), lt), iI));
          } else {
            v = add(v, mul(neg(lt), im));
            w = add(w, angResponse(q, cross(mul(v3(d.mrB[idx]), invN), mul(lt, R(-1))), iI));
          }
        }
      if (both)
        ++t;
    }
    d.velPred[b] = q4(v);
    d.angVelPred[b] = q4(w);
  }
}

// ---------------------------------------------------------------------------------------------
// projected Gauss-Seidel sweep of one colour (src/solver_velocity.hpp:641-858)
// batched form: the scene of a solve entry, its done flag for the loop (1 main velocity,
// 2 stabilization, 3 position) and the per-scene running maximum
template <class R>
__device__ __forceinline__ bool sceneDone(const Dev<R>& d, int s, int loop) {
  const SceneCtl<R>& S = d.scn[s];
  return loop == 1 ? S.velDone != 0 : loop == 2 ? S.stabDone != 0 : S.posDone != 0;
}
// LOCAL: the caller is one block per scene (kSweepScenes) and reduces the running max itself
template <class R, bool LOCAL = false>
__device__ __forceinline__ void loopMax(const Dev<R>& d, int s, bool position, R v, R& mx) {
  if (d.scn && !LOCAL)
    atomicMaxNonNeg(position ? &d.scn[s].maxOverlap : &d.scn[s].maxApproach, v);
  else
    runMax(mx, v);
}

// The per-substep constants of one manifold in the coloured velocity sweeps: its bodies' inverse
// masses, inverse inertias and orientations (fixed while the velocity solve runs), its averaged
// normal, lever arms, wall velocity, restitution and friction, and the normal's generalized inverse
// masses. Every value is the expression the sweep evaluates, so reading them from a record packed
// once per substep gives the same bits as recomputing them every sweep.
template <class R>
struct PgsStatic {
  int ra, rb;
  bool hasB;
  R imA, imB;
  V3<R> iIA, iIB;
  Q4<R> qA, qB;
  V3<R> N, TA, TB, rAa, rBa, dc, wvN;
  R eAvg, muAvg, lenN, Nsq, wAn0, wBn0;
};
template <class R>
__device__ __forceinline__ PgsStatic<R> pgsStatic(const Dev<R>& d, int idx) {
  const ManifoldView<R> v = loadManifold(d, idx);
  PgsStatic<R> s;
  s.ra = v.ra;
  s.rb = v.rb;
  s.hasB = d.mab[idx].y >= 0;
  s.imA = v.imA;
  s.imB = v.imB;
  s.iIA = v.iIA;
  s.iIB = v.iIB;
  s.qA = v.qA;
  s.qB = v.qB;
  s.N = v.N;
  s.TA = v.TA;
  s.TB = v.TB;
  s.rAa = v.rAa;
  s.rBa = v.rBa;
  s.dc = v.dc;
  s.wvN = mul(v.wv, v.invN);
  s.eAvg = v.eSum * v.invN;
  s.muAvg = v.muSum * v.invN;
  s.Nsq = dot(v.N, v.N);
  s.lenN = sqrt(s.Nsq);
  s.wAn0 = s.Nsq * v.imA + genInvMass(v.TA, v.iIA, v.qA);
  s.wBn0 = s.Nsq * v.imB + genInvMass(v.TB, v.iIB, v.qB);
  return s;
}
// The records of a colour-ordered manifold list (PgsRecs), slot-major (slot k of entry t at
// q[k * cap + t]): 0 (N, lenN), 1 (TA, Nsq), 2 (TB, wAn0), 3 (dc, wBn0), 4 (rAa, imA), 5 (rBa, imB),
// 6 (wvN, eAvg), 7 (iIA, muAvg), 8 (iIB, 0), 9 qA, 10 qB; ids (manifold, ra, rb, hasB). A sweep
// reads its entry's record with coalesced loads, then only the bodies' velocities depend on it.
// Entries [0, coff[ncol]) of the colour order: the coloured manifolds.
template <class R>
__global__ void kPackPgs(Dev<R> d, const int* order, const int* coff, int ncol, PgsRecs<R> r) {
  const long n = coff[ncol];
  GRID_STRIDE(t, n) {
    const int idx = order[t];
    const PgsStatic<R> s = pgsStatic(d, idx);
    const long c = r.cap;
    r.q[t] = Q4<R>{s.N.x, s.N.y, s.N.z, s.lenN};
    r.q[c + t] = Q4<R>{s.TA.x, s.TA.y, s.TA.z, s.Nsq};
    r.q[2 * c + t] = Q4<R>{s.TB.x, s.TB.y, s.TB.z, s.wAn0};
    r.q[3 * c + t] = Q4<R>{s.dc.x, s.dc.y, s.dc.z, s.wBn0};
    r.q[4 * c + t] = Q4<R>{s.rAa.x, s.rAa.y, s.rAa.z, s.imA};
    r.q[5 * c + t] = Q4<R>{s.rBa.x, s.rBa.y, s.rBa.z, s.imB};
    r.q[6 * c + t] = Q4<R>{s.wvN.x, s.wvN.y, s.wvN.z, s.eAvg};
    r.q[7 * c + t] = Q4<R>{s.iIA.x, s.iIA.y, s.iIA.z, s.muAvg};
    r.q[8 * c + t] = Q4<R>{s.iIB.x, s.iIB.y, s.iIB.z, R(0)};
    r.q[9 * c + t] = s.qA;
    r.q[10 * c + t] = s.qB;
    r.ids[t] = make_int4(idx, s.ra, s.rb, s.hasB ? 1 : 0);
  }
}
template <class R>
__device__ __forceinline__ PgsStatic<R> pgsRecord(const PgsRecs<R>& r, long t, int& idx) {
  const long c = r.cap;
  const int4 id = r.ids[t];
  const Q4<R> a = r.q[t], b = r.q[c + t], e = r.q[2 * c + t], f = r.q[3 * c + t], g = r.q[4 * c + t],
              h = r.q[5 * c + t], w = r.q[6 * c + t], ia = r.q[7 * c + t], ib = r.q[8 * c + t];
  PgsStatic<R> s;
  idx = id.x;
  s.ra = id.y;
  s.rb = id.z;
  s.hasB = id.w != 0;
  s.N = v3(a);
  s.lenN = a.w;
  s.TA = v3(b);
  s.Nsq = b.w;
  s.TB = v3(e);
  s.wAn0 = e.w;
  s.dc = v3(f);
  s.wBn0 = f.w;
  s.rAa = v3(g);
  s.imA = g.w;
  s.rBa = v3(h);
  s.imB = h.w;
  s.wvN = v3(w);
  s.eAvg = w.w;
  s.iIA = v3(ia);
  s.muAvg = ia.w;
  s.iIB = v3(ib);
  s.qA = r.q[9 * c + t];
  s.qB = r.q[10 * c + t];
  return s;
}

// one projected Gauss-Seidel update of manifold idx from its per-substep constants v; with QS it
// also raises *qs by the corrections of quasi-static contacts, |vn0| <= 4 vRest |N| (the residual
// of the multilevel pass, src/solver_velocity.hpp:722-723, 829-830)
template <class R, bool LOCAL = false, bool QS = false>
__device__ __forceinline__ void pgsCore(const Dev<R>& d, int idx, const PgsStatic<R>& v, R eG, R muG, int sc,
                                        const SolveP<R>& P, R& mx, R* qs = nullptr) {
  const int ra = v.ra, rb = v.rb;
  const bool hasB = v.hasB;
  const V3<R> vA = v3(d.velPred[ra]), wA = v3(d.angVelPred[ra]);
  V3<R> vB{0, 0, 0}, wB{0, 0, 0};
  R e = eG;
  if (hasB) {
    vB = v3(d.velPred[rb]);
    wB = v3(d.angVelPred[rb]);
  } else {
    vB = v.wvN;
  }
  if (v.eAvg >= R(0))
    e = v.eAvg;
  const R lenN = v.lenN;
  if (lenN < R(1e-9))
    return;
  const V3<R> vG = mul(v.dc, P.growthRate);
  R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
  vn += dot(vG, v.N);
  const R al = dot(v.N, v.dc);
  const R sgn = (al > R(0)) ? R(1) : R(-1);
  R wAn = v.wAn0;
  R wBn = v.wBn0;
  bool applyA = true, applyB = true;
  const uint8_t sf = d.sideFlags[idx];
  if (sf == 1) {
    wBn = R(0);
    applyB = false;
    e = R(0);
  } else if (sf == 2) {
    wAn = R(0);
    applyA = false;
    e = R(0);
  }
  const R wT = wAn + wBn;
  if (wT <= R(0))
    return;
  const R vn0 = d.vn0[idx];
  const R v0 = sgn * vn0;
  if (fabs(vn0) < P.vRest * lenN)
    e = R(0);
  const R target = (v0 > R(0)) ? -e * v0 : R(0);
  const R vt = sgn * vn;
  const R dp = (vt - target) / wT;
  const R pOld = d.lambda[idx];
  R pNew = pOld + dp;
  if (pNew < R(0))
    pNew = R(0);
  const R dA = pNew - pOld;
  V3<R> vA2 = vA, wA2 = wA, vB2 = vB, wB2 = wB;
  if (dA != R(0)) {
    d.lambda[idx] = pNew;
    loopMax<R, LOCAL>(d, sc, false, fabs(dA) * wT / lenN, mx);
    if (QS && fabs(vn0) <= R(4) * P.vRest * lenN)
      runMax(*qs, fabs(dA) * wT / lenN);
    const R lam = -sgn * dA;
    const V3<R> J = mul(v.N, lam), JA = mul(v.TA, lam), JB = mul(v.TB, lam);
    if (applyA) {
      vA2 = add(vA2, mul(J, v.imA));
      wA2 = add(wA2, angResponse(v.qA, JA, v.iIA));
    }
    if (hasB && applyB) {
      vB2 = add(vB2, mul(neg(J), v.imB));
      wB2 = add(wB2, angResponse(v.qB, JB, v.iIB));
    }
  }
  // friction cone
  R mu = muG;
  if (v.muAvg >= R(0))
    mu = v.muAvg;
  const V3<R> ltOld = v3(d.lambdaT[idx]);
  const bool haveOld = nonzero(ltOld);
  if (mu > R(0) || haveOld) {
    const V3<R> nh = mul(v.N, R(1) / lenN);
    const V3<R> vBf = hasB ? vB2 : v.wvN;
    const V3<R> wBf = hasB ? wB2 : V3<R>{0, 0, 0};
    const V3<R> vr = sub(add(vA2, cross(wA2, v.rAa)), add(vBf, cross(wBf, v.rBa)));
    const V3<R> vtv = sub(vr, mul(nh, dot(vr, nh)));
    R beta = P.eT;
    if (beta != R(0) && (sf != 0 || fabs(vn0) < P.vRest * lenN))
      beta = R(0);
    V3<R> err = vtv;
    if (beta != R(0)) {
      V3<R> w0 = v3(d.vt0[idx]);
      w0 = sub(w0, mul(nh, dot(w0, nh)));
      err = add(vtv, mul(w0, beta));
    }
    const R vl = sqrt(dot(err, err));
    V3<R> ltNew = ltOld;
    R wTt = v.imA + v.imB;
    if (vl > R(1e-9)) {
      const V3<R> th = mul(err, R(1) / vl);
      const R wAt = (sf == 2) ? R(0) : v.imA + genInvMass(cross(v.rAa, th), v.iIA, v.qA);
      const R wBt = (sf == 1 || !hasB) ? R(0) : v.imB + genInvMass(cross(v.rBa, th), v.iIB, v.qB);
      wTt = wAt + wBt;
      if (wTt > R(1e-9))
        ltNew = add(ltOld, mul(th, -vl / wTt));
    }
    ltNew = sub(ltNew, mul(nh, dot(ltNew, nh)));
    R nTot = fmax(d.lambda[idx], R(0)) * lenN;
    if (fabs(vn0) < P.vRest * lenN)
      nTot += fmax(d.posImp[idx], R(0));
    const R bound = mu * nTot;
    const R ll = sqrt(dot(ltNew, ltNew));
    if (ll > bound)
      ltNew = (bound > R(0)) ? mul(ltNew, bound / ll) : V3<R>{0, 0, 0};
    const V3<R> dd = sub(ltNew, ltOld);
    if (nonzero(dd)) {
      d.lambdaT[idx] = q4(ltNew);
      const R dl = sqrt(dot(dd, dd));
      if (wTt > R(1e-9)) {
        loopMax<R, LOCAL>(d, sc, false, dl * wTt, mx);
        if (QS && fabs(vn0) <= R(4) * P.vRest * lenN)
          runMax(*qs, dl * wTt);
      }
      if (applyA) {
        vA2 = add(vA2, mul(dd, v.imA));
        wA2 = add(wA2, angResponse(v.qA, cross(v.rAa, dd), v.iIA));
      }
      if (hasB && applyB) {
        vB2 = add(vB2, mul(neg(dd), v.imB));
        wB2 = add(wB2, angResponse(v.qB, cross(v.rBa, mul(dd, R(-1))), v.iIB));
      }
    }
  }
  d.velPred[ra] = q4(vA2);
  d.angVelPred[ra] = q4(wA2);
  if (hasB) {
    d.velPred[rb] = q4(vB2);
    d.angVelPred[rb] = q4(wB2);
  }
}

template <class R, bool LOCAL = false>
__device__ __forceinline__ void pgsOne(const Dev<R>& d, int idx, const SolveP<R>& P, R& mx, int loop) {
  int sc = 0;
  R eG = P.eN, muG = P.mu;
  if (d.scn) {
    sc = d.sceneOf[d.mab[idx].x];
    if (sceneDone(d, sc, loop))
      return;
    eG = d.scn[sc].eN;
    muG = d.scn[sc].mu;
  }
  pgsCore<R, LOCAL>(d, idx, pgsStatic(d, idx), eG, muG, sc, P, mx);
}
template <class R>
__global__ void kPGSColor(Dev<R> d, const int* order, const int* coff, int color, SolveP<R> P, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  const int b = coff[color], n = coff[color + 1] - b;
  // colour 62 is where the 62-colour mask saturates: it is not an independent set, so it
  // runs serially in manifold order, as the reference's serial sweep does
  const bool serial = color >= kSaturatedColor;
  if (serial && (blockIdx.x | threadIdx.x))
    return;
  R mx = R(0);
  for (long t = serial ? 0 : (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += serial ? 1 : (long)gridDim.x * blockDim.x) {
    pgsOne(d, order[b + t], P, mx, gate);
  }
  if (serial)
    atomicMaxNonNeg(&d.ctr->maxApproach, mx);
  else
    warpMaxAtomic(&d.ctr->maxApproach, mx);
}

// ---- "ordered" stabilization (level-ordered symmetric sweeps) ----
// height-from-floor levels (src/contact_preprocessing.hpp:263-305): 0 at a wall or plane contact,
// else 1 + min over supporting bodies; one relaxation sweep per launch, *changed counts updates.
// The relaxation's fixed point (shortest support paths) does not depend on the visit order.
constexpr int kLevelInf = 1 << 28;
static __global__ void kHeightInit(int* h, int n) {
  GRID_STRIDE(i, n) { h[i] = kLevelInf; }
}
template <class R>
__global__ void kHeightSweep(Dev<R> d, int nm, V3<R> gHat, int* h, int* changed) {
  int c = 0;
  GRID_STRIDE(idx, nm) {
    if (d.mnp[idx] <= 0)
      continue;
    const int2 ab = d.mab[idx];
    const int ra = d.realIdx[ab.x];
    if (ab.y < 0) {
      if (atomicMin(&h[ra], 0) > 0)
        ++c;
      continue;
    }
    const int rb = d.realIdx[ab.y];
    const V3<R> dx = sub(v3(d.posPred[ab.x]), v3(d.posPred[ab.y]));
    const R up = -(dx.x * gHat.x + dx.y * gHat.y + dx.z * gHat.z);
    const R thr = R(0.3) * sqrt(dot(dx, dx));
    if (up > thr) {
      const int cand = atomicAdd(&h[rb], 0);
      if (cand < kLevelInf && atomicMin(&h[ra], cand + 1) > cand + 1)
        ++c;
    } else if (up < -thr) {
      const int cand = atomicAdd(&h[ra], 0);
      if (cand < kLevelInf && atomicMin(&h[rb], cand + 1) > cand + 1)
        ++c;
    }
  }
  if (c)
    atomicAdd(changed, c);
}
// bucket keys (src/solver_velocity.hpp:914-965): level * 64 + colour of every active coloured
// manifold (its level is the lower of its bodies', clamped to 1023); the rest keyed out
template <class R>
__global__ void kLevelKeys(Dev<R> d, int nm, const int* h, int* keys, int* perm) {
  GRID_STRIDE(idx, nm) {
    perm[idx] = (int)idx;
    const int c = d.mColor[idx];
    if (d.mnp[idx] <= 0 || c < 0) {
      keys[idx] = INT_MAX;
      continue;
    }
    const int2 ab = d.mab[idx];
    int lv = h[d.realIdx[ab.x]];
    if (ab.y >= 0)
      lv = min(lv, h[d.realIdx[ab.y]]);
    keys[idx] = min(lv, 1023) * 64 + c;
  }
}
// one (level, colour) bucket of the sorted permutation; the saturated colour runs serially in
// permutation order, the others are independent sets
template <class R>
__global__ void kPGSBucket(Dev<R> d, const int* perm, int b, int n, int color, SolveP<R> P, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  const bool serial = color >= kSaturatedColor;
  if (serial && (blockIdx.x | threadIdx.x))
    return;
  R mx = R(0);
  for (long t = serial ? 0 : (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += serial ? 1 : (long)gridDim.x * blockDim.x)
    pgsOne(d, perm[b + t], P, mx, gate);
  if (serial)
    atomicMaxNonNeg(&d.ctr->maxApproach, mx);
  else
    warpMaxAtomic(&d.ctr->maxApproach, mx);
}

// one-shot coloured GS of one colour, g = 0 path (src/solver_velocity.hpp:989-1137)
template <class R, bool LOCAL = false>
__device__ __forceinline__ void gsOne(const Dev<R>& d, int idx, const SolveP<R>& P, R& mx) {
  int sc = 0;
  R eG = P.eN;
  if (d.scn) {
    sc = d.sceneOf[d.mab[idx].x];
    if (sceneDone(d, sc, 1))
      return;
    eG = d.scn[sc].eN;
  }
  const ManifoldView<R> v = loadManifold(d, idx);
  const bool hasB = d.mab[idx].y >= 0;
  const V3<R> vA = v3(d.velPred[v.ra]), wA = v3(d.angVelPred[v.ra]);
  V3<R> vB{0, 0, 0}, wB{0, 0, 0};
  if (hasB) {
    vB = v3(d.velPred[v.rb]);
    wB = v3(d.angVelPred[v.rb]);
  }
  R e = eG;
  if (!hasB)
    vB = mul(v.wv, v.invN);
  {
    const R ra2 = v.eSum * v.invN;
    if (ra2 >= R(0))
      e = ra2;
  }
  const R lenN = sqrt(dot(v.N, v.N));
  if (lenN < R(1e-9))
    return;
  const V3<R> vG = mul(v.dc, P.growthRate);
  R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
  vn += dot(vG, v.N);
  const R al = dot(v.N, v.dc);
  if (al > R(0)) {
    if (vn < R(0))
      return;
  } else {
    if (vn > R(0))
      return;
  }
  const R Nsq = dot(v.N, v.N);
  const R wAn = Nsq * v.imA + genInvMass(v.TA, v.iIA, v.qA);
  const R wBn = Nsq * v.imB + genInvMass(v.TB, v.iIB, v.qB);
  const R wT = wAn + wBn;
  if (wT <= R(0))
    return;
  loopMax<R, LOCAL>(d, sc, false, fabs(vn) / lenN, mx);
  if (fabs(vn) < P.vRest * lenN)
    e = R(0);
  const R lam = (-e * vn - vn) / wT;
  const V3<R> J = mul(v.N, lam), JA = mul(v.TA, lam), JB = mul(v.TB, lam);
  d.velPred[v.ra] = q4(add(vA, mul(J, v.imA)));
  d.angVelPred[v.ra] = q4(add(wA, angResponse(v.qA, JA, v.iIA)));
  if (hasB) {
    d.velPred[v.rb] = q4(add(vB, mul(neg(J), v.imB)));
    d.angVelPred[v.rb] = q4(add(wB, angResponse(v.qB, JB, v.iIB)));
  }
}
template <class R>
__global__ void kGSColor(Dev<R> d, const int* order, const int* coff, int color, SolveP<R> P, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  const int b = coff[color], n = coff[color + 1] - b;
  // colour 62 is where the 62-colour mask saturates: it is not an independent set, so it
  // runs serially in manifold order, as the reference's serial sweep does
  const bool serial = color >= kSaturatedColor;
  if (serial && (blockIdx.x | threadIdx.x))
    return;
  R mx = R(0);
  for (long t = serial ? 0 : (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += serial ? 1 : (long)gridDim.x * blockDim.x) {
    gsOne(d, order[b + t], P, mx);
  }
  if (serial)
    atomicMaxNonNeg(&d.ctr->maxApproach, mx);
  else
    warpMaxAtomic(&d.ctr->maxApproach, mx);
}

// Jacobi velocity solve (src/solver_velocity.hpp:38-226), gathered per real body; filt selects the
// manifolds left uncoloured (-1) for the colouring-saturation fallback
template <class R>
__device__ __forceinline__ bool jacobiImpulse(const Dev<R>& d, int idx, const SolveP<R>& P, bool filt, R& lam) {
  if (filt && d.mColor[idx] != -1)
    return false;
  if (d.mnp[idx] <= 0)
    return false;
  const int2 ab = d.mab[idx];
  const int ra = d.realIdx[ab.x];
  int rb = ab.y;
  if (ab.y >= 0) {
    rb = d.realIdx[ab.y];
    if (ra > rb)
      return false;
  }
  const ManifoldView<R> v = loadManifold(d, idx);
  const V3<R> vA = v3(d.velPred[ra]), wA = v3(d.angVelPred[ra]);
  V3<R> vB{0, 0, 0}, wB{0, 0, 0};
  if (ab.y >= 0) {
    vB = v3(d.velPred[rb]);
    wB = v3(d.angVelPred[rb]);
  }
  R e = P.eN;
  if (ab.y < 0)
    vB = mul(v.wv, v.invN);
  {
    const R ra2 = v.eSum * v.invN;
    if (ra2 >= R(0))
      e = ra2;
  }
  const R lenN = sqrt(dot(v.N, v.N));
  if (lenN < R(1e-9))
    return false;
  const V3<R> vG = mul(v.dc, P.growthRate);
  R vn = dot(vA, v.N) + dot(wA, v.TA) + dot(vB, neg(v.N)) + dot(wB, v.TB);
  vn += dot(vG, v.N);
  const R al = dot(v.N, v.dc);
  if (al > R(0)) {
    if (vn < R(0))
      return false;
  } else {
    if (vn > R(0))
      return false;
  }
  const R Nsq = dot(v.N, v.N);
  const R wT = (Nsq * v.imA + genInvMass(v.TA, v.iIA, v.qA)) + (Nsq * v.imB + genInvMass(v.TB, v.iIB, v.qB));
  if (wT <= R(0))
    return false;
  if (fabs(vn) < P.vRest * lenN)
    e = R(0);
  lam = (-e * vn - vn) / wT;
  return true;
}
// each manifold's impulse is computed once (pre-pass, reads the velocities before any delta)
template <class R>
__global__ void kJacobiImpulses(Dev<R> d, int nm, SolveP<R> P, int filt, R* lamOut, int* okOut, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(idx, nm) {
    R lam = R(0);
    okOut[idx] = jacobiImpulse(d, (int)idx, P, filt != 0, lam) ? 1 : 0;
    lamOut[idx] = lam;
  }
}
template <class R>
__global__ void kJacobiGather(Dev<R> d, int numReal, Incidence inc, const R* lam, const int* ok, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(b, numReal) {
    const int s = inc.off[b], e = inc.off[b + 1];
    if (s == e)
      continue;
    V3<R> dv = v3(d.dVel[b]), dw = v3(d.dAngVel[b]);
    int cnt = d.counts[b];
    const R im = d.invMass[b];
    const V3<R> iI = v3(d.invI[b]);
    const Q4<R> q = d.quat[b];
    for (int t = s; t < e; ++t) {
      const int idx = inc.ent[t] >> 1, side = inc.ent[t] & 1;
      if (!ok[idx])
        continue;
      const R l = lam[idx];
      const V3<R> J = mul(v3(d.mN[idx]), l);
      if (side == 0) {
        dv = add(dv, mul(J, im));
        dw = add(dw, angResponse(q, mul(v3(d.mTA[idx]), l), iI));
      } else {
        dv = add(dv, mul(neg(J), im));
        dw = add(dw, angResponse(q, mul(v3(d.mTB[idx]), l), iI));
      }
      cnt += 1;
    }
    d.dVel[b] = q4(dv);
    d.dAngVel[b] = q4(dw);
    d.counts[b] = cnt;
  }
}
// src/solver_velocity.hpp:234-255
template <class R>
__global__ void kApplyVelAveraged(Dev<R> d, int n, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(i, n) {
    const int c = d.counts[i];
    if (c <= 0)
      continue;
    const R f = fmin(R(1), R(2) / static_cast<R>(c));
    d.velPred[i] = q4(add(v3(d.velPred[i]), mul(v3(d.dVel[i]), f)));
    d.angVelPred[i] = q4(add(v3(d.angVelPred[i]), mul(v3(d.dAngVel[i]), f)));
    d.dVel[i] = Q4<R>{0, 0, 0, 0};
    d.dAngVel[i] = Q4<R>{0, 0, 0, 0};
    d.counts[i] = 0;
  }
}

// ---------------------------------------------------------------------------------------------
// legacy friction cluster (src/solver_friction.hpp)
template <class R>
__global__ void kPlaneLoad(Dev<R> d, int nc) {
  GRID_STRIDE(idx, nc) {
    const int2 ab = d.cab[idx];
    if (ab.y >= 0)
      continue;
    const int A = ab.x;
    const R im = d.invMass[A];
    if (im <= R(0))
      continue;
    const V3<R> rA = v3(d.crA[idx]), n = v3(d.cn[idx]), bv = v3(d.cbv[idx]);
    const V3<R> vAc = add(v3(d.velPred[A]), cross(v3(d.angVelPred[A]), rA));
    const R ap = -dot(sub(vAc, bv), n);
    if (ap <= R(0))
      continue;
    const R wn = computeW(rA, n, im, v3(d.invI[A]));
    d.crA[idx].w = (wn > R(1e-6)) ? ap / wn : R(0);
    atomicMaxNonNeg(&d.planeFric[2 * A], ap / im);
  }
}
template <class R>
__global__ void kAccumNormal(Dev<R> d, int nc, R growthRate, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(idx, nc) {
    const int2 ab = d.cab[idx];
    const V3<R> rA = v3(d.crA[idx]), rB = v3(d.crB[idx]), n = v3(d.cn[idx]);
    if (ab.y < 0) {
      const int A = ab.x;
      const R im = d.invMass[A];
      if (im <= R(0))
        continue;
      const V3<R> vAc = add(v3(d.velPred[A]), cross(v3(d.angVelPred[A]), rA));
      const R ap = -dot(sub(vAc, v3(d.cbv[idx])), n);
      if (ap <= R(0))
        continue;
      const R wn = computeW(rA, n, im, v3(d.invI[A]));
      if (wn > R(1e-6))
        d.crA[idx].w += ap / wn;
      continue;
    }
    const int ra = d.realIdx[ab.x], rb = d.realIdx[ab.y];
    if (ra > rb)
      continue;
    const R imA = d.invMass[ra], imB = d.invMass[rb];
    const V3<R> vAc = add(v3(d.velPred[ra]), cross(v3(d.angVelPred[ra]), rA));
    const V3<R> vBc = add(v3(d.velPred[rb]), cross(v3(d.angVelPred[rb]), rB));
    const V3<R> vr = add(sub(vAc, vBc), mul(sub(rA, rB), growthRate));
    const R ap = -dot(vr, n);
    if (ap <= R(0))
      continue;
    const R wn = computeW(rA, n, imA, v3(d.invI[ra])) + computeW(rB, n, imB, v3(d.invI[rb]));
    if (wn > R(1e-6))
      d.crA[idx].w += ap / wn;
  }
}
template <class R>
__global__ void kCountFriction(Dev<R> d, int nc) {
  GRID_STRIDE(idx, nc) {
    if (d.crA[idx].w <= R(0))
      continue;
    const int2 ab = d.cab[idx];
    atomicAdd(&d.planeFric[2 * d.realIdx[ab.x] + 1], R(1));
    if (ab.y >= 0)
      atomicAdd(&d.planeFric[2 * d.realIdx[ab.y] + 1], R(1));
  }
}
// per contact tangential impulse (src/solver_friction.hpp:152-217), reading pre-sweep velocities
template <class R>
__device__ __forceinline__ bool frictionImpulse(const Dev<R>& d, int idx, R muG, V3<R>& t, R& lt, V3<R>& rnA,
                                                V3<R>& rnB) {
  const R ln = d.crA[idx].w;
  if (ln <= R(0))
    return false;
  const int2 ab = d.cab[idx];
  const int ra = d.realIdx[ab.x];
  const int rb = ab.y >= 0 ? d.realIdx[ab.y] : -1;
  const R imA = d.invMass[ra], imB = ab.y >= 0 ? d.invMass[rb] : R(0);
  const V3<R> iA = v3(d.invI[ra]), iB = ab.y >= 0 ? v3(d.invI[rb]) : V3<R>{0, 0, 0};
  const V3<R> rA = v3(d.crA[idx]), rB = v3(d.crB[idx]), n = v3(d.cn[idx]);
  const V3<R> vAc = add(v3(d.velPred[ra]), cross(v3(d.angVelPred[ra]), rA));
  V3<R> vBc{0, 0, 0};
  if (ab.y >= 0)
    vBc = add(v3(d.velPred[rb]), cross(v3(d.angVelPred[rb]), rB));
  else
    vBc = v3(d.cbv[idx]);
  const V3<R> vr = sub(vAc, vBc);
  const R vn = dot(vr, n);
  const V3<R> vt = sub(vr, mul(n, vn));
  const R vl = sqrt(dot(vt, vt));
  if (vl < R(1e-7))
    return false;
  t = mul(vt, R(1) / vl);
  rnA = cross(rA, t);
  rnB = cross(rB, t);
  const R wt = imA + imB + rnA.x * rnA.x * iA.x + rnA.y * rnA.y * iA.y + rnA.z * rnA.z * iA.z +
               rnB.x * rnB.x * iB.x + rnB.y * rnB.y * iB.y + rnB.z * rnB.z * iB.z;
  if (wt < R(1e-6))
    return false;
  const R bound = ln;
  const R nA = d.planeFric[2 * ra + 1];
  const R nB = ab.y >= 0 ? d.planeFric[2 * rb + 1] : R(0);
  const R invn = R(1) / fmax(fmax(nA, nB), R(1));
  lt = -vl / wt;
  const R mu = (d.cbv[idx].w >= R(0)) ? d.cbv[idx].w : muG;
  const R maxf = mu * bound;
  if (lt < -maxf)
    lt = -maxf;
  lt *= invn;
  return true;
}
template <class R>
__global__ void kFrictionImpulses(Dev<R> d, int nc, R muG, Q4<R>* tl, Q4<R>* rnAo, Q4<R>* rnBo, int* ok) {
  GRID_STRIDE(idx, nc) {
    V3<R> t, rnA, rnB;
    R lt = R(0);
    ok[idx] = frictionImpulse(d, (int)idx, muG, t, lt, rnA, rnB) ? 1 : 0;
    tl[idx] = q4(t, lt);
    rnAo[idx] = q4(rnA);
    rnBo[idx] = q4(rnB);
  }
}
// deltas zeroed then gathered per real body in contact order (src/solver_friction.hpp:149-217)
template <class R>
__global__ void kFrictionGather(Dev<R> d, int n, Incidence inc, const Q4<R>* tl, const Q4<R>* rnA,
                                const Q4<R>* rnB, const int* ok) {
  GRID_STRIDE(b, n) {
    V3<R> dv{0, 0, 0}, dw{0, 0, 0};
    const int s = inc.off[b], e = inc.off[b + 1];
    const R im = d.invMass[b];
    const V3<R> iI = v3(d.invI[b]);
    for (int q = s; q < e; ++q) {
      const int idx = inc.ent[q] >> 1, side = inc.ent[q] & 1;
      if (!ok[idx])
        continue;
      const Q4<R> T = tl[idx];
      const R lt = T.w;
      if (side == 0) {
        const V3<R> r = v3(rnA[idx]);
        dv = add(dv, V3<R>{T.x * lt * im, T.y * lt * im, T.z * lt * im});
        dw = add(dw, V3<R>{r.x * iI.x * lt, r.y * iI.y * lt, r.z * iI.z * lt});
      } else {
        const V3<R> r = v3(rnB[idx]);
        dv = add(dv, V3<R>{-T.x * lt * im, -T.y * lt * im, -T.z * lt * im});
        dw = add(dw, V3<R>{-r.x * iI.x * lt, -r.y * iI.y * lt, -r.z * iI.z * lt});
      }
    }
    d.dVel[b] = q4(dv);
    d.dAngVel[b] = q4(dw);
  }
}

// ---------------------------------------------------------------------------------------------
// position solve (src/solver_position.hpp)
template <class R>
__device__ __forceinline__ bool posConstraint(const Dev<R>& d, int idx, V3<R>& n, R& C, R& wT, int& A, int& B) {
  const int2 ab = d.cab[idx];
  A = ab.x;
  B = ab.y;
  const R imA = d.invMass[A], imB = B >= 0 ? d.invMass[B] : R(0);
  const V3<R> pA = v3(d.posPred[A]);
  const Q4<R> qA = d.quatPred[A];
  V3<R> pB{0, 0, 0};
  Q4<R> qB{0, 0, 0, 1};
  if (B >= 0) {
    pB = v3(d.posPred[B]);
    qB = d.quatPred[B];
  }
  const Q4<R> cnq = d.cn[idx];
  const V3<R> cn = v3(cnq), crA = v3(d.crA[idx]), crB = v3(d.crB[idx]);
  const Q4<R> qAd = qmul(qA, qinv(d.quat[A]));
  const V3<R> rA = rot(qAd, crA);
  V3<R> rB = crB;
  n = cn;
  if (B >= 0) {
    const Q4<R> qBd = qmul(qB, qinv(d.quat[B]));
    rB = rot(qBd, rB);
    n = rot(qBd, n);
  }
  if (B < 0) {
    n = cn;
    C = dot(sub(add(pA, rA), crB), n);
  } else {
    C = dot(sub(add(pA, rA), add(pB, rB)), n);
  }
  if (C >= R(0))
    return false;
  const V3<R> iA = v3(d.invI[A]), iB = B >= 0 ? v3(d.invI[B]) : V3<R>{0, 0, 0};
  wT = computeW(rA, n, imA, iA) + computeW(rB, n, imB, iB);
  return true;
}
template <class R, bool LOCAL = false>
__device__ __forceinline__ void posGSOne(const Dev<R>& d, int idx, R& mx) {
  int sc = 0;
  if (d.scn) {
    sc = d.sceneOf[d.cab[idx].x];
    if (sceneDone(d, sc, 3))
      return;
  }
  V3<R> nv;
  R C = R(0), wT = R(0);
  int A, B;
  if (!posConstraint(d, idx, nv, C, wT, A, B))
    return;
  if (wT < R(1e-6))
    return;
  const R dl = -C / wT;
  d.posLamC[idx] += dl;
  const R imA = d.invMass[A];
  const V3<R> pA = v3(d.posPred[A]);
  d.posPred[A] = q4(add(pA, V3<R>{nv.x * dl * imA, nv.y * dl * imA, nv.z * dl * imA}));
  if (B >= 0) {
    const R imB = d.invMass[B];
    const V3<R> pB = v3(d.posPred[B]);
    d.posPred[B] = q4(add(pB, V3<R>{-nv.x * dl * imB, -nv.y * dl * imB, -nv.z * dl * imB}));
  }
  loopMax<R, LOCAL>(d, sc, true, -C, mx);
}
template <class R>
__global__ void kPosGSColor(Dev<R> d, const int* order, const int* coff, int color, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  const int b = coff[color], n = coff[color + 1] - b;
  // colour 62 is where the 62-colour mask saturates: it is not an independent set, so it
  // runs serially in manifold order, as the reference's serial sweep does
  const bool serial = color >= kSaturatedColor;
  if (serial && (blockIdx.x | threadIdx.x))
    return;
  R mx = R(0);
  for (long t = serial ? 0 : (long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += serial ? 1 : (long)gridDim.x * blockDim.x) {
    posGSOne(d, order[b + t], mx);
  }
  if (serial)
    atomicMaxNonNeg(&d.ctr->maxOverlap, mx);
  else
    warpMaxAtomic(&d.ctr->maxOverlap, mx);
}
// Jacobi position solve (src/solver_position.hpp:34-134): per-contact correction pre-pass, then a
// gather per body slot in contact order
template <class R>
__global__ void kPosJacobiPre(Dev<R> d, int nc, int filt, Q4<R>* corr, int* ok, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(idx, nc) {
    ok[idx] = 0;
    if (filt && d.cColor[idx] != -1)
      continue;
    V3<R> nv;
    R C = R(0), wT = R(0);
    int A, B;
    if (!posConstraint(d, (int)idx, nv, C, wT, A, B))
      continue;
    if (wT < R(1e-6))
      continue;
    const R dl = -C / wT;
    corr[idx] = q4(nv, dl);
    ok[idx] = 1;
    if (C < R(0))
      atomicMaxNonNeg(&d.ctr->maxOverlap, -C);
  }
}
template <class R>
__global__ void kPosJacobiGather(Dev<R> d, int n, Incidence inc, const Q4<R>* corr, const int* ok, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(b, n) {
    const int s = inc.off[b], e = inc.off[b + 1];
    if (s == e)
      continue;
    V3<R> dp = v3(d.dPos[b]);
    int cnt = d.counts[b];
    const R im = d.invMass[b];
    for (int q = s; q < e; ++q) {
      const int idx = inc.ent[q] >> 1, side = inc.ent[q] & 1;
      if (!ok[idx])
        continue;
      const Q4<R> c = corr[idx];
      const R dl = c.w;
      if (side == 0)
        dp = add(dp, V3<R>{c.x * dl * im, c.y * dl * im, c.z * dl * im});
      else
        dp = add(dp, V3<R>{-c.x * dl * im, -c.y * dl * im, -c.z * dl * im});
      cnt += 1;
    }
    d.dPos[b] = q4(dp);
    d.counts[b] = cnt;
  }
}
template <class R>
__global__ void kApplyUpdatesGated(Dev<R> d, int n, int gate) {
  if (!gateOpen(d.ctr, gate))
    return;
  GRID_STRIDE(i, n) {
    const int c = d.counts[i];
    if (c <= 0)
      continue;
    const R f = R(1) / static_cast<R>(c);
    d.posPred[i] = q4(add(v3(d.posPred[i]), mul(v3(d.dPos[i]), f)));
    d.velPred[i] = q4(add(v3(d.velPred[i]), mul(v3(d.dVel[i]), f)));
    d.dPos[i] = Q4<R>{0, 0, 0, 0};
    d.dVel[i] = Q4<R>{0, 0, 0, 0};
    d.counts[i] = 0;
  }
}

// incidence entries: entry 2i = (body of side A, i<<1), 2i+1 = (body of side B, i<<1|1) or none
template <class R, int KIND>
__global__ void kIncidenceKeys(Dev<R> d, int ne, int* keys, int* vals, int none) {
  // KIND 0: manifolds by real body; 1: contacts by real body; 2: contacts by raw slot;
  // 3: candidate pairs by raw slot
  GRID_STRIDE(i, ne) {
    int2 ab = (KIND == 0) ? d.mab[i] : (KIND == 3 ? d.pairs[i] : d.cab[i]);
    int a = ab.x, b = ab.y;
    if (KIND == 0 || KIND == 1) {
      a = d.realIdx[a];
      b = b >= 0 ? d.realIdx[b] : -1;
    }
    keys[2 * i] = a;
    vals[2 * i] = (int)(i << 1);
    keys[2 * i + 1] = b >= 0 ? b : none;
    vals[2 * i + 1] = (int)((i << 1) | 1);
  }
}
// off[c] = first sorted position whose key >= c, for c in [0, nb]
template <class K>
__global__ void kLowerBoundOffsets(int ne, const K* sortedKeys, int nb, int* off) {
  GRID_STRIDE(c, nb + 1) {
    int lo = 0, hi = ne;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (sortedKeys[mid] < (K)c)
        lo = mid + 1;
      else
        hi = mid;
    }
    off[c] = lo;
  }
}

}  // namespace pdem
