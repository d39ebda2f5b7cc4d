// Hertz-Mindlin soft-sphere engine (src/solver_hertz.hpp:41-606, src/sim.hpp:545-750).
//
// Explicit force model on a cached Verlet pair list: each pair's force / torques and Mindlin history
// update are computed by one thread, then each body gathers its pair contributions in pair order and
// its wall contributions in wall order (the reference's atomic order in the serial build), then a
// symplectic kick-drift. The pair list is rebuilt when any body moved half the skin; the shear
// history is carried across rebuilds by pair key (sorted keys + binary search).
#pragma once
#include "pdem_common.cuh"

namespace pdem {

template <class R>
__device__ __forceinline__ R hertzBetaD(R e) {
  if (e <= R(0))
    return R(-1);
  if (e >= R(1))
    return R(0);
  const R le = log(e);
  return le / sqrt(le * le + R(9.8696044));
}
template <class R>
__device__ __forceinline__ V3<R> hertzForce(R delta, V3<R> nh, V3<R> vr, R rS, R mS, R eS, R gS, R e, R mu,
                                            R dt, V3<R>& xi) {
  const R sq = sqrt(rS * delta);
  const R sn = R(2) * eS * sq;
  const R st = R(8) * gS * sq;
  const R kn = (R(4) / R(3)) * eS * sq;
  const R bd = hertzBetaD(e);
  const R etaN = R(-2) * R(0.9128709) * bd * sqrt(sn * mS);
  const R etaT = R(-2) * R(0.9128709) * bd * sqrt(st * mS);
  const R vn = dot(vr, nh);
  const R fs = kn * delta;
  const R fn = fs - etaN * vn;
  const V3<R> vt = sub(vr, mul(nh, vn));
  xi = add(xi, mul(vt, dt));
  xi = sub(xi, mul(nh, dot(xi, nh)));
  V3<R> ft = add(mul(xi, -st), mul(vt, -etaT));
  const R fl = sqrt(dot(ft, ft));
  const R fm = mu * fabs(fs);
  if (fl > fm) {
    const R s = (fl > R(1e-20)) ? fm / fl : R(0);
    ft = mul(ft, s);
    if (st > R(1e-20))
      xi = mul(add(ft, mul(vt, etaT)), R(-1) / st);
  }
  return add(mul(nh, fn), ft);
}
template <class R>
__device__ __forceinline__ void hertzStars(const Dev<R>& d, int ma, int mb, R& eS, R& gS) {
  const R Ei = d.hzE[ma], Ej = d.hzE[mb], ni = d.hzNu[ma], nj = d.hzNu[mb];
  eS = R(1) / ((R(1) - ni * ni) / Ei + (R(1) - nj * nj) / Ej);
  gS = R(1) / (R(2) * (R(2) - ni) * (R(1) + ni) / Ei + R(2) * (R(2) - nj) * (R(1) + nj) / Ej);
}
template <class R>
__device__ __forceinline__ void hertzEMu(const Dev<R>& d, int ma, int mb, R eG, R muG, R& e, R& mu) {
  if (d.pairMat) {
    const int t = (ma * kMaxMaterials + mb) * 2;
    e = d.pairMat[t];
    mu = d.pairMat[t + 1];
  } else {
    e = eG;
    mu = muG;
  }
}

template <class R>
struct HertzP {
  R dt, eG, muG, globalScale, contactFrac;
  int numWalls;
};

// sphere pairs (src/solver_hertz.hpp:88-144): per-pair force F on i, torques tA on i and tB on j
template <class R>
__global__ void kHertzPairs(Dev<R> d, int np, HertzP<R> P, Q4<R>* xi, Q4<R>* F, Q4<R>* TA, Q4<R>* TB, int* on) {
  GRID_STRIDE(idx, np) {
    const int2 pr = d.pairs[idx];
    const int i = pr.x, j = pr.y;
    const V3<R> dx = sub(v3(d.pos[i]), v3(d.pos[j]));
    const R dd = sqrt(dot(dx, dx));
    const R ri = d.rad[i], rj = d.rad[j];
    const R delta = ri + rj - dd;
    if (delta <= R(0) || dd < R(1e-12)) {
      xi[idx] = Q4<R>{0, 0, 0, 0};
      on[idx] = 0;
      continue;
    }
    const V3<R> nh = mul(dx, R(1) / dd);
    const V3<R> rA = mul(nh, -(ri - R(0.5) * delta));
    const V3<R> rB = mul(nh, (rj - R(0.5) * delta));
    const V3<R> vr = sub(add(v3(d.vel[i]), cross(v3(d.angVel[i]), rA)), add(v3(d.vel[j]), cross(v3(d.angVel[j]), rB)));
    const int ma = d.matId[i], mb = d.matId[j];
    R e, mu, eS, gS;
    hertzEMu(d, ma, mb, P.eG, P.muG, e, mu);
    hertzStars(d, ma, mb, eS, gS);
    const R rS = ri * rj / (ri + rj);
    const R imS = d.invMass[i] + d.invMass[j];
    const R mS = (imS > R(0)) ? R(1) / imS : R(0);
    V3<R> x = v3(xi[idx]);
    const V3<R> f = hertzForce(delta, nh, vr, rS, mS, eS, gS, e, mu, P.dt, x);
    xi[idx] = q4(x);
    F[idx] = q4(f);
    TA[idx] = q4(cross(rA, f));
    TB[idx] = q4(cross(rB, mul(f, R(-1))));
    on[idx] = 1;
  }
}

// point-shell pairs (src/solver_hertz.hpp:454-606), one thread per pair (ordered sums over points)
template <class R>
__global__ void kHertzShapePairs(Dev<R> d, int np, HertzP<R> P, Q4<R>* xi, R* snPrev, Q4<R>* F, Q4<R>* TA, Q4<R>* TB,
                                 int* on) {
  const ShapeDesc<R> dA = d.shapes[0], dB = d.shapes[0];
  GRID_STRIDE(idx, np) {
    const int2 pr = d.pairs[idx];
    const int A = pr.x, B = pr.y;
    const V3<R> pA = v3(d.pos[A]), pB = v3(d.pos[B]);
    const Q4<R> qA = d.quat[A], qB = d.quat[B];
    const R sA = d.scale[A] * P.globalScale, sB = d.scale[B] * P.globalScale;
    const int cnt = dA.numPoints;
    const bool sphA = dA.type == SHAPE_SPHERE;
    const int iter = cnt > 0 ? cnt : 1;
    const int ma = d.matId[A], mb = d.matId[B];
    R e, mu, eS, gS;
    hertzEMu(d, ma, mb, P.eG, P.muG, e, mu);
    hertzStars(d, ma, mb, eS, gS);
    const R rcA = (sphA ? R(1) : P.contactFrac) * dA.par[0] * sA;
    const R rcB = ((dB.type == SHAPE_SPHERE) ? R(1) : P.contactFrac) * dB.par[0] * sB;
    const R rS = rcA * rcB / (rcA + rcB);
    const R imS = d.invMass[A] + d.invMass[B];
    const R mS = (imS > R(0)) ? R(1) / imS : R(0);
    const R bd = hertzBetaD(e);
    const V3<R> vA = v3(d.vel[A]), wA = v3(d.angVel[A]), vB = v3(d.vel[B]), wB = v3(d.angVel[B]);
    R fnSum = 0, snSum = 0, dMax = 0;
    V3<R> cSum{0, 0, 0}, nSum{0, 0, 0}, fAcc{0, 0, 0}, tA{0, 0, 0}, tB{0, 0, 0};
    const R snP = snPrev[idx];
    const R dampC = (mS > R(0)) ? R(-2) * R(0.9128709) * bd * sqrt(mS) : R(0);
    for (int k = 0; k < iter; ++k) {
      V3<R> pl{0, 0, 0};
      R prad = 0;
      if (cnt > 0)
        pl = v3(d.shell[dA.shellOffset + k]);
      else if (sphA)
        prad = dA.par[0] * sA;
      const V3<R> pw = add(pA, rot(qA, mul(pl, sA)));
      const V3<R> pc = mul(invrot(qB, sub(pw, pB)), R(1) / sB);
      const R dist = sdfShape(pc, dB, d.sdfGrid) * sB;
      const R eff = dist - prad;
      if (eff >= R(0))
        continue;
      const R delta = -eff;
      const V3<R> nl = sdfNormal(pc, dB, d.sdfGrid, R(1e-4));
      const V3<R> nW = rot(qB, nl);
      const V3<R> ps = sub(pw, mul(nW, prad));
      const V3<R> rA = sub(ps, pA);
      const V3<R> rB = sub(add(ps, mul(nW, delta)), pB);
      const V3<R> vrP = sub(add(vA, cross(wA, rA)), add(vB, cross(wB, rB)));
      const R vnP = dot(vrP, nW);
      const R sq = sqrt(rS * delta);
      const R fs = (R(4) / R(3)) * eS * sq * delta;
      const R snI = R(2) * eS * sq;
      const R snTot = (snP > snI) ? snP : snI;
      const R eta = dampC * snI / sqrt(snTot);
      const V3<R> f = mul(nW, fs - eta * vnP);
      fAcc = add(fAcc, f);
      tA = add(tA, cross(rA, f));
      tB = add(tB, cross(rB, mul(f, R(-1))));
      fnSum += fs;
      snSum += R(2) * eS * sq;
      cSum = add(cSum, mul(ps, fs));
      nSum = add(nSum, mul(nW, fs));
      if (delta > dMax)
        dMax = delta;
    }
    if (fnSum <= R(0)) {
      xi[idx] = Q4<R>{0, 0, 0, 0};
      snPrev[idx] = R(0);
      on[idx] = 0;
      continue;
    }
    const V3<R> cpt = mul(cSum, R(1) / fnSum);
    V3<R> nh = nSum;
    const R nl2 = vlen(nh);
    if (nl2 > R(1e-9))
      nh = mul(nh, R(1) / nl2);
    const V3<R> rA = sub(cpt, pA), rB = sub(cpt, pB);
    const V3<R> vr = sub(add(vA, cross(wA, rA)), add(vB, cross(wB, rB)));
    snPrev[idx] = snSum;
    const V3<R> vt = sub(vr, mul(nh, dot(vr, nh)));
    const R st = R(8) * gS * sqrt(rS * dMax);
    const R etaT = R(-2) * R(0.9128709) * bd * sqrt(st * mS);
    V3<R> x = v3(xi[idx]);
    x = add(x, mul(vt, P.dt));
    x = sub(x, mul(nh, dot(x, nh)));
    V3<R> ft = add(mul(x, -st), mul(vt, -etaT));
    const R fl = vlen(ft);
    const R fm = mu * fnSum;
    if (fl > fm) {
      const R s = (fl > R(1e-20)) ? fm / fl : R(0);
      ft = mul(ft, s);
      if (st > R(1e-20))
        x = mul(add(ft, mul(vt, etaT)), R(-1) / st);
    }
    xi[idx] = q4(x);
    fAcc = add(fAcc, ft);
    tA = add(tA, cross(rA, ft));
    tB = add(tB, cross(rB, mul(ft, R(-1))));
    F[idx] = q4(fAcc);
    TA[idx] = q4(tA);
    TB[idx] = q4(tB);
    on[idx] = 1;
  }
}

// wall candidates (src/solver_hertz.hpp:343-370), counted per particle then written in (i, wall)
// order: code i * 8 + wall
template <class R, int MODE>
__global__ void kHertzWallCand(Dev<R> d, int n, int numWalls, R skin, int* cnt, const int* off, int* out, int cap) {
  GRID_STRIDE(i, n) {
    const V3<R> p = v3(d.pos[i]);
    int c = 0;
    for (int wi = 0; wi < numWalls; ++wi) {
      const R s = sampleWall(p, d.walls[wi], d.wallGrid);
      if (s < d.rad[i] + skin) {
        if (MODE) {
          const int at = off[i] + c;
          if (at < cap)
            out[at] = (int)i * 8 + wi;
        }
        ++c;
      }
    }
    if (!MODE)
      cnt[i] = c;
  }
}

// wall forces per candidate (src/solver_hertz.hpp:148-338)
template <class R>
__global__ void kHertzWalls(Dev<R> d, int ncand, HertzP<R> P, const int* cand, Q4<R>* xiWall, R* snWall,
                            int hasShapes, Q4<R>* F, Q4<R>* T, int* on) {
  GRID_STRIDE(ci, ncand) {
    on[ci] = 0;
    const int enc = cand[ci];
    const int i = enc / 8, wi = enc % 8;
    const V3<R> p = v3(d.pos[i]);
    const R r = d.rad[i];
    const WallDesc<R>& w = d.walls[wi];
    const int slot = i * kHertzMaxWalls + wi;
    const int ma = d.matId[i];
    R e, mu;
    if (w.materialId >= 0 && d.pairMat)
      hertzEMu(d, ma, w.materialId, P.eG, P.muG, e, mu);
    else {
      e = w.restitution;
      mu = w.friction;
    }
    const int mw = (w.materialId >= 0) ? w.materialId : ma;
    R eS, gS;
    hertzStars(d, ma, mw, eS, gS);
    const R mS = (d.invMass[i] > R(0)) ? R(1) / d.invMass[i] : R(0);
    const V3<R> wl{w.linVel[0], w.linVel[1], w.linVel[2]}, wa{w.angVel[0], w.angVel[1], w.angVel[2]},
        wc{w.center[0], w.center[1], w.center[2]};
    const ShapeDesc<R> dS = d.shapes[d.shapeId[i]];
    if (hasShapes && dS.numPoints > 0) {
      const Q4<R> qP = d.quat[i];
      const R es = d.scale[i] * P.globalScale;
      const R rc = P.contactFrac * dS.par[0] * es;
      const R bd = hertzBetaD(e);
      const V3<R> vP = v3(d.vel[i]), wP = v3(d.angVel[i]);
      const R snP = snWall[slot];
      const R dampC = (mS > R(0)) ? R(-2) * R(0.9128709) * bd * sqrt(mS) : R(0);
      R fnSum = 0, snSum = 0, dMax = 0;
      V3<R> cSum{0, 0, 0}, nSum{0, 0, 0}, fAcc{0, 0, 0}, tAcc{0, 0, 0};
      for (int k = 0; k < dS.numPoints; ++k) {
        const V3<R> pW = add(p, rot(qP, mul(v3(d.shell[dS.shellOffset + k]), es)));
        const R sd = sampleWall(pW, w, d.wallGrid);
        if (sd >= R(0))
          continue;
        const R delta = -sd;
        const R hx = R(0.5) / w.invSpacing[0];
        const V3<R> gr = wallGradient(pW, w, d.wallGrid, hx);
        const R gl = vlen(gr);
        if (gl < R(1e-12))
          continue;
        const V3<R> nh = mul(gr, R(1) / gl);
        const V3<R> rA = sub(pW, p);
        const V3<R> vW = add(wl, cross(wa, sub(pW, wc)));
        const V3<R> vrP = sub(add(vP, cross(wP, rA)), vW);
        const R vnP = dot(vrP, nh);
        const R sq = sqrt(rc * delta);
        const R fs = (R(4) / R(3)) * eS * sq * delta;
        const R snI = R(2) * eS * sq;
        const R snTot = (snP > snI) ? snP : snI;
        const R eta = dampC * snI / sqrt(snTot);
        const V3<R> f = mul(nh, fs - eta * vnP);
        fAcc = add(fAcc, f);
        tAcc = add(tAcc, cross(rA, f));
        fnSum += fs;
        snSum += R(2) * eS * sq;
        cSum = add(cSum, mul(pW, fs));
        nSum = add(nSum, mul(nh, fs));
        if (delta > dMax)
          dMax = delta;
      }
      if (fnSum <= R(0)) {
        xiWall[slot] = Q4<R>{0, 0, 0, 0};
        snWall[slot] = R(0);
        continue;
      }
      const V3<R> cpt = mul(cSum, R(1) / fnSum);
      V3<R> nh = nSum;
      const R nl = vlen(nh);
      if (nl > R(1e-9))
        nh = mul(nh, R(1) / nl);
      const V3<R> rA = sub(cpt, p);
      const V3<R> vW = add(wl, cross(wa, sub(cpt, wc)));
      const V3<R> vr = sub(add(vP, cross(wP, rA)), vW);
      snWall[slot] = snSum;
      const V3<R> vt = sub(vr, mul(nh, dot(vr, nh)));
      const R st = R(8) * gS * sqrt(rc * dMax);
      const R etaT = R(-2) * R(0.9128709) * bd * sqrt(st * mS);
      V3<R> x = v3(xiWall[slot]);
      x = add(x, mul(vt, P.dt));
      x = sub(x, mul(nh, dot(x, nh)));
      V3<R> ft = add(mul(x, -st), mul(vt, -etaT));
      const R fl = vlen(ft);
      const R fm = mu * fnSum;
      if (fl > fm) {
        const R s2 = (fl > R(1e-20)) ? fm / fl : R(0);
        ft = mul(ft, s2);
        if (st > R(1e-20))
          x = mul(add(ft, mul(vt, etaT)), R(-1) / st);
      }
      xiWall[slot] = q4(x);
      fAcc = add(fAcc, ft);
      tAcc = add(tAcc, cross(rA, ft));
      F[ci] = q4(fAcc);
      T[ci] = q4(tAcc);
      on[ci] = 1;
      continue;
    }
    const R sw = sampleWall(p, w, d.wallGrid);
    const R delta = r - sw;
    if (delta <= R(0)) {
      xiWall[slot] = Q4<R>{0, 0, 0, 0};
      continue;
    }
    const R hx = R(0.5) / w.invSpacing[0];
    const V3<R> gr = wallGradient(p, w, d.wallGrid, hx);
    const R gl = sqrt(dot(gr, gr));
    if (gl < R(1e-12))
      continue;
    const V3<R> nh = mul(gr, R(1) / gl);
    const V3<R> rA = mul(nh, -(r - R(0.5) * delta));
    const V3<R> cpt = add(p, rA);
    const V3<R> vW = add(wl, cross(wa, sub(cpt, wc)));
    const V3<R> vr = sub(add(v3(d.vel[i]), cross(v3(d.angVel[i]), rA)), vW);
    V3<R> x = v3(xiWall[slot]);
    const V3<R> f = hertzForce(delta, nh, vr, r, mS, eS, gS, e, mu, P.dt, x);
    xiWall[slot] = q4(x);
    F[ci] = q4(f);
    T[ci] = q4(cross(rA, f));
    on[ci] = 1;
  }
}

// per body: pair contributions in pair order, then wall contributions in wall order; then the
// symplectic kick-drift (src/solver_hertz.hpp:374-425) with the forces consumed
template <class R>
__global__ void kHertzGatherIntegrate(Dev<R> d, int n, const int* incOff, const int* incEnt, const Q4<R>* F,
                                      const Q4<R>* TA, const Q4<R>* TB, const int* on, const int* candOff,
                                      int ncand, const Q4<R>* FW, const Q4<R>* TW, const int* onW, V3<R> g, R dt, int orient) {
  GRID_STRIDE(i, n) {
    // the reference accumulates into the (normally zero) delta arrays it uses as force/torque
    V3<R> f = v3(d.dVel[i]), t = v3(d.dAngVel[i]);
    for (int q = incOff[i]; q < incOff[i + 1]; ++q) {
      const int idx = incEnt[q] >> 1, side = incEnt[q] & 1;
      if (!on[idx])
        continue;
      if (side == 0) {
        f = add(f, v3(F[idx]));
        t = add(t, v3(TA[idx]));
      } else {
        f = add(f, neg(v3(F[idx])));
        t = add(t, v3(TB[idx]));
      }
    }
    if (candOff)
      for (int q = candOff[i]; q < candOff[i + 1] && q < ncand; ++q)
        if (onW[q]) {
          f = add(f, v3(FW[q]));
          t = add(t, v3(TW[q]));
        }
    const R im = d.invMass[i];
    if (im > R(0)) {
      const V3<R> iI = v3(d.invI[i]);
      V3<R> dw;
      if (iI.x == iI.y && iI.y == iI.z) {
        dw = V3<R>{t.x * iI.x, t.y * iI.x, t.z * iI.x};
      } else {
        const V3<R> tl = invrot(d.quat[i], t);
        dw = rot(d.quat[i], V3<R>{tl.x * iI.x, tl.y * iI.y, tl.z * iI.z});
      }
      V3<R> v = v3(d.vel[i]), w = v3(d.angVel[i]), x = v3(d.pos[i]);
      v.x += (f.x * im + g.x) * dt;
      w.x += dw.x * dt;
      x.x += v.x * dt;
      v.y += (f.y * im + g.y) * dt;
      w.y += dw.y * dt;
      x.y += v.y * dt;
      v.z += (f.z * im + g.z) * dt;
      w.z += dw.z * dt;
      x.z += v.z * dt;
      d.vel[i] = q4(v);
      d.angVel[i] = q4(w);
      d.pos[i] = q4(x);
      if (orient) {
        Q4<R> q = d.quat[i];
        const Q4<R> dq{R(0.5) * dt * (w.x * q.w + w.y * q.z - w.z * q.y),
                       R(0.5) * dt * (w.y * q.w + w.z * q.x - w.x * q.z),
                       R(0.5) * dt * (w.z * q.w + w.x * q.y - w.y * q.x),
                       R(0.5) * dt * (-w.x * q.x - w.y * q.y - w.z * q.z)};
        q = Q4<R>{q.x + dq.x, q.y + dq.y, q.z + dq.z, q.w + dq.w};
        const R qn = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        if (qn > R(1e-12))
          d.quat[i] = Q4<R>{q.x / qn, q.y / qn, q.z / qn, q.w / qn};
      }
    }
    d.dVel[i] = Q4<R>{0, 0, 0, 0};
    d.dAngVel[i] = Q4<R>{0, 0, 0, 0};
  }
}

template <class R>
__global__ void kHertzMaxDisp2(Dev<R> d, int n, const Q4<R>* ref, R* out) {
  R mx = R(0);
  GRID_STRIDE(i, n) {
    const V3<R> dd = sub(v3(d.pos[i]), v3(ref[i]));
    runMax(mx, dot(dd, dd));
  }
  blockMaxAtomic(out, mx);  // one atomic per block on the one word
}
// carry the shear history onto the rebuilt list (src/sim.hpp:558-585)
template <class R>
__global__ void kHertzCarry(Dev<R> d, int np, int prevCount, const u64* prevKeys, const Q4<R>* prevXi, u64* keys,
                            Q4<R>* xi) {
  GRID_STRIDE(idx, np) {
    const int2 pr = d.pairs[idx];
    const unsigned a = (unsigned)pr.x, b = (unsigned)pr.y;
    const unsigned lo = a < b ? a : b, hi = a < b ? b : a;
    const u64 k = ((u64)hi << 32) | lo;
    keys[idx] = k;
    int l = 0, h = prevCount;
    while (l < h) {
      const int m = (l + h) >> 1;
      if (prevKeys[m] < k)
        l = m + 1;
      else
        h = m;
    }
    const bool hit = l < prevCount && prevKeys[l] == k;
    xi[idx] = hit ? prevXi[l] : Q4<R>{0, 0, 0, 0};
  }
}
template <class R>
__global__ void kHertzGatherPrev(int n, const int* perm, const Q4<R>* xi, Q4<R>* prevXi) {
  GRID_STRIDE(i, n) prevXi[i] = xi[perm[i]];
}

}  // namespace pdem
