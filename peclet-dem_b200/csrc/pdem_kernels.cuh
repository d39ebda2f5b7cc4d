// Kernels of the B200 XPBD substep (src/sim.hpp:97-488 and the headers it calls).
//
// One kernel per reference stage, each reproducing the reference arithmetic exactly (same
// expression order, no FMA contraction) and the canonical serial order of every accumulation:
//  * ghosts, pairs and contacts are emitted by count -> exclusive scan -> write passes, so their
//    order is (particle, image), (i, j), (pair, shell point) / (particle, plane, point) /
//    (particle, wall, point) regardless of thread scheduling;
//  * manifold sums walk each manifold's contacts in ascending contact index (stable key sort);
//  * impulses that the reference scatters with atomics are gathered per body over an incidence
//    list sorted by source index;
//  * colour classes are independent sets, so a per-colour kernel updates bodies in place.
#pragma once
#include <cstdint>

#include "pdem_common.cuh"

namespace pdem {

// =============================================================================================
// integration (src/integration.hpp)
// =============================================================================================

// integration.hpp:44-93 — velocity predict (gravity, external force, gyroscopic term), x* and
// q*, deltas cleared
template <class R>
__global__ void kPredict(Dev<R> d, int n, V3<R> g, R dt) {
  GRID_STRIDE(i, n) {
    const R im = d.invMass[i];
    V3<R> v = v3(d.vel[i]);
    if (im > R(0)) {
      v = add(v, mul(g, dt));
      v = add(v, mul(v3(d.extForce[i]), im * dt));
    }
    d.velPred[i] = q4(v);
    V3<R> wp = v3(d.angVel[i]);
    if (im > R(0)) {
      const V3<R> ii = v3(d.invI[i]);
      if (ii.x > R(0) || ii.y > R(0) || ii.z > R(0)) {
        const Q4<R> q = d.quat[i];
        V3<R> wb = invrot(q, v3(d.angVel[i]));
        const V3<R> Ib{(ii.x > R(1e-9)) ? R(1) / ii.x : R(0), (ii.y > R(1e-9)) ? R(1) / ii.y : R(0),
                       (ii.z > R(1e-9)) ? R(1) / ii.z : R(0)};
        const V3<R> Lb{Ib.x * wb.x, Ib.y * wb.y, Ib.z * wb.z};
        const V3<R> wxL = cross(wb, Lb);
        const V3<R> al{-ii.x * wxL.x, -ii.y * wxL.y, -ii.z * wxL.z};
        wb = add(wb, mul(al, dt));
        wp = rot(q, wb);
      }
    }
    d.angVelPred[i] = q4(wp);
    V3<R> x = v3(d.pos[i]);
    if (im > R(0))
      x = add(x, mul(v, dt));
    d.posPred[i] = q4(x);
    d.quatPred[i] = d.quat[i];
    d.dVel[i] = Q4<R>{0, 0, 0, 0};
    d.dAngVel[i] = Q4<R>{0, 0, 0, 0};
    d.dPos[i] = Q4<R>{0, 0, 0, 0};
    d.counts[i] = 0;
  }
}

// integration.hpp:97-109
template <class R>
__global__ void kApplyVelocityDeltas(Dev<R> d, int n) {
  GRID_STRIDE(i, n) {
    d.velPred[i] = q4(add(v3(d.velPred[i]), v3(d.dVel[i])));
    d.angVelPred[i] = q4(add(v3(d.angVelPred[i]), v3(d.dAngVel[i])));
    d.dVel[i] = Q4<R>{0, 0, 0, 0};
    d.dAngVel[i] = Q4<R>{0, 0, 0, 0};
  }
}

// integration.hpp:112-148 — v persist, trapezoidal x*, quaternion integrate + normalise
template <class R>
__global__ void kApplyVelPredictPos(Dev<R> d, int n, R dt) {
  GRID_STRIDE(i, n) {
    const V3<R> vs = v3(d.vel[i]);
    const V3<R> vf = v3(d.velPred[i]);
    d.vel[i] = q4(vf);
    const R im = d.invMass[i];
    V3<R> x = v3(d.pos[i]);
    if (im > R(0))
      x = add(x, mul(add(vs, vf), R(0.5) * dt));
    d.posPred[i] = q4(x);
    const Q4<R> q = d.quat[i];
    const V3<R> w = v3(d.angVelPred[i]);
    d.angVel[i] = q4(w);
    Q4<R> qp = q;
    if (im > R(0)) {
      qp.x += R(0.5) * dt * (w.x * q.w + w.y * q.z - w.z * q.y);
      qp.y += R(0.5) * dt * (w.y * q.w + w.z * q.x - w.x * q.z);
      qp.z += R(0.5) * dt * (w.z * q.w + w.x * q.y - w.y * q.x);
      qp.w += R(0.5) * dt * (-w.x * q.x - w.y * q.y - w.z * q.z);
      const R l = sqrt(qp.x * qp.x + qp.y * qp.y + qp.z * qp.z + qp.w * qp.w);
      if (l > R(1e-9)) {
        const R s = R(1) / l;
        qp = Q4<R>{qp.x * s, qp.y * s, qp.z * s, qp.w * s};
      }
    }
    d.quatPred[i] = qp;
  }
}

// integration.hpp:168-184
template <class R>
__global__ void kApplyUpdates(Dev<R> d, int n) {
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

template <class R>
struct DomainP {
  R mn[3], mx[3], sz[3];
  int per[3];
};

// integration.hpp:187-215
template <class R>
__global__ void kFinalCommit(Dev<R> d, int n, DomainP<R> dom) {
  GRID_STRIDE(i, n) {
    Q4<R> p = d.posPred[i];
    R* c = &p.x;
    for (int a = 0; a < 3; ++a)
      if (dom.per[a]) {
        if (c[a] < dom.mn[a])
          c[a] += dom.sz[a];
        else if (c[a] >= dom.mx[a])
          c[a] -= dom.sz[a];
      }
    p.w = R(0);
    d.pos[i] = p;
    d.quat[i] = d.quatPred[i];
  }
}

// host rows (n x cols doubles, uploaded as they are) <-> the aligned 4-wide records of a field
template <class R>
__global__ void kPackRows(const double* src, int n, int cols, Q4<R>* dst) {
  GRID_STRIDE(i, n) {
    const double* r = src + (long)cols * i;
    dst[i] = Q4<R>{(R)r[0], (R)r[1], (R)r[2], cols == 4 ? (R)r[3] : R(0)};
  }
}
template <class R>
__global__ void kUnpackRows(const Q4<R>* src, int n, int cols, double* dst) {
  GRID_STRIDE(i, n) {
    const Q4<R> q = src[i];
    double* r = dst + (long)cols * i;
    r[0] = q.x;
    r[1] = q.y;
    r[2] = q.z;
    if (cols == 4)
      r[3] = q.w;
  }
}

// FP32-mixed form, end of a substep: the FP64 master positions and orientations advance by the
// substep's single-precision increment (the difference of two nearby floats, exact), periodic
// wrapping is applied in double, and the single-precision state is re-derived from the master,
// so rounding does not accumulate in the stored state across substeps.
template <class R>
__global__ void kMixedCommit(Dev<R> d, int n, DomainP<R> dom, Q4<double>* posD, Q4<double>* quatD) {
  GRID_STRIDE(i, n) {
    const Q4<R> pp = d.posPred[i], p0 = d.pos[i], qp = d.quatPred[i], q0 = d.quat[i];
    Q4<double> x = posD[i];
    x.x += (double)(pp.x - p0.x);
    x.y += (double)(pp.y - p0.y);
    x.z += (double)(pp.z - p0.z);
    double* c = &x.x;
    for (int a = 0; a < 3; ++a)
      if (dom.per[a]) {
        if (c[a] < (double)dom.mn[a])
          c[a] += (double)dom.sz[a];
        else if (c[a] >= (double)dom.mx[a])
          c[a] -= (double)dom.sz[a];
      }
    x.w = 0.0;
    Q4<double> q = quatD[i];
    q.x += (double)(qp.x - q0.x);
    q.y += (double)(qp.y - q0.y);
    q.z += (double)(qp.z - q0.z);
    q.w += (double)(qp.w - q0.w);
    const double qn = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (qn > 1e-12) {
      q.x /= qn, q.y /= qn, q.z /= qn, q.w /= qn;
    }
    posD[i] = x;
    quatD[i] = q;
    d.pos[i] = Q4<R>{(R)x.x, (R)x.y, (R)x.z, R(0)};
    d.quat[i] = Q4<R>{(R)q.x, (R)q.y, (R)q.z, (R)q.w};
  }
}

// integration.hpp:229-249 — kinetic energies summed in double in ascending index (one thread:
// the thermostat is an opt-in diagnostic path and must reproduce the serial sum bit for bit)
template <class R>
__global__ void kThermoEnergy(Dev<R> d, int n, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0)
    return;
  double kt = 0.0, kr = 0.0;
  for (int i = 0; i < n; ++i) {
    const R im = d.invMass[i];
    const V3<R> v = v3(d.vel[i]);
    if (im > R(0))
      kt += 0.5 * (1.0 / (double)im) * (double)(v.x * v.x + v.y * v.y + v.z * v.z);
    const V3<R> ii = v3(d.invI[i]);
    if (ii.x > R(0) || ii.y > R(0) || ii.z > R(0)) {
      const V3<R> wb = invrot(d.quat[i], v3(d.angVel[i]));
      const double Ix = (ii.x > R(0)) ? 1.0 / (double)ii.x : 0.0;
      const double Iy = (ii.y > R(0)) ? 1.0 / (double)ii.y : 0.0;
      const double Iz = (ii.z > R(0)) ? 1.0 / (double)ii.z : 0.0;
      kr += 0.5 * (Ix * (double)wb.x * (double)wb.x + Iy * (double)wb.y * (double)wb.y +
                   Iz * (double)wb.z * (double)wb.z);
    }
  }
  out[0] = kt;
  out[1] = kr;
}
template <class R>
__global__ void kThermoScale(Dev<R> d, int n, R lt, R lr) {
  GRID_STRIDE(i, n) {
    d.vel[i] = q4(mul(v3(d.vel[i]), lt));
    d.angVel[i] = q4(mul(v3(d.angVel[i]), lr));
  }
}

// integration.hpp:275-283
template <class R>
__global__ void kGrowthScales(Dev<R> d, int n, R factor) {
  GRID_STRIDE(i, n) d.scale[i] = d.targetScale[i] * factor;
}

// sim.hpp:61-70 partial: max scale over [0, n) (non-negative scales; order-free max)
template <class R>
__global__ void kMaxScale(Dev<R> d, int n, R* out) {
  R m = R(0);
  GRID_STRIDE(i, n) runMax(m, d.scale[i]);
  blockMaxAtomic(out, m);
}

// batched form: largest scale of every scene (out[s] zeroed by the host)
template <class R>
__global__ void kSceneMaxScale(Dev<R> d, int n, R* out) {
  GRID_STRIDE(i, n) atomicMaxNonNeg(&out[d.sceneOf[i]], d.scale[i]);
}
// batched form, start of a substep: per-scene parameters (margin, restitution, friction; params =
// 3 values per scene) and loop state reset as the single-scene Counters are; maxApproach persists
template <class R>
__global__ void kSceneBegin(SceneCtl<R>* scn, int S, const R* params) {
  GRID_STRIDE(s, S) {
    SceneCtl<R> q = scn[s];
    const R keep = q.maxApproach;
    q = SceneCtl<R>{};
    q.maxApproach = keep;
    q.margin = params[3 * s];
    q.eN = params[3 * s + 1];
    q.mu = params[3 * s + 2];
    scn[s] = q;
  }
}
// batched form: first entry of every scene in the body-sorted range [b, e) of an entry array whose
// first body is ab[].x (pair / plane / wall contacts, manifolds); out[S] = e
__global__ void kSceneBounds(const int2* ab, int b, int e, int S, const int* sceneFirst, int* out) {
  GRID_STRIDE(s, S + 1) {
    const int body = sceneFirst[s];
    int lo = b, hi = e;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (ab[mid].x < body)
        lo = mid + 1;
      else
        hi = mid;
    }
    out[s] = lo;
  }
}

// per-detection counter reset; maxApproach persists across substeps like the reference's View
// (a step with no velocity sweep reads the previous one's residual)
template <class R>
__global__ void kResetCounters(Counters<R>* c) {
  if (threadIdx.x | blockIdx.x)
    return;
  const R keep = c->maxApproach;
  *c = Counters<R>{};
  c->maxApproach = keep;
}

template <class R>
__global__ void kIota(int* a, int n) {
  GRID_STRIDE(i, n) a[i] = (int)i;
}

template <class R>
__global__ void kRadii(Dev<R> d, int n, R gs, R bR) {
  GRID_STRIDE(i, n) d.rad[i] = d.scale[i] * gs * bR;
}

// =============================================================================================
// periodic ghosts (src/periodicity.hpp:43-94): count images per real particle, scan, emit in
// (particle, image) order; slots beyond capacity are dropped like the reference's overflow
// =============================================================================================
template <class R>
__device__ __forceinline__ void ghostShifts(const DomainP<R>& dom, V3<R> p, R skin, int s[3]) {
  s[0] = dom.per[0] ? ((p.x < dom.mn[0] + skin) ? 1 : ((p.x > dom.mx[0] - skin) ? -1 : 0)) : 0;
  s[1] = dom.per[1] ? ((p.y < dom.mn[1] + skin) ? 1 : ((p.y > dom.mx[1] - skin) ? -1 : 0)) : 0;
  s[2] = dom.per[2] ? ((p.z < dom.mn[2] + skin) ? 1 : ((p.z > dom.mx[2] - skin) ? -1 : 0)) : 0;
}
template <class R>
__global__ void kGhostCount(Dev<R> d, int n, DomainP<R> dom, R skin, int* cnt) {
  GRID_STRIDE(i, n) {
    int s[3];
    ghostShifts(dom, v3(d.pos[i]), skin, s);
    const int nx = s[0] ? 2 : 1, ny = s[1] ? 2 : 1, nz = s[2] ? 2 : 1;
    cnt[i] = nx * ny * nz - 1;
  }
}
template <class R>
__global__ void kGhostWrite(Dev<R> d, int n, DomainP<R> dom, R skin, const int* off) {
  GRID_STRIDE(i, n) {
    const V3<R> p = v3(d.pos[i]);
    int s[3];
    ghostShifts(dom, p, skin, s);
    const int ax[2] = {0, s[0]}, ay[2] = {0, s[1]}, az[2] = {0, s[2]};
    const int nx = s[0] ? 2 : 1, ny = s[1] ? 2 : 1, nz = s[2] ? 2 : 1;
    const V3<R> pp = v3(d.posPred[i]);
    int slot = n + off[i];
    for (int a = 0; a < nx; ++a)
      for (int b = 0; b < ny; ++b)
        for (int c = 0; c < nz; ++c) {
          const int ix = ax[a], iy = ay[b], iz = az[c];
          if (ix == 0 && iy == 0 && iz == 0)
            continue;
          const int g = slot++;
          if (g >= d.cap)
            continue;
          const V3<R> sh{ix * dom.sz[0], iy * dom.sz[1], iz * dom.sz[2]};
          d.pos[g] = q4(add(p, sh));
          d.posPred[g] = q4(add(pp, sh));
          d.invMass[g] = d.invMass[i];
          d.vel[g] = d.vel[i];
          d.velPred[g] = d.velPred[i];
          d.quat[g] = d.quat[i];
          d.quatPred[g] = d.quatPred[i];
          d.angVel[g] = d.angVel[i];
          d.angVelPred[g] = d.angVelPred[i];
          d.scale[g] = d.scale[i];
          d.shapeId[g] = d.shapeId[i];
          d.realIdx[g] = (int)i;
        }
  }
}

}  // namespace pdem
