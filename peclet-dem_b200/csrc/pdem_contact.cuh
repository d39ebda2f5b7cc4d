// Narrowphase, contact -> manifold reduction, warm-start ledger, support levels and colouring.
//
// Narrowphase (src/narrowphase.hpp:179-449): A's point shell (or, for a sphere, its centre with the
// sphere radius) probes B's canonical-space SDF; plane and world-grid wall contacts per particle.
// Analytic spheres run one thread per pair/particle; point shells run one warp per pair/particle
// with the warp's points in shell order, the per-warp ballot prefix giving each contact its slot,
// so contacts come out in (pair, k) / (particle, plane, k) / (particle, wall, k) order.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include "pdem_common.cuh"

namespace pdem {
namespace cg = cooperative_groups;

template <class R>
struct NarrowP {
  R margin, globalScale;
  int numPlanes, numWalls;
  int haveMat;
};

// walls that body i meets: all of them, or (batched form) those of its scene, in wall order
template <class R>
__device__ __forceinline__ int wallBegin(const Dev<R>& d, int i) {
  return d.sceneWallOff ? d.sceneWallOff[d.sceneOf[i]] : 0;
}
template <class R>
__device__ __forceinline__ int wallEnd(const Dev<R>& d, const NarrowP<R>& P, int i) {
  return d.sceneWallOff ? d.sceneWallOff[d.sceneOf[i] + 1] : P.numWalls;
}
template <class R>
__device__ __forceinline__ int wallAt(const Dev<R>& d, int q) {
  return d.sceneWallIdx ? d.sceneWallIdx[q] : q;
}
// contact margin of body i's scene, and the running max of the overlap (per scene when batched)
template <class R>
__device__ __forceinline__ R marginOf(const Dev<R>& d, const NarrowP<R>& P, int i) {
  return d.scn ? d.scn[d.sceneOf[i]].margin : P.margin;
}
template <class R>
__device__ __forceinline__ void overlapMax(const Dev<R>& d, int i, R v, R& mo) {
  if (d.scn) {
    // the lanes here that share a scene (a scene's bodies are contiguous, so usually the whole
    // warp) reduce first: one atomic per scene per warp, not one per overlapping body
    const int sc = d.sceneOf[i];
    const auto peers = cg::labeled_partition(cg::coalesced_threads(), sc);
    const R m = cg::reduce(peers, v, cg::greater<R>());
    if (peers.thread_rank() == 0)
      atomicMaxNonNeg(&d.scn[sc].maxOverlap, m);
  } else {
    runMax(mo, v);
  }
}

// ---------------------------------------------------------------------------------------------
// body-body probe of point k of A against B (src/narrowphase.hpp:192-265)
template <class R>
struct Probe {
  V3<R> pw, pc;
  R prad, eff;
};
template <class R>
__device__ __forceinline__ Probe<R> probeBody(const Dev<R>& d, int A, int B, int k, const ShapeDesc<R>& dA,
                                             const ShapeDesc<R>& dB, R gs, const Q4<R>* shell = nullptr) {
  const V3<R> pA = v3(d.posPred[A]), pB = v3(d.posPred[B]);
  const Q4<R> qA = d.quatPred[A], qB = d.quatPred[B];
  const R sA = d.scale[A] * gs, sB = d.scale[B] * gs;
  V3<R> pl{0, 0, 0};
  Probe<R> r;
  r.prad = R(0);
  if (dA.numPoints > 0)
    pl = v3(shell ? shell[k] : d.shell[dA.shellOffset + k]);
  else if (dA.type == SHAPE_SPHERE)
    r.prad = dA.par[0] * sA;
  r.pw = add(pA, rot(qA, mul(pl, sA)));
  const V3<R> plB = invrot(qB, sub(r.pw, pB));
  r.pc = mul(plB, R(1) / sB);
  const R dist = sdfShape(r.pc, dB, d.sdfGrid) * sB;
  r.eff = dist - r.prad;
  return r;
}
template <class R>
__device__ __forceinline__ void writeBodyContact(const Dev<R>& d, int slot, int A, int B, const Probe<R>& p,
                                                 const ShapeDesc<R>& dB, const NarrowP<R>& np) {
  const Q4<R> qB = d.quatPred[B];
  const V3<R> pA = v3(d.posPred[A]), pB = v3(d.posPred[B]);
  const V3<R> nl = sdfNormal(p.pc, dB, d.sdfGrid, R(1e-4));
  const V3<R> nw = rot(qB, nl);
  const V3<R> ps = sub(p.pw, mul(nw, p.prad));
  const V3<R> rA = sub(ps, pA);
  const V3<R> rB = sub(sub(ps, mul(nw, p.eff)), pB);
  R e = R(-1), mu = R(-1);
  if (np.haveMat) {
    const int t = (int(d.matId[A]) * kMaxMaterials + int(d.matId[B])) * 2;
    e = d.pairMat[t];
    mu = d.pairMat[t + 1];
  }
  d.cab[slot] = make_int2(A, B);
  d.cn[slot] = q4(nw, p.eff);
  d.crA[slot] = q4(rA, R(0));
  d.crB[slot] = q4(rB, e);
  d.cbv[slot] = Q4<R>{0, 0, 0, mu};
}

// spheres (no shell): one thread per pair. MODE 0: count + max overlap; MODE 1: write
template <class R, int MODE>
__global__ void kNarrowSphere(Dev<R> d, int np, NarrowP<R> P, int* cnt, const int* off) {
  const ShapeDesc<R> dA = d.shapes[0], dB = d.shapes[0];
  R mo = R(0);
  GRID_STRIDE(idx, np) {
    // the write pass revisits only the pairs the count pass found in contact (off[idx + 1] is
    // the exclusive scan of the 0/1 counts)
    if (MODE == 1 && off[idx + 1] == off[idx])
      continue;
    const int2 pr = d.pairs[idx];
    const Probe<R> p = probeBody(d, pr.x, pr.y, 0, dA, dB, P.globalScale);
    const bool hit = p.eff < marginOf(d, P, pr.x);
    if (MODE == 0) {
      if (p.eff < R(0))
        overlapMax(d, pr.x, -p.eff, mo);
      cnt[idx] = hit ? 1 : 0;
    } else if (hit) {
      const int s = off[idx];
      if (s < d.maxContacts)
        writeBodyContact(d, s, pr.x, pr.y, p, dB, P);
    }
  }
  if (MODE == 0)
    warpMaxAtomic(&d.ctr->maxOverlap, mo);
}

// spheres, write pass: one thread per contact slot s, whose pair is hitIdx[s] (the pairs the count
// pass found in contact, in pair order), so every lane of a warp writes a contact
__global__ void kHitIndex(int np, const int* off, int* hitIdx) {
  GRID_STRIDE(idx, np) {
    const int o = off[idx];
    if (off[idx + 1] != o)
      hitIdx[o] = (int)idx;
  }
}
template <class R>
__global__ void kNarrowSphereWrite(Dev<R> d, int nhit, NarrowP<R> P, const int* hitIdx) {
  const ShapeDesc<R> dA = d.shapes[0], dB = d.shapes[0];
  GRID_STRIDE(s, nhit) {
    if (s >= d.maxContacts)
      break;
    const int2 pr = d.pairs[hitIdx[s]];
    const Probe<R> p = probeBody(d, pr.x, pr.y, 0, dA, dB, P.globalScale);
    writeBodyContact(d, (int)s, pr.x, pr.y, p, dB, P);
  }
}

// ---- one-dimensional bulk copies (TMA) into shared memory, completed on an mbarrier ----
__device__ __forceinline__ unsigned smemAddr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbarInit(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbarExpectTx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
// src and dst 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulkCopyToShared(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smemAddr(dst)),
               "l"(src), "r"(bytes), "r"(smemAddr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbarTryWait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
constexpr long kStageSpins = 1L << 22;  // polls of a staging wait before the block reads global memory

// point shells: one warp per pair, lanes over shell points in order. With stageBytes > 0 (the
// shape's whole shell, kept small) the block first copies the shell into shared memory with one
// bulk copy: every warp of the block probes the same points. A staging wait that runs out (it
// should not: the copy is a few KB) leaves the block reading the shell from global memory, after
// waiting, bounded again, for the copy so that none is in flight when the block ends.
template <class R, int MODE>
__global__ void kNarrowShell(Dev<R> d, int np, NarrowP<R> P, int* cnt, const int* off, int stageBytes) {
  extern __shared__ __align__(128) unsigned char shellSmem[];
  __shared__ __align__(8) unsigned long long stageBar;
  const ShapeDesc<R> dA = d.shapes[0], dB = d.shapes[0];
  const Q4<R>* shell = nullptr;
  if (stageBytes > 0) {
    if (threadIdx.x == 0) {
      mbarInit(&stageBar, 1);
      mbarExpectTx(&stageBar, (unsigned)stageBytes);
      bulkCopyToShared(shellSmem, d.shell + dA.shellOffset, (unsigned)stageBytes, &stageBar);
    }
    __syncthreads();  // the barrier is initialised before anyone polls it
    long spins = 0;
    bool ok = false;
    while (!(ok = mbarTryWait(&stageBar, 0)) && ++spins < kStageSpins) {
    }
    if (__syncthreads_and(ok)) {
      shell = reinterpret_cast<const Q4<R>*>(shellSmem);
    } else {
      while (!mbarTryWait(&stageBar, 0) && ++spins < 2 * kStageSpins) {
      }
    }
  }
  const int lane = threadIdx.x & 31;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  const int K = dA.numPoints > 0 ? dA.numPoints : 1;
  R mo = R(0);
  for (long idx = warp; idx < np; idx += nwarps) {
    const int2 pr = d.pairs[idx];
    int running = MODE ? off[idx] : 0;
    int total = 0;
    for (int k0 = 0; k0 < K; k0 += 32) {
      const int k = k0 + lane;
      bool hit = false;
      Probe<R> p;
      if (k < K) {
        p = probeBody(d, pr.x, pr.y, k, dA, dB, P.globalScale, shell);
        hit = p.eff < marginOf(d, P, pr.x);
        if (MODE == 0 && p.eff < R(0))
          overlapMax(d, pr.x, -p.eff, mo);
      }
      const unsigned b = __ballot_sync(0xffffffffu, hit);
      if (MODE == 1 && hit) {
        const int s = running + __popc(b & ((1u << lane) - 1u));
        if (s < d.maxContacts)
          writeBodyContact(d, s, pr.x, pr.y, p, dB, P);
      }
      running += __popc(b);
      total += __popc(b);
    }
    if (MODE == 0 && lane == 0)
      cnt[idx] = total;
  }
  if (MODE == 0)
    warpMaxAtomic(&d.ctr->maxOverlap, mo);
}

// ---------------------------------------------------------------------------------------------
// planes (src/narrowphase.hpp:371-449) and walls (:278-367), per real particle
template <class R>
struct BoundaryProbe {
  V3<R> rA, n, pWall;
  R dist;
  bool hit;
};

template <class R>
__device__ __forceinline__ BoundaryProbe<R> probePlane(const Dev<R>& d, int i, int pl, int k, const ShapeDesc<R>& sd,
                                                      R s, R margin) {
  const PlaneDesc<R> P = d.planes[pl];
  const V3<R> pp{P.p[0], P.p[1], P.p[2]}, pn{P.n[0], P.n[1], P.n[2]};
  const V3<R> pA = v3(d.posPred[i]);
  BoundaryProbe<R> r;
  if (sd.numPoints > 0) {
    r.rA = rot(d.quatPred[i], mul(v3(d.shell[sd.shellOffset + k]), s));
    const V3<R> pw = add(pA, r.rA);
    r.dist = dot(sub(pw, pp), pn);
  } else {
    R bR = sd.par[0];
    if (bR == R(0))
      bR = R(1);
    const R radius = bR * s;
    r.dist = dot(sub(pA, pp), pn) - radius;
    r.rA = mul(pn, -radius);
  }
  r.n = pn;
  r.pWall = pp;
  r.hit = r.dist < margin;
  return r;
}
// A shell particle whose centre is farther from plane pl than its shell's reach plus the margin has
// no point within the margin and none below the plane: every point's distance is the centre's plus
// the projection of its offset rot(q, p s), and rot(q, v) = q v q* + (1 - |q|^2) v has norm at most
// (|q|^2 + |1 - |q|^2|) |v| <= that factor * shellR * s. The test keeps a slack of 1e-4 of the
// magnitudes involved (far above the rounding of either computation), so it only skips particles
// whose probes would all miss.
template <class R>
__device__ __forceinline__ bool planeOutOfReach(const Dev<R>& d, int i, int pl, const ShapeDesc<R>& sd, R s,
                                                R margin) {
  if (sd.numPoints <= 0)
    return false;
  const PlaneDesc<R> P = d.planes[pl];
  const V3<R> pp{P.p[0], P.p[1], P.p[2]}, pn{P.n[0], P.n[1], P.n[2]};
  const V3<R> pA = v3(d.posPred[i]);
  const R distC = dot(sub(pA, pp), pn);
  const Q4<R> q = d.quatPred[i];
  const R qn2 = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
  const R reach = sd.shellR * s * (qn2 + fabs(R(1) - qn2)) * sqrt(dot(pn, pn));
  const R mag = fabs(distC) + reach + fabs(margin) + fabs(pA.x) + fabs(pA.y) + fabs(pA.z) + fabs(pp.x) +
                fabs(pp.y) + fabs(pp.z);
  return distC - reach > margin + R(1e-4) * mag;
}
template <class R>
__device__ __forceinline__ BoundaryProbe<R> probeWall(const Dev<R>& d, int i, int wi, int k, const ShapeDesc<R>& sd,
                                                     R s, R margin, bool needNormal) {
  const WallDesc<R>& w = d.walls[wi];
  const V3<R> pA = v3(d.posPred[i]);
  R bR = sd.par[0];
  if (bR == R(0))
    bR = R(1);
  const R radius = bR * s;
  BoundaryProbe<R> r;
  V3<R> rA{0, 0, 0};
  if (sd.numPoints > 0)
    rA = rot(d.quatPred[i], mul(v3(d.shell[sd.shellOffset + k]), s));
  const V3<R> pw = add(pA, rA);
  const R sdf = sampleWall(pw, w, d.wallGrid);
  r.dist = (sd.numPoints > 0) ? sdf : sdf - radius;
  r.hit = r.dist < margin;
  if (needNormal && r.hit) {
    V3<R> n = wallGradient(pw, w, d.wallGrid, R(1e-4));
    const R ln = vlen(n);
    n = (ln > R(1e-9)) ? mul(n, R(1) / ln) : V3<R>{0, 1, 0};
    r.n = n;
    r.rA = (sd.numPoints > 0) ? rA : mul(n, -radius);
    const V3<R> ps = add(pA, r.rA);
    r.pWall = sub(ps, mul(n, r.dist));
  }
  return r;
}
template <class R>
__device__ __forceinline__ void writeBoundaryContact(const Dev<R>& d, int slot, int i, const BoundaryProbe<R>& b,
                                                     bool wall, int wi, int haveMat) {
  d.cab[slot] = make_int2(i, -1);
  d.cn[slot] = q4(b.n, b.dist);
  d.crA[slot] = q4(b.rA, R(0));
  if (!wall) {
    d.crB[slot] = q4(b.pWall, R(-1));
    d.cbv[slot] = Q4<R>{0, 0, 0, R(-1)};
    return;
  }
  const WallDesc<R>& w = d.walls[wi];
  const V3<R> r = sub(b.pWall, V3<R>{w.center[0], w.center[1], w.center[2]});
  const V3<R> vW = add(V3<R>{w.linVel[0], w.linVel[1], w.linVel[2]}, cross(V3<R>{w.angVel[0], w.angVel[1], w.angVel[2]}, r));
  R e, mu;
  if (w.materialId >= 0 && haveMat) {
    const int t = (int(d.matId[i]) * kMaxMaterials + w.materialId) * 2;
    e = d.pairMat[t];
    mu = d.pairMat[t + 1];
  } else {
    e = w.restitution;
    mu = w.friction;
  }
  d.crB[slot] = q4(b.pWall, e);
  d.cbv[slot] = q4(vW, mu);
}

// one warp per real particle, planes then walls, lanes over shell points (or lane 0 for a
// sphere). MODE 0 counts (planes in cntP, walls in cntW) and records the max overlap; MODE 1 writes
// at base + offsets.
template <class R, int MODE>
__global__ void kBoundary(Dev<R> d, int numReal, NarrowP<R> P, int* cntP, int* cntW, const int* offP,
                          const int* offW, int basePlanes, int baseWalls) {
  const ShapeDesc<R> sd = d.shapes[0];
  const int lane = threadIdx.x & 31;
  const long warp = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  const int K = sd.numPoints > 0 ? sd.numPoints : 1;
  R mo = R(0);
  for (long i = warp; i < numReal; i += nwarps) {
    const R s = d.scale[i] * P.globalScale;
    int run = MODE ? basePlanes + offP[i] : 0, tot = 0;
    for (int pl = 0; pl < P.numPlanes; ++pl) {
      if (planeOutOfReach(d, (int)i, pl, sd, s, marginOf(d, P, (int)i)))
        continue;  // uniform over the warp (one particle)
      for (int k0 = 0; k0 < K; k0 += 32) {
        const int k = k0 + lane;
        BoundaryProbe<R> b;
        b.hit = false;
        if (k < K) {
          b = probePlane(d, (int)i, pl, k, sd, s, marginOf(d, P, (int)i));
          if (MODE == 0 && b.dist < R(0))
            overlapMax(d, (int)i, -b.dist, mo);
        }
        const unsigned m = __ballot_sync(0xffffffffu, b.hit);
        if (MODE == 1 && b.hit) {
          const int slot = run + __popc(m & ((1u << lane) - 1u));
          if (slot < d.maxContacts)
            writeBoundaryContact(d, slot, (int)i, b, false, 0, 0);
        }
        run += __popc(m);
        tot += __popc(m);
      }
    }
    if (MODE == 0 && lane == 0)
      cntP[i] = tot;
    run = MODE ? baseWalls + offW[i] : 0;
    tot = 0;
    for (int q = wallBegin(d, (int)i); q < wallEnd(d, P, (int)i); ++q) {
      const int wi = wallAt(d, q);
      for (int k0 = 0; k0 < K; k0 += 32) {
        const int k = k0 + lane;
        BoundaryProbe<R> b;
        b.hit = false;
        if (k < K) {
          b = probeWall(d, (int)i, wi, k, sd, s, marginOf(d, P, (int)i), MODE == 1);
          if (MODE == 0 && b.dist < R(0))
            overlapMax(d, (int)i, -b.dist, mo);
        }
        const unsigned m = __ballot_sync(0xffffffffu, b.hit);
        if (MODE == 1 && b.hit) {
          const int slot = run + __popc(m & ((1u << lane) - 1u));
          if (slot < d.maxContacts)
            writeBoundaryContact(d, slot, (int)i, b, true, wi, P.haveMat);
        }
        run += __popc(m);
        tot += __popc(m);
      }
    }
    if (MODE == 0 && lane == 0)
      cntW[i] = tot;
  }
  if (MODE == 0)
    warpMaxAtomic(&d.ctr->maxOverlap, mo);
}

// single-point shapes (spheres): one thread per particle, same slots as kBoundary. The write pass
// (MODE 1) writes the plane contacts only, visiting the particles that have some; the wall contacts
// are written by kBoundaryWallSphere, one thread per contact.
template <class R, int MODE>
__global__ void kBoundarySphere(Dev<R> d, int numReal, NarrowP<R> P, int* cntP, int* cntW, const int* offP,
                                int basePlanes) {
  const ShapeDesc<R> sd = d.shapes[0];
  R mo = R(0);
  GRID_STRIDE(i, numReal) {
    if (MODE == 1 && offP[i + 1] == offP[i])
      continue;
    const R s = d.scale[i] * P.globalScale;
    int run = MODE ? basePlanes + offP[i] : 0, tot = 0;
    for (int pl = 0; pl < P.numPlanes; ++pl) {
      const BoundaryProbe<R> b = probePlane(d, (int)i, pl, 0, sd, s, marginOf(d, P, (int)i));
      if (MODE == 0 && b.dist < R(0))
        overlapMax(d, (int)i, -b.dist, mo);
      if (b.hit) {
        if (MODE == 1 && run < d.maxContacts)
          writeBoundaryContact(d, run, (int)i, b, false, 0, 0);
        ++run;
        ++tot;
      }
    }
    if (MODE == 1)
      continue;
    cntP[i] = tot;
    tot = 0;
    for (int q = wallBegin(d, (int)i); q < wallEnd(d, P, (int)i); ++q) {
      const int wi = wallAt(d, q);
      const BoundaryProbe<R> b = probeWall(d, (int)i, wi, 0, sd, s, marginOf(d, P, (int)i), false);
      if (b.dist < R(0))
        overlapMax(d, (int)i, -b.dist, mo);
      if (b.hit)
        ++tot;
    }
    cntW[i] = tot;
  }
  if (MODE == 0)
    warpMaxAtomic(&d.ctr->maxOverlap, mo);
}
// wall contacts of spheres, one thread per contact: contact t belongs to the particle i with
// offW[i] <= t < offW[i + 1] (offW: exclusive scan of the count pass's wall hits, numReal + 1
// entries) and is its (t - offW[i])-th hitting wall in wall order, the count pass's hit test
// repeated; the slot is baseWalls + t, as in the per-particle order. Only the contacts pay for the
// wall normal (six more grid samples), and no lane idles beside them.
template <class R>
__global__ void kBoundaryWallSphere(Dev<R> d, int total, int numReal, NarrowP<R> P, const int* offW, int baseWalls) {
  const ShapeDesc<R> sd = d.shapes[0];
  GRID_STRIDE(t, total) {
    int lo = 0, hi = numReal;  // largest i with offW[i] <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (offW[mid] <= (int)t)
        lo = mid;
      else
        hi = mid - 1;
    }
    const int i = lo;
    int k = (int)t - offW[i];
    const R s = d.scale[i] * P.globalScale;
    const R margin = marginOf(d, P, i);
    for (int q = wallBegin(d, i); q < wallEnd(d, P, i); ++q) {
      const int wi = wallAt(d, q);
      if (!probeWall(d, i, wi, 0, sd, s, margin, false).hit)
        continue;
      if (k-- > 0)
        continue;
      const int slot = baseWalls + (int)t;
      if (slot < d.maxContacts)
        writeBoundaryContact(d, slot, i, probeWall(d, i, wi, 0, sd, s, margin, true), true, wi, P.haveMat);
      break;
    }
  }
}

// =============================================================================================
// contact -> manifold (src/contact_preprocessing.hpp:320-471)
// =============================================================================================
// Key of a contact's body pair, (smaller index, larger index or "none" for a boundary contact),
// packed as u << bits | v with the all-ones v for "none": the same order as the reference's
// (u << 32 | v) pair key with 0xFFFFFFFF for a boundary, in 2 * bits bits (fewer sort passes).
// bits is chosen so that every body index is below 2^bits - 1.
template <class R>
__global__ void kContactKeys(Dev<R> d, int nc, int bits, u64* keys, int* vals) {
  const u64 none = (1ull << bits) - 1ull;
  GRID_STRIDE(i, nc) {
    const int2 ab = d.cab[i];
    u64 k;
    if (ab.y < 0)
      k = ((u64)(unsigned)ab.x << bits) | none;
    else {
      const unsigned u = ab.x < ab.y ? ab.x : ab.y, v = ab.x < ab.y ? ab.y : ab.x;
      k = ((u64)u << bits) | v;
    }
    keys[i] = k;
    vals[i] = (int)i;
  }
}
// The stable key sort of the contact list, done as a rank scatter. The narrowphase writes
// [body-pair contacts in pair order] ++ [plane contacts by particle] ++ [wall contacts by particle];
// the broadphase gives pairs (lo, hi), lo < hi, lo real, sorted by (lo, hi), so the pair contacts
// are already in key order. A boundary key (i, none) sorts after every pair key (i, v) and before
// (i + 1, ...), and the plane contacts of a particle precede its wall contacts (list order). Ranks:
// pair contact p with first body a -> p + the boundary contacts of particles below a (offP[a] +
// offW[a]); the k-th plane contact of particle i -> the pair contacts with first body <= i, +
// offP[i] + offW[i] + k; its k-th wall contact -> the same base + offP[i + 1] - offP[i] + k. A list
// that breaks these premises (pair contacts out of key order, a non-real first body, counts that do
// not match the offsets) sets *bad and the caller sorts instead; every write stays inside [0, nc).
template <class R>
__global__ void kContactRanks(Dev<R> d, int nc, int nPair, int nPlane, int numReal, const int* offP,
                              const int* offW, int bits, u64* keysOut, int* permOut, int* bad) {
  const u64 none = (1ull << bits) - 1ull;
  auto pairKey = [&](int2 ab) {
    const unsigned u = ab.x < ab.y ? ab.x : ab.y, v = ab.x < ab.y ? ab.y : ab.x;
    return ((u64)u << bits) | v;
  };
  GRID_STRIDE(t, nc) {
    const int2 ab = d.cab[t];
    long rank = -1;
    u64 k = 0;
    if (t < nPair) {
      const int a = ab.x < ab.y ? ab.x : ab.y;
      if (ab.y < 0 || a < 0 || a >= numReal || (t > 0 && pairKey(d.cab[t - 1]) > pairKey(ab))) {
        atomicOr(bad, 1);
        continue;
      }
      k = pairKey(ab);
      rank = t + offP[a] + offW[a];
    } else {
      const int i = ab.x;
      if (ab.y >= 0 || i < 0 || i >= numReal) {
        atomicOr(bad, 1);
        continue;
      }
      k = ((u64)(unsigned)i << bits) | none;
      int lo = 0, hi = nPair;  // pair contacts with first body <= i
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const int2 m = d.cab[mid];
        if ((m.x < m.y ? m.x : m.y) <= i)
          lo = mid + 1;
        else
          hi = mid;
      }
      const bool plane = t < nPair + nPlane;
      const long kk = plane ? t - nPair - offP[i] : t - nPair - nPlane - offW[i];
      const long cnt = plane ? offP[i + 1] - offP[i] : offW[i + 1] - offW[i];
      if (kk < 0 || kk >= cnt) {
        atomicOr(bad, 1);
        continue;
      }
      rank = (long)lo + (plane ? offP[i] : offP[i + 1]) + offW[i] + kk;
    }
    if (rank < 0 || rank >= nc) {
      atomicOr(bad, 1);
      continue;
    }
    keysOut[rank] = k;
    permOut[rank] = (int)t;
  }
}
__global__ void kSegHeads(int n, const u64* keys, int* head) {
  GRID_STRIDE(p, n) head[p] = (p == 0 || keys[p] != keys[p - 1]) ? 1 : 0;
}
// segStart[s] = first sorted position of segment s (inclusive scan of heads gives s + 1)
__global__ void kSegStarts(int n, const int* headScan, int* segStart) {
  GRID_STRIDE(p, n) {
    const int s = headScan[p] - 1;
    if (p == 0 || headScan[p] != headScan[p - 1])
      segStart[s] = (int)p;
  }
}
// one thread per manifold: ordered sums over the segment's contacts (ascending contact index)
template <class R>
__global__ void kReduceManifolds(Dev<R> d, int nm, int nc, int bits, const int* segStart, const u64* keys,
                                 const int* perm) {
  const u64 none = (1ull << bits) - 1ull;
  GRID_STRIDE(m, nm) {
    const int b = segStart[m], e = (m + 1 < nm) ? segStart[m + 1] : nc;
    const u64 k = keys[b];
    const int A = (int)(k >> bits);
    const u64 v = k & none;
    const int B = (v == none) ? -1 : (int)v;
    int npts = 0;
    V3<R> N{0, 0, 0}, TA{0, 0, 0}, TB{0, 0, 0}, rA{0, 0, 0}, rB{0, 0, 0}, wv{0, 0, 0};
    R es = 0, mus = 0;
    for (int p = b; p < e; ++p) {
      const int c = perm[p];
      d.cSlot[c] = (int)m;
      const Q4<R> cn = d.cn[c];
      const R dist = cn.w;
      if (dist > R(0))
        continue;  // inactive contact: contributes an all-zero manifold (x + 0 = x)
      const int2 ab = d.cab[c];
      const bool flip = (ab.y >= 0 && ab.y < ab.x);
      const V3<R> n = v3(cn);
      const V3<R> na = flip ? n : neg(n);
      const V3<R> sh{n.x * dist * R(0.5), n.y * dist * R(0.5), n.z * dist * R(0.5)};
      const Q4<R> crA = d.crA[c], crB = d.crB[c], cbv = d.cbv[c];
      const V3<R> ra = sub(v3(crA), sh);
      const V3<R> rb = add(v3(crB), sh);
      const V3<R> rc = flip ? rb : ra, ro = flip ? ra : rb;
      npts += 1;
      N = add(N, na);
      TA = add(TA, cross(rc, na));
      TB = add(TB, cross(ro, neg(na)));
      rA = add(rA, rc);
      rB = add(rB, ro);
      wv = add(wv, v3(cbv));
      es += crB.w;
      mus += cbv.w;
    }
    d.mab[m] = make_int2(A, B);
    d.mnp[m] = npts;
    d.mN[m] = q4(N, es);
    d.mTA[m] = q4(TA, mus);
    d.mTB[m] = q4(TB);
    d.mrA[m] = q4(rA);
    d.mrB[m] = q4(rB);
    d.mwv[m] = q4(wv);
  }
}

// =============================================================================================
// warm-start ledger (src/contact_preprocessing.hpp:70-192,501-538)
// =============================================================================================
__device__ __forceinline__ int lowerBound(const u64* keys, int n, u64 k) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}
template <class R>
__device__ __forceinline__ u64 realPairKey(const Dev<R>& d, int2 ab) {
  const unsigned a = (unsigned)d.realIdx[ab.x];
  const unsigned b = ab.y >= 0 ? (unsigned)d.realIdx[ab.y] : 0xFFFFFFFFu;
  const unsigned hi = a < b ? a : b, lo = a < b ? b : a;
  return ((u64)hi << 32) | lo;
}
// gatherWarmLambda (:113-156) followed by markPersistentManifolds (:78-108): the second writes the
// keys, so periodic-duplicate manifolds keep their real key but a zero warm start
template <class R>
__global__ void kGatherWarm(Dev<R> d, int nm, int prevCount) {
  GRID_STRIDE(i, nm) {
    const int2 ab = d.mab[i];
    const int npts = d.mnp[i];
    if (npts <= 0) {
      d.pairKeys[i] = ~0ull;
      d.persistent[i] = 0;
      d.lambda[i] = R(0);
      d.lambdaT[i] = Q4<R>{0, 0, 0, 0};
      d.posImp[i] = R(0);
      continue;
    }
    const u64 k = realPairKey(d, ab);
    const int lo = lowerBound(d.prevKeys, prevCount, k);
    const bool hit = lo < prevCount && d.prevKeys[lo] == k;
    const bool dup = ab.y >= 0 && d.realIdx[ab.x] > d.realIdx[ab.y];
    d.pairKeys[i] = k;
    d.persistent[i] = hit ? 1 : 0;
    const bool warm = hit && !dup;
    d.lambda[i] = warm ? d.prevLambda[lo] : R(0);
    d.lambdaT[i] = warm ? d.prevLambdaT[lo] : Q4<R>{0, 0, 0, 0};
    d.posImp[i] = warm ? d.prevPosImp[lo] : R(0);
  }
}
// ledger sort keys: the 64-bit pair key (u << 32 | v, v = 0xFFFFFFFF for a boundary, all ones for
// an empty manifold) packed order-preservingly into 2 * bits bits, with the manifold index as value
__global__ void kLedgerKeys(int nm, int bits, const u64* pairKeys, u64* packed, int* vals) {
  const u64 none = (1ull << bits) - 1ull;
  GRID_STRIDE(i, nm) {
    const u64 k = pairKeys[i];
    const u64 u = k >> 32, v = k & 0xFFFFFFFFull;
    packed[i] = ((u == 0xFFFFFFFFull ? none : u) << bits) | (v == 0xFFFFFFFFull ? none : v);
    vals[i] = (int)i;
  }
}
// The ledger's stable key sort when no body has a ghost image: a manifold's real key is then its
// own body-pair key, and the manifold list is in that key order (it is the contact list's key
// order, boundary key (i, none) after the pairs of i). Empty manifolds carry the all-ones key and
// sort last in list order. So the sorted order is the non-empty manifolds, then the empty ones,
// each in list order: flags -> exclusive scan (pos) -> this scatter.
__global__ void kLedgerFlags(int nm, const u64* pairKeys, int* flag) {
  GRID_STRIDE(i, nm) flag[i] = pairKeys[i] != ~0ull ? 1 : 0;
}
__global__ void kLedgerRanks(int nm, int bits, const u64* pairKeys, const int* flag, const int* pos, u64* keysOut,
                             int* permOut) {
  const u64 none = (1ull << bits) - 1ull;
  const int live = pos[nm];
  GRID_STRIDE(i, nm) {
    const u64 k = pairKeys[i];
    const u64 u = k >> 32, v = k & 0xFFFFFFFFull;
    const int r = flag[i] ? pos[i] : live + (int)i - pos[i];
    keysOut[r] = ((u == 0xFFFFFFFFull ? none : u) << bits) | (v == 0xFFFFFFFFull ? none : v);
    permOut[r] = (int)i;
  }
}
// The ledger's stable key sort with ghost images present. Three kinds of manifold:
// - in order: live, second body not a ghost. The real key equals the list key, so these come in
//   key order (unique keys);
// - ghost: live, second body a ghost image. These are compacted in list order and sorted alone;
// - empty: the all-ones key, last, in list order.
// Ranks: an in-order manifold m -> rpos[m] + the ghost entries before (key, m); the ghost entry at
// sorted place q -> q + the in-order manifolds before (key, index), i.e. rpos[L] for L = the lower
// bound of the key among the list keys, plus the one with the same key if its index is smaller; an
// empty manifold -> all live ones + its place among the empty ones (m - rpos[m] - gpos[m]).
__device__ __forceinline__ u64 ledgerPack(u64 k, int bits) {
  const u64 none = (1ull << bits) - 1ull;
  const u64 u = k >> 32, v = k & 0xFFFFFFFFull;
  return ((u == 0xFFFFFFFFull ? none : u) << bits) | (v == 0xFFFFFFFFull ? none : v);
}
template <class R>
__global__ void kLedgerClass(Dev<R> d, int nm, int bits, int numReal, const u64* pairKeys, u64* keys, int* inOrder,
                             int* ghost) {
  GRID_STRIDE(m, nm) {
    const u64 k = pairKeys[m];
    keys[m] = ledgerPack(k, bits);
    const bool live = k != ~0ull, g = d.mab[m].y >= numReal;  // a boundary's second body is -1
    inOrder[m] = (live && !g) ? 1 : 0;
    ghost[m] = (live && g) ? 1 : 0;
  }
}
__global__ void kLedgerApart(int nm, const u64* keys, const int* ghost, const int* gpos, u64* oKeys, int* oIdx) {
  GRID_STRIDE(m, nm) {
    if (ghost[m]) {
      oKeys[gpos[m]] = keys[m];
      oIdx[gpos[m]] = (int)m;
    }
  }
}
template <class R>
__global__ void kLedgerMerge(Dev<R> d, int nm, int nG, int bits, const u64* keys, const int* inOrder, const int* rpos,
                             const int* ghost, const int* gpos, const u64* gKeys, const int* gIdx, u64* keysOut,
                             int* permOut) {
  const u64 none = (1ull << bits) - 1ull;
  const int live = rpos[nm] + gpos[nm];
  GRID_STRIDE(t, (long)nm + nG) {
    u64 k;
    int r, idx;
    if (t < nm) {
      idx = (int)t;
      if (ghost[idx])
        continue;  // placed by its sorted entry
      k = keys[idx];
      if (!inOrder[idx]) {
        r = live + idx - rpos[idx] - gpos[idx];
      } else {
        int lo = 0, hi = nG;  // ghost entries before (k, idx)
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (gKeys[mid] < k || (gKeys[mid] == k && gIdx[mid] < idx))
            lo = mid + 1;
          else
            hi = mid;
        }
        r = rpos[idx] + lo;
      }
    } else {
      const int q = (int)(t - nm);
      k = gKeys[q];
      idx = gIdx[q];
      int lo = 0, hi = nm;  // list keys below k
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const int2 ab = d.mab[mid];
        const u64 raw = ((u64)(unsigned)ab.x << bits) | (ab.y >= 0 ? (u64)(unsigned)ab.y : none);
        if (raw < k)
          lo = mid + 1;
        else
          hi = mid;
      }
      r = q + rpos[lo] + ((lo < nm && inOrder[lo] && keys[lo] == k && lo < idx) ? 1 : 0);
    }
    keysOut[r] = k;
    permOut[r] = idx;
  }
}

// commitPairKeysLambda (:160-192): keys/perm already stably sorted by key
template <class R>
__global__ void kCommitLedger(Dev<R> d, int nm, const int* perm) {
  GRID_STRIDE(i, nm) {
    const int j = perm[i];
    d.prevKeys[i] = d.pairKeys[j];
    d.prevLambda[i] = d.lambda[j];
    d.prevLambdaT[i] = d.lambdaT[j];
  }
}
// commitPosImpulse (:501-538). Per manifold: sum of l/dt over its contacts in ascending contact
// index (the reference's scatter order); then the ledger slot of each key receives the value of the
// LAST manifold (highest index) carrying that key, as the serial scatter leaves it.
template <class R>
__global__ void kPosLoad(Dev<R> d, int nm, int nc, const int* segStart, const int* cperm, R dt, R* scratch) {
  GRID_STRIDE(m, nm) {
    const int b = segStart[m], e = (m + 1 < nm) ? segStart[m + 1] : nc;
    R acc = R(0);
    for (int p = b; p < e; ++p) {
      const R l = d.posLamC[cperm[p]];
      if (l != R(0))
        acc += l / dt;
    }
    scratch[m] = acc;
  }
}
template <class R>
__global__ void kPosLoadScatter(Dev<R> d, int nm, const int* perm, const R* scratch) {
  GRID_STRIDE(s, nm) {
    const u64 k = d.prevKeys[s];
    if (k == ~0ull)
      continue;
    if (s > 0 && d.prevKeys[s - 1] == k)
      continue;  // not the first of its key group
    int e = (int)s;
    while (e + 1 < nm && d.prevKeys[e + 1] == k)
      ++e;
    d.prevPosImp[s] = scratch[perm[e]];
  }
}

// =============================================================================================
// support levels (src/contact_preprocessing.hpp:213-253)
// =============================================================================================
template <class R>
__global__ void kGroundDecay(Dev<R> d, int n, int decay) {
  GRID_STRIDE(i, n) {
    const int g = (int)d.grounded[i] - decay;
    d.grounded[i] = (uint8_t)(g > 0 ? g : 0);
  }
}
// Edge of the support graph: kind 0 = none, 1 = wall (dst := 255), 2 = src supports dst.
// Directions depend only on positions, fixed for the substep's sweeps.
template <class R>
__global__ void kGroundEdges(Dev<R> d, int nm, V3<R> gHat, int4* edges) {
  GRID_STRIDE(i, nm) {
    int4 e = make_int4(0, 0, 0, 0);
    if (d.mnp[i] > 0) {
      const int2 ab = d.mab[i];
      const int ra = d.realIdx[ab.x];
      if (ab.y < 0) {
        e = make_int4(1, ra, ra, 0);
      } else {
        const int rb = d.realIdx[ab.y];
        const V3<R> dx = sub(v3(d.posPred[ab.x]), v3(d.posPred[ab.y]));
        const R up = -(dx.x * gHat.x + dx.y * gHat.y + dx.z * gHat.z);
        const R thr = R(0.3) * sqrt(dot(dx, dx));
        if (up > thr)
          e = make_int4(2, rb, ra, 0);
        else if (up < -thr)
          e = make_int4(2, ra, rb, 0);
      }
    }
    edges[i] = e;
  }
}
// Serial in-order sweeps (the reference's serial sweep reads levels updated earlier in the same
// sweep). One warp walks the edges in windows of 32 (edges prefetched several windows ahead):
//  fast path: every lane pushes (level_before_window[src] - 1) with an order-free max; if no
//             source level changed inside the window, that is exactly the sequential result;
//  exact path: otherwise each lane's source level is recomputed from the pre-window level and the
//             pushes of EARLIER lanes whose destination is that source (fixed point over the
//             window; those lanes are found once per window from the destinations in shared
//             memory), and the exact pushes are applied. Fast-path pushes never exceed the exact
//             ones (levels only grow), so applying both gives the sequential result.
// A sweep that changes nothing ends the loop (later sweeps would repeat it unchanged).
// Levels live in shared memory when they fit, else in a global scratch array.
constexpr int kGroundPF = 8;
// one warp: the sweeps over edges[0, nm) whose bodies are [b0, b0 + nb) with levels in L[i - b0]
__device__ __forceinline__ void groundSweepsWarp(int nm, int b0, int nb, int sweeps, const int4* edges,
                                                 uint8_t* grounded, int* L) {
  const int lane = threadIdx.x & 31;
  __shared__ int sDst[32], sPush[32];  // one warp per block: the window's destinations and pushes
  for (int i = lane; i < nb; i += 32)
    L[i] = grounded[b0 + i];
  __threadfence_block();
  __syncwarp();
  const int nwin = (nm + 31) / 32;
  for (int s = 0; s < sweeps; ++s) {
    int sweepChanged = 0;
    for (int w0 = 0; w0 < nwin; w0 += kGroundPF) {
      int4 buf[kGroundPF];
#pragma unroll
      for (int q = 0; q < kGroundPF; ++q) {
        const int ei = (w0 + q) * 32 + lane;
        buf[q] = (ei < nm) ? edges[ei] : make_int4(0, 0, 0, 0);
      }
#pragma unroll
      for (int q = 0; q < kGroundPF; ++q) {
        if (w0 + q >= nwin)
          break;
        const int kind = buf[q].x, src = buf[q].y - b0, dst = buf[q].z - b0;
        const int L0s = (kind == 2) ? L[src] : 0;
        const int L0d = (kind != 0) ? L[dst] : 0;
        int c = (kind == 1) ? 255 : (kind == 2 ? L0s - 1 : 0);
        bool contrib = (kind == 1) || (kind == 2 && c > 0);
        __syncwarp();
        if (contrib && c > L0d)
          atomicMax(&L[dst], c);
        __threadfence_block();
        __syncwarp();
        const bool srcMoved = (kind == 2) && L[src] != L0s;
        const bool dstMoved = (kind != 0) && L[dst] != L0d;
        if (__any_sync(0xffffffffu, dstMoved))
          sweepChanged = 1;
        if (__any_sync(0xffffffffu, srcMoved)) {
          // earlier lanes of the window that push to this lane's source: one scan of the window's
          // destinations, then fixed-point rounds that read only those lanes' pushes
          sDst[lane] = (kind != 0) ? dst : -1;
          __syncwarp();
          unsigned from = 0;
#pragma unroll
          for (int t = 0; t < 32; ++t)
            if (t < lane && kind == 2 && sDst[t] == src)
              from |= 1u << t;
          for (int it = 0; it < 33; ++it) {
            sPush[lane] = contrib ? c : -1;
            __syncwarp();
            int best = L0s;
            for (unsigned m = from; m; m &= m - 1) {
              const int cT = sPush[__ffs(m) - 1];
              if (cT > best)
                best = cT;
            }
            const int nc = (kind == 2) ? best - 1 : c;
            const bool ch = nc != c;
            c = nc;
            contrib = (kind == 1) || (kind == 2 && c > 0);
            __syncwarp();  // this round's reads of the pushes come before the next round's writes
            if (!__any_sync(0xffffffffu, ch))
              break;
          }
          if (contrib)
            atomicMax(&L[dst], c);
          __threadfence_block();
          __syncwarp();
        }
      }
    }
    if (!__any_sync(0xffffffffu, sweepChanged))
      break;
  }
  __syncwarp();
  for (int i = lane; i < nb; i += 32)
    grounded[b0 + i] = (uint8_t)L[i];
}
__global__ void kGroundSweeps(int nm, int numReal, int sweeps, const int4* edges, uint8_t* grounded,
                              int* gscratch, int useShared) {
  extern __shared__ int slvl[];
  groundSweepsWarp(nm, 0, numReal, sweeps, edges, grounded, useShared ? slvl : gscratch);
}
// The same support levels from the least fixed point, in parallel. The serial sweeps only raise
// levels, each raise is an edge relaxation (wall: 255; support: the source's level - 1 when
// positive), so they climb towards the least fixed point F above the decayed levels L0, the same
// whatever the order of relaxations; when they reach F within `sweeps` sweeps, their result is F.
// One block (a) computes F by parallel relaxation passes, (b) finds, for every body, the sweep in
// which the serial order first gives it F: a body at L0 = F before sweep 1; otherwise the earliest
// (sweep, edge) over the edges that deliver F, where a support edge e from u delivers in u's sweep
// if e comes after the edge that finished u, else in the next sweep (a shortest-path relaxation on
// that acyclic edge set: F drops by one along it). (c) If every body is final within `sweeps`
// sweeps the levels are F; otherwise warp 0 runs the exact serial sweeps from L0 (still in
// `grounded`). Shared memory: the times (8 bytes a body), the edges (8 bytes each: kind in the top
// bits of the source, then the destination) and the levels (4 bytes a body).
constexpr int kGroundBlock = 1024;
constexpr int kGroundPassCap = 4096;  // relaxation passes before the exact serial sweeps take over
__global__ void __launch_bounds__(kGroundBlock) kGroundLevels(int nm, int nb, int sweeps, const int4* edges,
                                                              uint8_t* grounded) {
  extern __shared__ __align__(16) unsigned char gsm[];
  using ull = unsigned long long;
  ull* T = reinterpret_cast<ull*>(gsm);
  int2* E = reinterpret_cast<int2*>(T + nb);
  int* L = reinterpret_cast<int*>(E + nm);
  volatile int* VL = L;
  volatile ull* VT = T;
  const int tid = threadIdx.x;
  for (int i = tid; i < nb; i += blockDim.x)
    L[i] = grounded[i];
  for (int e = tid; e < nm; e += blockDim.x) {
    const int4 g = edges[e];
    E[e] = make_int2((int)(((unsigned)g.x << 30) | (unsigned)g.y), g.z);
  }
  __syncthreads();
  // every thread walks a contiguous run of edges in index order
  const int per = (nm + (int)blockDim.x - 1) / (int)blockDim.x;
  const int e0 = min(nm, tid * per), e1 = min(nm, e0 + per);
  bool fast = true;
  for (int pass = 0;; ++pass) {  // (a) F
    int ch = 0;
    for (int e = e0; e < e1; ++e) {
      const int2 g = E[e];
      const int kind = (int)((unsigned)g.x >> 30), src = g.x & 0x3fffffff, dst = g.y;
      const int c = kind == 1 ? 255 : (kind == 2 ? VL[src] - 1 : 0);
      if (c > 0 && c > VL[dst]) {
        atomicMax(&L[dst], c);
        ch = 1;
      }
    }
    if (!__syncthreads_or(ch))
      break;
    if (pass + 1 >= kGroundPassCap) {
      fast = false;
      break;
    }
  }
  const ull kInf = ~0ull, kStart = 1ull << 32;  // (sweep << 32) | (edge + 1); 1 << 32: final before sweep 1
  for (int i = tid; i < nb; i += blockDim.x)
    T[i] = L[i] == (int)grounded[i] ? kStart : kInf;
  __syncthreads();
  for (int pass = 0; fast; ++pass) {  // (b) the sweep in which each body becomes final
    int ch = 0;
    for (int e = e0; e < e1; ++e) {
      const int2 g = E[e];
      const int kind = (int)((unsigned)g.x >> 30), src = g.x & 0x3fffffff, dst = g.y;
      ull te = kInf;
      if (kind == 1 && VL[dst] == 255) {
        te = kStart | (ull)(e + 1);
      } else if (kind == 2 && VL[dst] > 0 && VL[src] - 1 == VL[dst]) {
        const ull tu = VT[src];
        if (tu != kInf) {
          const ull ku = tu >> 32;
          const long iu = (long)(tu & 0xffffffffull) - 1;
          te = (((long)e > iu ? ku : ku + 1) << 32) | (ull)(e + 1);
        }
      }
      if (te < VT[dst]) {
        atomicMin(&T[dst], te);
        ch = 1;
      }
    }
    if (!__syncthreads_or(ch))
      break;
    if (pass + 1 >= kGroundPassCap)
      fast = false;
  }
  int late = !fast;
  for (int i = tid; i < nb && !late; i += blockDim.x)
    late = T[i] == kInf || (T[i] >> 32) > (ull)sweeps;
  late = __syncthreads_or(late);
  if (!late) {  // (c)
    for (int i = tid; i < nb; i += blockDim.x)
      grounded[i] = (uint8_t)L[i];
    return;
  }
  if (tid < 32)
    groundSweepsWarp(nm, 0, nb, sweeps, edges, grounded, L);
}
// batched form: one warp (block) per scene over its own edge range manFirst[s..s+1) and bodies
// bodyFirst[s..s+1): the sweeps of independent scenes are independent, and each stops on its own
__global__ void kGroundSweepsScenes(const int* manFirst, const int* bodyFirst, int sweeps, const int4* edges,
                                    uint8_t* grounded, int* gscratch, int useShared) {
  extern __shared__ int slvl[];
  const int s = blockIdx.x;
  const int b0 = bodyFirst[s], nb = bodyFirst[s + 1] - b0;
  const int e0 = manFirst[s], ne = manFirst[s + 1] - e0;
  groundSweepsWarp(ne, b0, nb, sweeps, edges + e0, grounded, useShared ? slvl : gscratch + b0);
}

// =============================================================================================
// Jones-Plassmann colouring (src/solver_velocity.hpp:277-374, src/solver_position.hpp:155-241)
// =============================================================================================
// ends of edge i: manifolds use real body indices, contacts raw slots
template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorEnds(const Dev<R>& d, int i, int& ea, int& eb) {
  if (MANIFOLD) {
    const int2 ab = d.mab[i];
    ea = d.realIdx[ab.x];
    eb = ab.y >= 0 ? d.realIdx[ab.y] : -1;
  } else {
    const int2 ab = d.cab[i];
    ea = ab.x;
    eb = ab.y;
  }
}
// colour priority of entry i with first body ea: the key of its scene-local index (batched form)
template <class R, bool MANIFOLD>
__device__ __forceinline__ long long entryKey(const Dev<R>& d, int i, int ea) {
  if (!d.sceneOf)
    return colorKey(i);
  const int s = d.sceneOf[ea];
  return colorKey(MANIFOLD ? localManifold(d, i, s) : localContact(d, i, s));
}
// Topology reuse. The colourings, colour orders, manifold grouping, incidence lists and ledger
// order are functions of the contact list's body pairs (and, for the manifold side, of each
// manifold's real ends and whether it is active). When those equal the previous substep's, the
// products of that substep are still exact and are kept. These kernels compare and record.
__global__ void kSameInt2(const int2* cur, int2* prev, int n, int* differ) {
  GRID_STRIDE(i, n) {
    const int2 a = cur[i], b = prev[i];
    if (a.x != b.x || a.y != b.y)
      *differ = 1;
    prev[i] = a;
  }
}
template <class R>
__global__ void kSameManifolds(Dev<R> d, int nm, int4* prev, int* differ) {
  GRID_STRIDE(i, nm) {
    const int2 ab = d.mab[i];
    const int ra = d.realIdx[ab.x], rb = ab.y >= 0 ? d.realIdx[ab.y] : -1;
    const int init = (d.mnp[i] <= 0 || (ab.y >= 0 && ra > rb)) ? -2 : -1;
    const int4 sig = make_int4(ra, rb, init, 0), old = prev[i];
    if (sig.x != old.x || sig.y != old.y || sig.z != old.z)
      *differ = 1;
    prev[i] = sig;
  }
}
// colour keys for the stable colour-sorted execution order
// batched form: the (scene, colour) order in one launch, one block per scene. A scene's entries are
// the concatenation, in index order, of its slice of each of nr body-sorted ranges (firsts: nr
// arrays of S + 1 first entries; manifolds: one range; contacts: pairs, planes, walls), so the
// stable sort by (scene, colour) is, per scene, a stable counting sort by colour placed after the
// entries of the scenes before it. off[s * 64 + c] is the first position of (s, c); off[S * 64] = ne.
__global__ void __launch_bounds__(256) kColorOrderScenes(const int* col, const int* firsts, int nr, int S, int ne,
                                                         int* order, int* off) {
  __shared__ int run[64];
  __shared__ int cnt[8][64];
  const int s = blockIdx.x;
  int lo[3] = {0, 0, 0}, len[3] = {0, 0, 0}, base = 0, total = 0;
  for (int r = 0; r < nr; ++r) {
    const int* f = firsts + (long)r * (S + 1);
    lo[r] = f[s];
    len[r] = f[s + 1] - f[s];
    base += f[s] - f[0];
    total += len[r];
  }
  auto entry = [&](int v) { return v < len[0] ? lo[0] + v : v < len[0] + len[1] ? lo[1] + v - len[0] : lo[2] + v - len[0] - len[1]; };
  if (threadIdx.x < 64)
    run[threadIdx.x] = 0;
  __syncthreads();
  for (int v = threadIdx.x; v < total; v += blockDim.x) {
    const int c = col[entry(v)];
    atomicAdd(&run[c >= 0 ? c : 63], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // counts -> first positions
    int acc = base;
    for (int c = 0; c < 64; ++c) {
      const int n = run[c];
      run[c] = acc;
      off[(long)s * 64 + c] = acc;
      acc += n;
    }
    if (s == 0)
      off[(long)S * 64] = ne;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (int t0 = 0; t0 < total; t0 += blockDim.x) {
    for (int k = threadIdx.x; k < nw * 64; k += blockDim.x)
      (&cnt[0][0])[k] = 0;
    __syncthreads();
    const int v = t0 + (int)threadIdx.x;
    const int i = v < total ? entry(v) : -1;
    const int key = i >= 0 ? (col[i] >= 0 ? col[i] : 63) : 64;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int below = __popc(peers & ((1u << lane) - 1u));
    if (key < 64 && below == 0)
      cnt[w][key] = __popc(peers);
    __syncthreads();
    if (key < 64) {
      int pos = run[key] + below;
      for (int u = 0; u < w; ++u)
        pos += cnt[u][key];
      order[pos] = i;
    }
    __syncthreads();
    if (threadIdx.x < 64) {
      int tot = 0;
      for (int u = 0; u < nw; ++u)
        tot += cnt[u][threadIdx.x];
      run[threadIdx.x] += tot;
    }
    __syncthreads();
  }
}
}  // namespace pdem
