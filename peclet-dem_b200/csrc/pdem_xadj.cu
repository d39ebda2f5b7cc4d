// Adjoint of the XPBD substep on the B200 (plain FP64 path, spheres and planes).
//
// Forward (xadjStep): each substep runs the production step (Sim<double>::step) unchanged; around
// it the record keeps what the reverse pass needs and cannot recompute cheaply:
//   - the start state (x, q, v, w) and the warm-start ledger the step reads (keys, lambda,
//     lambda_T, position impulse), i.e. a checkpoint of the compact state every substep;
//   - the frozen discrete decisions: the contact list (body pairs, plane of each wall contact,
//     manifold slot), the manifold list, both colourings (colour-ordered lists and offsets), the
//     side flags of the stabilization pass and the sweep counts of the three adaptive loops.
// Reverse (xadjBackward), substep by substep from the last:
//   1. replay: the substep recomputed from its checkpoint with the local maps of pdem_xadj.cuh
//      (the forward's expressions), colour by colour over the frozen colouring, storing the
//      input of every sweep update (the tape: velocity, impulses per manifold and sweep, the two
//      positions per contact and sweep) — the intermediates are recomputed, not stored, between
//      checkpoints;
//   2. reverse: position sweeps, velocity commit, stabilization and main PGS sweeps in reverse
//      colour and sweep order (within a colour the updates touch disjoint bodies, as in the
//      forward), then warm start, approach velocities, the ledger gather, the manifold sums, the
//      contact geometry and the velocity prediction; each update's vector-Jacobian product comes
//      from its local map in forward-mode chunks;
//   3. the adjoint of the ledger the substep read is handed to the previous substep's manifolds
//      by pair key (the keys are sorted, as the ledger's).
// The friction and restitution branches, the impulse clamps and the active position contacts are
// those the replay takes, which are the forward's (same expressions on the same values); the
// contact set, colours and sweep counts are the forward's. Gradients: start positions,
// orientations, velocities, angular velocities and (eN, eT, mu). Young's modulus does not enter
// the XPBD step (it has no stiffness); its gradient is defined on the Hertz path.
//
// Scope (refused with std::invalid_argument otherwise): FP64, one scene, sphere shapes without
// point shells, isotropic inverse inertia, planes as the only walls, gravity on and coloured
// Gauss-Seidel (the PGS path), stabilization off, one-sided or escalate, no periodicity, growth,
// thermostat or pair materials, every entry coloured (no Jacobi leftovers) and no saturated
// colour.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <vector>

#include <cooperative_groups.h>

#include "pdem_sim.cuh"
#include "pdem_xadj.cuh"
#include "pdem_xadj_api.cuh"

namespace pdem {

using namespace xadj;
using D4 = Q4<double>;
namespace cg = cooperative_groups;

namespace {

constexpr int kB = 256;
constexpr int kBR = 128;   // the reverse kernels (up to 255 registers a thread)
constexpr int kBPgs = 64;  // the hand-written PGS reverse: one entry a thread, few entries a colour
// the persistent sweep loops: one cluster of kClusterBlocks blocks (the non-portable size 16),
// for manifold lists up to kClusterEntries (larger ones sweep colour by colour in separate launches)
constexpr int kClusterBlocks = 16;
constexpr int kClusterEntries = 1 << 16;
constexpr int kMaxColours = 62;  // the first saturated colour of the 62-colour masks

__device__ __forceinline__ u64 manKey(int2 ab) {
  if (ab.y < 0)
    return ((u64)(unsigned)ab.x << 32) | 0xFFFFFFFFull;
  const unsigned u = ab.x < ab.y ? ab.x : ab.y, v = ab.x < ab.y ? ab.y : ab.x;
  return ((u64)u << 32) | v;
}
__device__ __forceinline__ int lowerBoundKeys(const u64* keys, int n, u64 k) {
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
// position of key k among the manifold keys of a manifold list (ascending), or -1
__device__ __forceinline__ int findManifold(const int2* mab, int nm, u64 k) {
  int lo = 0, hi = nm;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (manKey(mab[mid]) < k)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < nm && manKey(mab[lo]) == k) ? lo : -1;
}
__device__ __forceinline__ void atomicAdd3(D4* p, const double* v) {
  atomicAdd(&p->x, v[0]);
  atomicAdd(&p->y, v[1]);
  atomicAdd(&p->z, v[2]);
}
__device__ __forceinline__ void atomicAdd4(D4* p, const double* v) {
  atomicAdd3(p, v);
  atomicAdd(&p->w, v[3]);
}
__device__ __forceinline__ void put3(double* a, int o, D4 v) {
  a[o] = v.x, a[o + 1] = v.y, a[o + 2] = v.z;
}
__device__ __forceinline__ void put4(double* a, int o, D4 v) {
  a[o] = v.x, a[o + 1] = v.y, a[o + 2] = v.z, a[o + 3] = v.w;
}
__device__ __forceinline__ D4 get3(const double* a, int o, double w = 0.0) {
  return D4{a[o], a[o + 1], a[o + 2], w};
}
__device__ __forceinline__ D4 get4(const double* a, int o) {
  return D4{a[o], a[o + 1], a[o + 2], a[o + 3]};
}
__device__ __forceinline__ void add3(D4& p, const double* v) {
  p.x += v[0], p.y += v[1], p.z += v[2];
}
__device__ __forceinline__ void add4(D4& p, const double* v) {
  p.x += v[0], p.y += v[1], p.z += v[2], p.w += v[3];
}
__device__ __forceinline__ V3<double> v3d(D4 a) {
  return V3<double>{a.x, a.y, a.z};
}

// constants of the scene (one per rollout)
struct XScene {
  int n;
  double dt, gs, par, eps, eN, eT, mu;
  V3<double> g;
  const double* invMass;
  const D4* invI;
  const double* scale;
  const D4* extF;
  const PlaneDesc<double>* planes;
};

// one recorded substep, device side
struct XView {
  int nc, nm, L, ncolV, ncolP;
  const int2* cab;
  const int* cSlot;
  const int* cOrder;
  const int* cOff;
  const int* cPlane;
  const int2* mab;
  const int* mOrder;
  const int* mOff;
  const int* mC0;
  const int* mCn;
  const uint8_t* sf;
  const D4* st;  // x [0, n), q [n, 2n), v [2n, 3n), w [3n, 4n)
  const u64* lkeys;
  const D4* lval;  // lambda_T | lambda
  const double* lpos;
};

// the reverse workspace
struct XWork {
  // bodies
  D4 *vP0, *wP0, *xP0, *vP, *wP, *vF, *wF, *xP, *qP;
  D4 *gx, *gq, *gv, *gw;          // adjoint of the substep's end state
  D4 *ax, *aq, *av, *aw;          // adjoint of its start state
  D4 *axP, *aqP, *avP, *awP, *axP0;
  // contacts
  D4 *cgN, *cgA, *cgB;            // n | dist, rA, rB
  D4 *acgN, *acgA, *acgB;
  double *posLam, *aposLam;
  // manifolds
  D4* geo;                        // [5 nm]: N, TA, TB, rA, rB (sums)
  D4* ageo;
  int *np, *src;
  D4 *lam0, *lam, *vn;            // lambda_T | lambda; vt0 | vn0
  D4 *alam, *avn, *ath;
  double *posIn, *aposIn;
  D4* alamOut;                    // adjoint of the substep's final lambda_T | lambda
  double* aposOut;                // adjoint of its position impulse (the next substep's ledger)
  D4* alamPrev;                   // the same for the previous substep (filled by the ledger map)
  double* aposPrev;
  D4* alL;                        // adjoint of the ledger the substep read
  double* apL;
  // tapes
  D4* tv;                         // [sweeps][nm][4]: vA | p, wA | lt.x, vB | lt.y, wB | lt.z
  D4* tp;                         // [sweeps][nc][2]: xA, xB
  double* theta;                  // [3] d/d(eN, eT, mu)
  double* err;                    // [2] replay deviation from the recorded next state (max)
  u64* hash;                      // branch signature of the replays (null: not collected)
};

// order-free branch signature: a sum over the sweep updates of a mixed (substep, sweep, entry,
// branch bits) word (splitmix64 finaliser), summed per warp before one atomic
__device__ __forceinline__ u64 mixWord(u64 x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__device__ __forceinline__ void warpHashAdd(u64* h, u64 v) {
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v)
    atomicAdd(reinterpret_cast<unsigned long long*>(h), (unsigned long long)v);
}

__device__ __forceinline__ void atomicMaxPos(double* p, double v) {
  if (v > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}

// ---------------- replay ----------------
__global__ void kxPredict(XScene sc, XView r, XWork w) {
  GRID_STRIDE(i, sc.n) {
    double in[kPredIn], out[kPredOut];
    put3(in, 0, r.st[i]);
    put4(in, 3, r.st[sc.n + i]);
    put3(in, 7, r.st[2 * sc.n + i]);
    put3(in, 10, r.st[3 * sc.n + i]);
    const BodyC b{sc.invMass[i], v3d(sc.invI[i])};
    const StepC s{sc.dt, sc.g, 0.0, sc.eps};
    predictMap<double>(in, out, b, s, v3d(sc.extF[i]));
    w.vP0[i] = w.vP[i] = get3(out, 0);
    w.wP0[i] = w.wP[i] = get3(out, 3);
    w.xP0[i] = get3(out, 6);
  }
}

__device__ __forceinline__ ConC conC(const XScene& sc, int a, int b) {
  return ConC{sc.scale[a] * sc.gs, sc.scale[b] * sc.gs, sc.par, sc.par, sc.eps};
}
__device__ __forceinline__ double planeRadius(const XScene& sc, int a) {
  const double bR = sc.par == 0.0 ? 1.0 : sc.par;
  return bR * (sc.scale[a] * sc.gs);
}

__global__ void kxContacts(XScene sc, XView r, XWork w) {
  GRID_STRIDE(k, r.nc) {
    const int2 ab = r.cab[k];
    if (ab.y >= 0) {
      double in[kConIn], out[kConOut];
      put3(in, 0, w.xP0[ab.x]);
      put4(in, 3, r.st[sc.n + ab.x]);
      put3(in, 7, w.xP0[ab.y]);
      put4(in, 10, r.st[sc.n + ab.y]);
      contactMap<double>(in, out, conC(sc, ab.x, ab.y));
      w.cgN[k] = get3(out, 0, out[9]);
      w.cgA[k] = get3(out, 3);
      w.cgB[k] = get3(out, 6);
    } else {
      const PlaneDesc<double> pl = sc.planes[r.cPlane[k]];
      const V3<double> n{pl.n[0], pl.n[1], pl.n[2]}, p{pl.p[0], pl.p[1], pl.p[2]};
      const double radius = planeRadius(sc, ab.x);
      const double dist = dot(sub(v3d(w.xP0[ab.x]), p), n) - radius;
      w.cgN[k] = D4{n.x, n.y, n.z, dist};
      w.cgA[k] = q4(mul(n, -radius));
      w.cgB[k] = q4(p);
    }
  }
}

__device__ __forceinline__ void conIn(const XWork& w, int k, double* in) {
  put3(in, 0, w.cgN[k]);
  put3(in, 3, w.cgA[k]);
  put3(in, 6, w.cgB[k]);
  in[9] = w.cgN[k].w;
}

__global__ void kxManifolds(XScene sc, XView r, XWork w) {
  GRID_STRIDE(m, r.nm) {
    double sum[kManOut];
    for (int j = 0; j < kManOut; ++j)
      sum[j] = 0.0;
    int np = 0;
    const int c0 = r.mC0[m], cn = r.mCn[m];
    for (int k = c0; k < c0 + cn; ++k) {
      if (!(w.cgN[k].w <= 0.0))
        continue;
      const int2 ab = r.cab[k];
      double in[kManIn], out[kManOut];
      conIn(w, k, in);
      manifoldMap<double>(in, out, ab.y >= 0 && ab.y < ab.x);
      for (int j = 0; j < kManOut; ++j)
        sum[j] = sum[j] + out[j];
      ++np;
    }
    for (int j = 0; j < 5; ++j)
      w.geo[5 * m + j] = get3(sum, 3 * j);
    w.np[m] = np;
  }
}

__global__ void kxGather(XScene sc, XView r, XWork w) {
  GRID_STRIDE(m, r.nm) {
    D4 l0{0, 0, 0, 0};
    double pi = 0.0;
    int src = -1;
    if (w.np[m] > 0) {
      const u64 k = manKey(r.mab[m]);
      const int j = lowerBoundKeys(r.lkeys, r.L, k);
      if (j < r.L && r.lkeys[j] == k) {
        l0 = r.lval[j];
        pi = r.lpos[j];
        src = j;
      }
    }
    w.lam0[m] = w.lam[m] = l0;
    w.posIn[m] = pi;
    w.src[m] = src;
  }
}

__device__ __forceinline__ ManC manC(const XScene& sc, const XView& r, const XWork& w, int m, int sf) {
  const int2 ab = r.mab[m];
  const bool hasB = ab.y >= 0;
  ManC c;
  c.invN = 1.0 / static_cast<double>(w.np[m]);
  c.hasB = hasB;
  c.wv = V3<double>{0.0, 0.0, 0.0};
  c.imA = sc.invMass[ab.x];
  c.imB = hasB ? sc.invMass[ab.y] : 0.0;
  c.iIA = v3d(sc.invI[ab.x]);
  c.iIB = hasB ? v3d(sc.invI[ab.y]) : V3<double>{0.0, 0.0, 0.0};
  c.eAvg = -1.0;
  c.muAvg = -1.0;
  c.sf = sf;
  return c;
}
__device__ __forceinline__ void geoIn(const XWork& w, int m, double* in, int o) {
  for (int j = 0; j < 5; ++j)
    put3(in, o + 3 * j, w.geo[5 * m + j]);
}
__device__ __forceinline__ void quatIn(const XScene& sc, const XView& r, int2 ab, double* in, int o) {
  put4(in, o, r.st[sc.n + ab.x]);
  put4(in, o + 4, ab.y >= 0 ? r.st[sc.n + ab.y] : D4{0.0, 0.0, 0.0, 1.0});
}

__global__ void kxVn0(XScene sc, XView r, XWork w) {
  GRID_STRIDE(m, r.nm) {
    if (w.np[m] <= 0) {
      w.vn[m] = D4{0, 0, 0, 0};
      continue;
    }
    const int2 ab = r.mab[m];
    double in[kVn0In], out[kVn0Out];
    for (int j = 0; j < 12; ++j)
      in[j] = 0.0;
    put3(in, 0, w.vP0[ab.x]);
    put3(in, 3, w.wP0[ab.x]);
    if (ab.y >= 0) {
      put3(in, 6, w.vP0[ab.y]);
      put3(in, 9, w.wP0[ab.y]);
    }
    geoIn(w, m, in, 12);
    vn0Map<double>(in, out, manC(sc, r, w, m, 0));
    w.vn[m] = D4{out[1], out[2], out[3], out[0]};
  }
}

__device__ __forceinline__ void velIn(const XWork& w, int2 ab, double* in) {
  for (int j = 0; j < 12; ++j)
    in[j] = 0.0;
  put3(in, 0, w.vP[ab.x]);
  put3(in, 3, w.wP[ab.x]);
  if (ab.y >= 0) {
    put3(in, 6, w.vP[ab.y]);
    put3(in, 9, w.wP[ab.y]);
  }
}
__device__ __forceinline__ void velOut(const XWork& w, int2 ab, const double* out) {
  w.vP[ab.x] = get3(out, 0);
  w.wP[ab.x] = get3(out, 3);
  if (ab.y >= 0) {
    w.vP[ab.y] = get3(out, 6);
    w.wP[ab.y] = get3(out, 9);
  }
}

__global__ void kxWarm(XScene sc, XView r, XWork w, int col) {
  const int b = r.mOff[col], cnt = r.mOff[col + 1] - b;
  GRID_STRIDE(t, cnt) {
    const int m = r.mOrder[b + t];
    if (w.np[m] <= 0)
      continue;
    const int2 ab = r.mab[m];
    double in[kWarmIn], out[kWarmOut];
    velIn(w, ab, in);
    in[12] = w.lam0[m].w;
    put3(in, 13, w.lam0[m]);
    geoIn(w, m, in, 16);
    quatIn(sc, r, ab, in, 31);
    warmMap<double>(in, out, manC(sc, r, w, m, 0));
    velOut(w, ab, out);
    w.lam[m] = get3(out, 12, w.lam0[m].w);
  }
}

__device__ __forceinline__ void pgsIn(const XScene& sc, const XView& r, const XWork& w, int m, int2 ab, double* in) {
  in[12] = w.lam[m].w;
  put3(in, 13, w.lam[m]);
  geoIn(w, m, in, 16);
  quatIn(sc, r, ab, in, 31);
  in[39] = w.vn[m].w;
  put3(in, 40, w.vn[m]);
  in[43] = w.posIn[m];
  in[44] = sc.eN;
  in[45] = sc.eT;
  in[46] = sc.mu;
}

// one PGS update of the replay: manifold m at sweep `sweep` (its inputs kept on the tape)
__device__ __forceinline__ void pgsFwdEntry(const XScene& sc, const XView& r, const XWork& w, int m, int sweep,
                                            double vRest, int stab, int tag, u64& hs) {
  if (w.np[m] <= 0)
    return;
  const int2 ab = r.mab[m];
  double in[kPgsIn], out[kPgsOut];
  velIn(w, ab, in);
  pgsIn(sc, r, w, m, ab, in);
  D4* tape = w.tv + 4 * ((long)sweep * r.nm + m);
  tape[0] = get3(in, 0, in[12]);
  tape[1] = get3(in, 3, in[13]);
  tape[2] = get3(in, 6, in[14]);
  tape[3] = get3(in, 9, in[15]);
  unsigned bits = 0;
  pgsMap<double>(in, out, manC(sc, r, w, m, stab ? (int)r.sf[m] : 0), vRest, w.hash ? &bits : nullptr);
  if (w.hash)
    hs += mixWord(((u64)(unsigned)tag << 40) ^ ((u64)(unsigned)sweep << 28) ^ ((u64)(unsigned)m << 8) ^ bits);
  velOut(w, ab, out);
  w.lam[m] = get3(out, 13, out[12]);
}

__global__ void kxPgs(XScene sc, XView r, XWork w, int col, int sweep, double vRest, int stab, int tag) {
  const int b = r.mOff[col], cnt = r.mOff[col + 1] - b;
  u64 hs = 0;
  GRID_STRIDE(t, cnt) { pgsFwdEntry(sc, r, w, r.mOrder[b + t], sweep, vRest, stab, tag, hs); }
  if (w.hash)
    warpHashAdd(w.hash, hs);
}

// the replay's main and stabilization sweeps in one persistent launch of one thread-block
// cluster: colour by colour, a cluster barrier between colours (the blocks take fixed contiguous
// slices of each colour, so an entry's constants stay in its SM's L1 across the sweeps)
__global__ void __launch_bounds__(kB) kxPgsCluster(XScene sc, XView r, XWork w, int velSweeps, int stabSweeps,
                                                   double vRest, int tag) {
  const int nb = gridDim.x;
  u64 hs = 0;
  for (int it = 0; it < velSweeps + stabSweeps; ++it) {
    const int stab = it >= velSweeps ? 1 : 0;
    for (int c = 0; c < r.ncolV; ++c) {
      const int b = r.mOff[c], cnt = r.mOff[c + 1] - b;
      const int lo = (int)((long)cnt * blockIdx.x / nb), hi = (int)((long)cnt * (blockIdx.x + 1) / nb);
      for (int t = lo + threadIdx.x; t < hi; t += blockDim.x)
        pgsFwdEntry(sc, r, w, r.mOrder[b + t], it, vRest, stab, tag, hs);
      cg::this_cluster().sync();
    }
  }
  if (w.hash)
    warpHashAdd(w.hash, hs);
}

__global__ void kxIntegrate(XScene sc, XView r, XWork w) {
  GRID_STRIDE(i, sc.n) {
    double in[kIntIn], out[kIntOut];
    put3(in, 0, r.st[i]);
    put4(in, 3, r.st[sc.n + i]);
    put3(in, 7, r.st[2 * sc.n + i]);
    put3(in, 10, w.vP[i]);
    put3(in, 13, w.wP[i]);
    integrateMap<double>(in, out, sc.invMass[i], sc.dt);
    w.vF[i] = w.vP[i];
    w.wF[i] = w.wP[i];
    w.xP[i] = get3(out, 0);
    w.qP[i] = get4(out, 3);
  }
}

__device__ __forceinline__ PosC posC(const XScene& sc, int2 ab) {
  const bool hasB = ab.y >= 0;
  PosC c;
  c.hasB = hasB;
  c.imA = sc.invMass[ab.x];
  c.imB = hasB ? sc.invMass[ab.y] : 0.0;
  c.iIA = v3d(sc.invI[ab.x]);
  c.iIB = hasB ? v3d(sc.invI[ab.y]) : V3<double>{0.0, 0.0, 0.0};
  return c;
}
__device__ __forceinline__ void posIn(const XScene& sc, const XView& r, const XWork& w, int k, int2 ab, D4 xA, D4 xB,
                                      double* in) {
  const D4 id{0.0, 0.0, 0.0, 1.0};
  put3(in, 0, xA);
  put3(in, 3, xB);
  put4(in, 6, w.qP[ab.x]);
  put4(in, 10, ab.y >= 0 ? w.qP[ab.y] : id);
  put4(in, 14, r.st[sc.n + ab.x]);
  put4(in, 18, ab.y >= 0 ? r.st[sc.n + ab.y] : id);
  put3(in, 22, w.cgN[k]);
  put3(in, 25, w.cgA[k]);
  put3(in, 28, w.cgB[k]);
}

__global__ void kxPos(XScene sc, XView r, XWork w, int col, int sweep, int tag) {
  const int b = r.cOff[col], cnt = r.cOff[col + 1] - b;
  u64 hs = 0;
  GRID_STRIDE(t, cnt) {
    const int k = r.cOrder[b + t];
    const int2 ab = r.cab[k];
    const D4 xA = w.xP[ab.x], xB = ab.y >= 0 ? w.xP[ab.y] : D4{0, 0, 0, 0};
    D4* tape = w.tp + 2 * ((long)sweep * r.nc + k);
    tape[0] = xA;
    tape[1] = xB;
    double in[kPosIn], out[kPosOut];
    posIn(sc, r, w, k, ab, xA, xB, in);
    unsigned bits = 0;
    posMap<double>(in, out, posC(sc, ab), w.hash ? &bits : nullptr);
    if (w.hash)
      hs += mixWord(((u64)(unsigned)tag << 40) ^ ((u64)(unsigned)(sweep + 4096) << 28) ^ ((u64)(unsigned)k << 8) ^ bits);
    w.xP[ab.x] = get3(out, 0);
    if (ab.y >= 0)
      w.xP[ab.y] = get3(out, 3);
    w.posLam[k] += out[6];
  }
  if (w.hash)
    warpHashAdd(w.hash, hs);
}

// the replay's end state against the recorded start of the next substep
__global__ void kxCheck(XScene sc, XView next, XWork w) {
  double ex = 0.0, ev = 0.0;
  GRID_STRIDE(i, sc.n) {
    const D4 x = w.xP[i], X = next.st[i], v = w.vF[i], V = next.st[2 * sc.n + i];
    ex = ::fmax(ex, ::fmax(::fabs(x.x - X.x), ::fmax(::fabs(x.y - X.y), ::fabs(x.z - X.z))));
    ev = ::fmax(ev, ::fmax(::fabs(v.x - V.x), ::fmax(::fabs(v.y - V.y), ::fabs(v.z - V.z))));
  }
  atomicMaxPos(&w.err[0], ex / sc.gs);
  atomicMaxPos(&w.err[1], ev);
}

// ---------------- reverse ----------------
__global__ void kxRevInit(XScene sc, XView r, XWork w) {
  const long nmax = max((long)sc.n, max((long)r.nc, (long)r.nm));
  GRID_STRIDE(i, nmax) {
    const D4 z{0, 0, 0, 0};
    if (i < sc.n) {
      w.axP[i] = w.gx[i];
      w.aqP[i] = w.gq[i];
      w.ax[i] = w.aq[i] = w.av[i] = w.aw[i] = w.axP0[i] = z;
    }
    if (i < r.nc) {
      const int m = r.cSlot[i];
      w.aposLam[i] = (w.np[m] > 0 ? w.aposOut[m] : 0.0) / sc.dt;
      w.acgN[i] = w.acgA[i] = w.acgB[i] = z;
    }
    if (i < r.nm) {
      for (int j = 0; j < 5; ++j)
        w.ageo[5 * i + j] = z;
      w.avn[i] = w.ath[i] = z;
      w.aposIn[i] = 0.0;
      w.alam[i] = w.alamOut[i];
    }
  }
}

__global__ void __launch_bounds__(kBR) kxPosRev(XScene sc, XView r, XWork w, int col, int sweep) {
  __shared__ double sx[kBR / kGroup][kPosIn];
  const int b = r.cOff[col], cnt = r.cOff[col + 1] - b;
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < cnt; t0 += (long)gridDim.x * per) {
    const long t = t0 + slot;
    const int k = t < cnt ? r.cOrder[b + t] : -1;
    int2 ab{0, -1};
    if (k >= 0) {
      ab = r.cab[k];
      if (lane * kLanes < kPosIn) {
        const D4* tape = w.tp + 2 * ((long)sweep * r.nc + k);
        double in[kPosIn], yb[kPosOut], part[kLanes];
        posIn(sc, r, w, k, ab, tape[0], tape[1], in);
        for (int j = 0; j < kPosOut; ++j)
          yb[j] = 0.0;
        put3(yb, 0, w.axP[ab.x]);
        if (ab.y >= 0)
          put3(yb, 3, w.axP[ab.y]);
        yb[6] = w.aposLam[k];
        const PosC pc = posC(sc, ab);
        vjpChunk<kPosIn, kPosOut>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { posMap(x, y, pc); });
        for (int l = 0; l < kLanes && lane * kLanes + l < kPosIn; ++l)
          sx[slot][lane * kLanes + l] = part[l];
      }
    }
    __syncthreads();
    if (k >= 0 && lane == 0) {
      const double* xb = sx[slot];
      w.axP[ab.x] = get3(xb, 0);
      add4(w.aqP[ab.x], xb + 6);
      add4(w.aq[ab.x], xb + 14);
      if (ab.y >= 0) {
        w.axP[ab.y] = get3(xb, 3);
        add4(w.aqP[ab.y], xb + 10);
        add4(w.aq[ab.y], xb + 18);
      }
      add3(w.acgN[k], xb + 22);
      add3(w.acgA[k], xb + 25);
      add3(w.acgB[k], xb + 28);
    }
    __syncthreads();
  }
}

// the hand-written reverses of the position update, the warm start and the approach velocity:
// one entry a thread (the grouped kernels above and below reverse the same maps through
// forward-mode chunks: the cross-check)
__global__ void kxPosRevH(XScene sc, XView r, XWork w, int col, int sweep) {
  const int b = r.cOff[col], cnt = r.cOff[col + 1] - b;
  GRID_STRIDE(t, cnt) {
    const int k = r.cOrder[b + t];
    const int2 ab = r.cab[k];
    const D4* tape = w.tp + 2 * ((long)sweep * r.nc + k);
    double in[kPosIn], yb[kPosOut], xb[kPosIn];
    posIn(sc, r, w, k, ab, tape[0], tape[1], in);
    for (int j = 0; j < kPosOut; ++j)
      yb[j] = 0.0;
    put3(yb, 0, w.axP[ab.x]);
    if (ab.y >= 0)
      put3(yb, 3, w.axP[ab.y]);
    yb[6] = w.aposLam[k];
    for (int j = 0; j < kPosIn; ++j)
      xb[j] = 0.0;
    posRev(in, yb, xb, posC(sc, ab));
    w.axP[ab.x] = get3(xb, 0);
    add4(w.aqP[ab.x], xb + 6);
    add4(w.aq[ab.x], xb + 14);
    if (ab.y >= 0) {
      w.axP[ab.y] = get3(xb, 3);
      add4(w.aqP[ab.y], xb + 10);
      add4(w.aq[ab.y], xb + 18);
    }
    add3(w.acgN[k], xb + 22);
    add3(w.acgA[k], xb + 25);
    add3(w.acgB[k], xb + 28);
  }
}
// over every manifold in one launch: the body adjoints it reads are the sweeps' (not changed
// here), and its orientation adjoints accumulate with atomics
__global__ void kxWarmRevH(XScene sc, XView r, XWork w) {
  GRID_STRIDE(t, r.nm) {
    const int m = (int)t;
    if (w.np[m] <= 0)
      continue;
    const int2 ab = r.mab[m];
    double in[kWarmIn], yb[kWarmOut], xb[kWarmIn];
    for (int j = 0; j < 12; ++j)
      in[j] = 0.0;
    in[12] = w.lam0[m].w;
    put3(in, 13, w.lam0[m]);
    geoIn(w, m, in, 16);
    quatIn(sc, r, ab, in, 31);
    for (int j = 0; j < kWarmOut; ++j)
      yb[j] = 0.0;
    put3(yb, 0, w.avP[ab.x]);
    put3(yb, 3, w.awP[ab.x]);
    if (ab.y >= 0) {
      put3(yb, 6, w.avP[ab.y]);
      put3(yb, 9, w.awP[ab.y]);
    }
    put3(yb, 12, w.alam[m]);
    for (int j = 0; j < kWarmIn; ++j)
      xb[j] = 0.0;
    warmRev(in, yb, xb, manC(sc, r, w, m, 0));
    w.alam[m] = get3(xb, 13, w.alam[m].w + xb[12]);
    for (int j = 0; j < 5; ++j)
      add3(w.ageo[5 * m + j], xb + 16 + 3 * j);
    atomicAdd4(&w.aq[ab.x], xb + 31);
    if (ab.y >= 0)
      atomicAdd4(&w.aq[ab.y], xb + 35);
  }
}
// over every manifold in one launch, after every warm-start reverse: the velocity adjoints become
// those of the predicted velocities (atomics: manifolds share bodies)
__global__ void kxVn0RevH(XScene sc, XView r, XWork w) {
  GRID_STRIDE(t, r.nm) {
    const int m = (int)t;
    if (w.np[m] <= 0)
      continue;
    const int2 ab = r.mab[m];
    double in[kVn0In], yb[kVn0Out], xb[kVn0In];
    for (int j = 0; j < 12; ++j)
      in[j] = 0.0;
    put3(in, 0, w.vP0[ab.x]);
    put3(in, 3, w.wP0[ab.x]);
    if (ab.y >= 0) {
      put3(in, 6, w.vP0[ab.y]);
      put3(in, 9, w.wP0[ab.y]);
    }
    geoIn(w, m, in, 12);
    yb[0] = w.avn[m].w;
    put3(yb, 1, w.avn[m]);
    for (int j = 0; j < kVn0In; ++j)
      xb[j] = 0.0;
    vn0Rev(in, yb, xb, manC(sc, r, w, m, 0));
    atomicAdd3(&w.avP[ab.x], xb);
    atomicAdd3(&w.awP[ab.x], xb + 3);
    if (ab.y >= 0) {
      atomicAdd3(&w.avP[ab.y], xb + 6);
      atomicAdd3(&w.awP[ab.y], xb + 9);
    }
    for (int j = 0; j < 5; ++j)
      add3(w.ageo[5 * m + j], xb + 12 + 3 * j);
  }
}

__global__ void __launch_bounds__(kBR) kxIntegrateRev(XScene sc, XView r, XWork w) {
  __shared__ double sx[kBR / kGroup][kIntIn];
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < sc.n; t0 += (long)gridDim.x * per) {
    const long i = t0 + slot;
    if (i < sc.n && lane * kLanes < kIntIn) {
      double in[kIntIn], yb[kIntOut], part[kLanes];
      put3(in, 0, r.st[i]);
      put4(in, 3, r.st[sc.n + i]);
      put3(in, 7, r.st[2 * sc.n + i]);
      put3(in, 10, w.vF[i]);
      put3(in, 13, w.wF[i]);
      put3(yb, 0, w.axP[i]);
      put4(yb, 3, w.aqP[i]);
      const double im = sc.invMass[i], dt = sc.dt;
      vjpChunk<kIntIn, kIntOut>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { integrateMap(x, y, im, dt); });
      for (int l = 0; l < kLanes && lane * kLanes + l < kIntIn; ++l)
        sx[slot][lane * kLanes + l] = part[l];
    }
    __syncthreads();
    if (i < sc.n && lane == 0) {
      const double* xb = sx[slot];
      add3(w.ax[i], xb);
      add4(w.aq[i], xb + 3);
      add3(w.av[i], xb + 7);
      D4 a = w.gv[i], c = w.gw[i];
      add3(a, xb + 10);
      add3(c, xb + 13);
      w.avP[i] = a;
      w.awP[i] = c;
    }
    __syncthreads();
  }
}

// the reverse of one PGS update (manifold m at sweep `sweep`). MODE 0: the hand-written reverse
// (pgsRev); MODE 1: the forward-mode local Jacobian (the check)
template <int MODE>
__device__ __forceinline__ void pgsRevEntry(const XScene& sc, const XView& r, const XWork& w, int m, int sweep,
                                            double vRest, int stab) {
  if (w.np[m] <= 0)
    return;
  const int2 ab = r.mab[m];
  const bool hasB = ab.y >= 0;
  const D4* tape = w.tv + 4 * ((long)sweep * r.nm + m);
  double in[kPgsIn], yb[kPgsOut], xb[kPgsIn];
  put3(in, 0, tape[0]);
  put3(in, 3, tape[1]);
  put3(in, 6, tape[2]);
  put3(in, 9, tape[3]);
  in[12] = tape[0].w;
  in[13] = tape[1].w;
  in[14] = tape[2].w;
  in[15] = tape[3].w;
  geoIn(w, m, in, 16);
  quatIn(sc, r, ab, in, 31);
  in[39] = w.vn[m].w;
  put3(in, 40, w.vn[m]);
  in[43] = w.posIn[m];
  in[44] = sc.eN;
  in[45] = sc.eT;
  in[46] = sc.mu;
  for (int j = 0; j < kPgsOut; ++j)
    yb[j] = 0.0;
  put3(yb, 0, w.avP[ab.x]);
  put3(yb, 3, w.awP[ab.x]);
  if (hasB) {
    put3(yb, 6, w.avP[ab.y]);
    put3(yb, 9, w.awP[ab.y]);
  }
  yb[12] = w.alam[m].w;
  put3(yb, 13, w.alam[m]);
  for (int j = 0; j < kPgsIn; ++j)
    xb[j] = 0.0;
  const ManC mc = manC(sc, r, w, m, stab ? (int)r.sf[m] : 0);
  if (MODE == 0)
    pgsRev(in, yb, xb, mc, vRest);
  else
    vjp<kPgsIn, kPgsOut>(in, yb, xb, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { pgsMap(x, y, mc, vRest); });
  w.avP[ab.x] = get3(xb, 0);
  w.awP[ab.x] = get3(xb, 3);
  add4(w.aq[ab.x], xb + 31);
  if (hasB) {
    w.avP[ab.y] = get3(xb, 6);
    w.awP[ab.y] = get3(xb, 9);
    add4(w.aq[ab.y], xb + 35);
  }
  w.alam[m] = get3(xb, 13, xb[12]);
  for (int j = 0; j < 5; ++j)
    add3(w.ageo[5 * m + j], xb + 16 + 3 * j);
  D4 av = w.avn[m];
  av.w += xb[39];
  add3(av, xb + 40);
  w.avn[m] = av;
  w.aposIn[m] += xb[43];
  add3(w.ath[m], xb + 44);
}

template <int MODE>
__global__ void kxPgsRev(XScene sc, XView r, XWork w, int col, int sweep, double vRest, int stab) {
  const int b = r.mOff[col], cnt = r.mOff[col + 1] - b;
  GRID_STRIDE(t, cnt) { pgsRevEntry<MODE>(sc, r, w, r.mOrder[b + t], sweep, vRest, stab); }
}

// the reverse of both PGS loops in one persistent cluster launch: sweeps and colours in reverse
// order, the same slices of each colour per block as the replay's
__global__ void __launch_bounds__(kB) kxPgsRevCluster(XScene sc, XView r, XWork w, int velSweeps, int stabSweeps,
                                                      double vRest) {
  const int nb = gridDim.x;
  for (int it = velSweeps + stabSweeps - 1; it >= 0; --it) {
    const int stab = it >= velSweeps ? 1 : 0;
    for (int c = r.ncolV - 1; c >= 0; --c) {
      const int b = r.mOff[c], cnt = r.mOff[c + 1] - b;
      const int lo = (int)((long)cnt * blockIdx.x / nb), hi = (int)((long)cnt * (blockIdx.x + 1) / nb);
      for (int t = lo + threadIdx.x; t < hi; t += blockDim.x)
        pgsRevEntry<0>(sc, r, w, r.mOrder[b + t], it, vRest, stab);
      cg::this_cluster().sync();
    }
  }
}

__global__ void __launch_bounds__(kBR) kxWarmRev(XScene sc, XView r, XWork w, int col) {
  __shared__ double sx[kBR / kGroup][kWarmIn];
  const int b = r.mOff[col], cnt = r.mOff[col + 1] - b;
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < cnt; t0 += (long)gridDim.x * per) {
    const long t = t0 + slot;
    int m = t < cnt ? r.mOrder[b + t] : -1;
    if (m >= 0 && w.np[m] <= 0)
      m = -1;
    int2 ab{0, -1};
    if (m >= 0) {
      ab = r.mab[m];
      if (lane * kLanes < kWarmIn) {
        double in[kWarmIn], yb[kWarmOut], part[kLanes];
        for (int j = 0; j < 12; ++j)
          in[j] = 0.0;  // the increments do not depend on the velocities
        in[12] = w.lam0[m].w;
        put3(in, 13, w.lam0[m]);
        geoIn(w, m, in, 16);
        quatIn(sc, r, ab, in, 31);
        for (int j = 0; j < kWarmOut; ++j)
          yb[j] = 0.0;
        put3(yb, 0, w.avP[ab.x]);
        put3(yb, 3, w.awP[ab.x]);
        if (ab.y >= 0) {
          put3(yb, 6, w.avP[ab.y]);
          put3(yb, 9, w.awP[ab.y]);
        }
        put3(yb, 12, w.alam[m]);
        const ManC mc = manC(sc, r, w, m, 0);
        vjpChunk<kWarmIn, kWarmOut>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { warmMap(x, y, mc); });
        for (int l = 0; l < kLanes && lane * kLanes + l < kWarmIn; ++l)
          sx[slot][lane * kLanes + l] = part[l];
      }
    }
    __syncthreads();
    if (m >= 0 && lane == 0) {
      const double* xb = sx[slot];
      // lambda enters the sweeps unchanged and the warm start; lambda_T only through the warm start
      w.alam[m] = get3(xb, 13, w.alam[m].w + xb[12]);
      for (int j = 0; j < 5; ++j)
        add3(w.ageo[5 * m + j], xb + 16 + 3 * j);
      add4(w.aq[ab.x], xb + 31);
      if (ab.y >= 0)
        add4(w.aq[ab.y], xb + 35);
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBR) kxVn0Rev(XScene sc, XView r, XWork w, int col) {
  __shared__ double sx[kBR / kGroup][kVn0In];
  const int b = r.mOff[col], cnt = r.mOff[col + 1] - b;
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < cnt; t0 += (long)gridDim.x * per) {
    const long t = t0 + slot;
    int m = t < cnt ? r.mOrder[b + t] : -1;
    if (m >= 0 && w.np[m] <= 0)
      m = -1;
    int2 ab{0, -1};
    if (m >= 0) {
      ab = r.mab[m];
      if (lane * kLanes < kVn0In) {
        double in[kVn0In], yb[kVn0Out], part[kLanes];
        for (int j = 0; j < 12; ++j)
          in[j] = 0.0;
        put3(in, 0, w.vP0[ab.x]);
        put3(in, 3, w.wP0[ab.x]);
        if (ab.y >= 0) {
          put3(in, 6, w.vP0[ab.y]);
          put3(in, 9, w.wP0[ab.y]);
        }
        geoIn(w, m, in, 12);
        yb[0] = w.avn[m].w;
        put3(yb, 1, w.avn[m]);
        const ManC mc = manC(sc, r, w, m, 0);
        vjpChunk<kVn0In, kVn0Out>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { vn0Map(x, y, mc); });
        for (int l = 0; l < kLanes && lane * kLanes + l < kVn0In; ++l)
          sx[slot][lane * kLanes + l] = part[l];
      }
    }
    __syncthreads();
    if (m >= 0 && lane == 0) {
      const double* xb = sx[slot];
      add3(w.avP[ab.x], xb);
      add3(w.awP[ab.x], xb + 3);
      if (ab.y >= 0) {
        add3(w.avP[ab.y], xb + 6);
        add3(w.awP[ab.y], xb + 9);
      }
      for (int j = 0; j < 5; ++j)
        add3(w.ageo[5 * m + j], xb + 12 + 3 * j);
    }
    __syncthreads();
  }
}

__global__ void kxGatherRev(XScene sc, XView r, XWork w) {
  GRID_STRIDE(m, r.nm) {
    const int j = w.src[m];
    if (j >= 0) {
      w.alL[j] = w.alam[m];
      w.apL[j] = w.aposIn[m];
    }
  }
}

__global__ void __launch_bounds__(kBR) kxManifoldRev(XScene sc, XView r, XWork w) {
  __shared__ double sx[kBR / kGroup][kManIn];
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < r.nc; t0 += (long)gridDim.x * per) {
    const long k = t0 + slot;
    const bool on = k < r.nc && w.cgN[k].w <= 0.0;
    if (on && lane * kLanes < kManIn) {
      const int m = r.cSlot[k];
      const int2 ab = r.cab[k];
      double in[kManIn], yb[kManOut], part[kLanes];
      conIn(w, (int)k, in);
      for (int j = 0; j < 5; ++j)
        put3(yb, 3 * j, w.ageo[5 * m + j]);
      const bool flip = ab.y >= 0 && ab.y < ab.x;
      vjpChunk<kManIn, kManOut>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { manifoldMap(x, y, flip); });
      for (int l = 0; l < kLanes && lane * kLanes + l < kManIn; ++l)
        sx[slot][lane * kLanes + l] = part[l];
    }
    __syncthreads();
    if (on && lane == 0) {
      const double* xb = sx[slot];
      add3(w.acgN[k], xb);
      add3(w.acgA[k], xb + 3);
      add3(w.acgB[k], xb + 6);
      w.acgN[k].w += xb[9];
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBR) kxContactRev(XScene sc, XView r, XWork w) {
  __shared__ double sx[kBR / kGroup][kConIn];
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < r.nc; t0 += (long)gridDim.x * per) {
    const long k = t0 + slot;
    int2 ab{0, -1};
    if (k < r.nc) {
      ab = r.cab[k];
      if (ab.y >= 0 && lane * kLanes < kConIn) {
        double in[kConIn], yb[kConOut], part[kLanes];
        put3(in, 0, w.xP0[ab.x]);
        put4(in, 3, r.st[sc.n + ab.x]);
        put3(in, 7, w.xP0[ab.y]);
        put4(in, 10, r.st[sc.n + ab.y]);
        put3(yb, 0, w.acgN[k]);
        put3(yb, 3, w.acgA[k]);
        put3(yb, 6, w.acgB[k]);
        yb[9] = w.acgN[k].w;
        const ConC cc = conC(sc, ab.x, ab.y);
        vjpChunk<kConIn, kConOut>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { contactMap(x, y, cc); });
        for (int l = 0; l < kLanes && lane * kLanes + l < kConIn; ++l)
          sx[slot][lane * kLanes + l] = part[l];
      }
    }
    __syncthreads();
    if (k < r.nc && lane == 0) {
      if (ab.y >= 0) {
        const double* xb = sx[slot];
        atomicAdd3(&w.axP0[ab.x], xb);
        atomicAdd4(&w.aq[ab.x], xb + 3);
        atomicAdd3(&w.axP0[ab.y], xb + 7);
        atomicAdd4(&w.aq[ab.y], xb + 10);
      } else {
        // only the distance of a plane contact moves with the body: dist = (x - p) . n - radius
        const D4 n = w.cgN[k];
        const double g = w.acgN[k].w;
        const double v[3] = {g * n.x, g * n.y, g * n.z};
        atomicAdd3(&w.axP0[ab.x], v);
      }
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kBR) kxPredictRev(XScene sc, XView r, XWork w) {
  __shared__ double sx[kBR / kGroup][kPredIn];
  const int lane = threadIdx.x % kGroup, slot = threadIdx.x / kGroup, per = blockDim.x / kGroup;
  for (long t0 = (long)blockIdx.x * per; t0 < sc.n; t0 += (long)gridDim.x * per) {
    const long i = t0 + slot;
    if (i < sc.n && lane * kLanes < kPredIn) {
      double in[kPredIn], yb[kPredOut], part[kLanes];
      put3(in, 0, r.st[i]);
      put4(in, 3, r.st[sc.n + i]);
      put3(in, 7, r.st[2 * sc.n + i]);
      put3(in, 10, r.st[3 * sc.n + i]);
      put3(yb, 0, w.avP[i]);
      put3(yb, 3, w.awP[i]);
      put3(yb, 6, w.axP0[i]);
      const BodyC bc{sc.invMass[i], v3d(sc.invI[i])};
      const StepC st{sc.dt, sc.g, 0.0, sc.eps};
      const V3<double> F = v3d(sc.extF[i]);
      vjpChunk<kPredIn, kPredOut>(in, yb, part, lane, [&](const Dd<kLanes>* x, Dd<kLanes>* y) { predictMap(x, y, bc, st, F); });
      for (int l = 0; l < kLanes && lane * kLanes + l < kPredIn; ++l)
        sx[slot][lane * kLanes + l] = part[l];
    }
    __syncthreads();
    if (i < sc.n && lane == 0) {
      const double* xb = sx[slot];
      add3(w.ax[i], xb);
      add4(w.aq[i], xb + 3);
      add3(w.av[i], xb + 7);
      add3(w.aw[i], xb + 10);
    }
    __syncthreads();
  }
}

// sum of the per-manifold parameter adjoints into theta (one atomic per block)
__global__ void kxThetaSum(XView r, XWork w) {
  __shared__ double s[3][kB];
  double a = 0.0, b = 0.0, c = 0.0;
  GRID_STRIDE(m, r.nm) {
    a += w.ath[m].x;
    b += w.ath[m].y;
    c += w.ath[m].z;
  }
  s[0][threadIdx.x] = a, s[1][threadIdx.x] = b, s[2][threadIdx.x] = c;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int j = 0; j < 3; ++j)
        s[j][threadIdx.x] += s[j][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int j = 0; j < 3; ++j)
      atomicAdd(&w.theta[j], s[j][0]);
}

// the adjoint of the ledger a substep read, handed to the previous substep's manifolds by key
__global__ void kxLedgerMap(XView cur, XView prev, XWork w) {
  GRID_STRIDE(j, cur.L) {
    const D4 a = w.alL[j];
    const double p = w.apL[j];
    if (a.x == 0.0 && a.y == 0.0 && a.z == 0.0 && a.w == 0.0 && p == 0.0)
      continue;
    const int m = findManifold(prev.mab, prev.nm, cur.lkeys[j]);
    if (m >= 0) {
      w.alamPrev[m] = a;
      w.aposPrev[m] = p;
    }
  }
}

// ---------------- recording ----------------
// manifold contact ranges (contacts of a manifold are contiguous in the canonical contact order for
// spheres and planes); bad[0] counts manifolds whose contacts are not
__global__ void kxRanges(int nc, int nm, const int* cSlot, int* c0, int* cn, int* bad) {
  GRID_STRIDE(k, nc) {
    const int m = cSlot[k];
    if (k == 0 || cSlot[k - 1] != m)
      c0[m] = (int)k;
    atomicAdd(&cn[m], 1);
  }
}
__global__ void kxRangesCheck(int nc, int nm, const int* cSlot, const int* c0, const int* cn, int* bad) {
  GRID_STRIDE(m, nm) {
    const int a = c0[m], c = cn[m];
    bool ok = c > 0 && a >= 0 && a + c <= nc;
    for (int k = a; ok && k < a + c; ++k)
      ok = cSlot[k] == (int)m;
    if (!ok)
      atomicAdd(bad, 1);
  }
}
// plane of each wall contact (by its normal and point); bad[1] counts contacts with no plane
template <class R>
__global__ void kxPlanes(int nc, const int2* cab, const Q4<R>* cn, const Q4<R>* crB, const PlaneDesc<R>* planes,
                         int np, int* cPlane, int* bad) {
  GRID_STRIDE(k, nc) {
    int id = -1;
    if (cab[k].y < 0) {
      for (int j = 0; j < np && id < 0; ++j) {
        const PlaneDesc<R>& p = planes[j];
        if (p.n[0] == cn[k].x && p.n[1] == cn[k].y && p.n[2] == cn[k].z && p.p[0] == crB[k].x &&
            p.p[1] == crB[k].y && p.p[2] == crB[k].z)
          id = j;
      }
      if (id < 0)
        atomicAdd(&bad[1], 1);
    }
    cPlane[k] = id;
  }
}
// entries left uncoloured by the colourings (colour -1; inactive manifolds carry -2 and need no
// update): bad[2] manifolds, bad[3] contacts
__global__ void kxLeftover(int nm, const int* mColor, int nc, const int* cColor, int* bad) {
  GRID_STRIDE(i, max(nm, nc)) {
    if (i < nm && mColor[i] == -1)
      atomicAdd(&bad[2], 1);
    if (i < nc && cColor[i] == -1)
      atomicAdd(&bad[3], 1);
  }
}
// rows of 3 / 4 doubles <-> 4-wide records
__global__ void kxPack(int n, const double* a, int cols, D4* out) {
  GRID_STRIDE(i, n) {
    out[i] = D4{a[cols * i], a[cols * i + 1], a[cols * i + 2], cols == 4 ? a[cols * i + 3] : 0.0};
  }
}
__global__ void kxUnpack(int n, const D4* a, int cols, double* out) {
  GRID_STRIDE(i, n) {
    out[cols * i] = a[i].x;
    out[cols * i + 1] = a[i].y;
    out[cols * i + 2] = a[i].z;
    if (cols == 4)
      out[cols * i + 3] = a[i].w;
  }
}
__global__ void kxLedgerVals(int L, const double* lam, const D4* lt, D4* out) {
  GRID_STRIDE(j, L) { out[j] = D4{lt[j].x, lt[j].y, lt[j].z, lam[j]}; }
}

}  // namespace

// ---------------- host side ----------------
// one cluster of `blocks` blocks on `st`; false (nothing launched) when such a cluster cannot be
// resident (the answer is cached per kernel)
template <class K, class... A>
bool launchOneCluster(K kernel, int blocks, int block, cudaStream_t st, A... args) {
  static int ok = -1;  // one cache per kernel instantiation
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = blocks;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (ok < 0) {
    int clusters = 0;
    if (blocks > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
      (void)cudaGetLastError();
    if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) != cudaSuccess)
      (void)cudaGetLastError();
    ok = clusters >= 1 ? 1 : 0;
  }
  if (!ok)
    return false;
  cudaCheck(cudaLaunchKernelEx(&cfg, kernel, args...), "xadj cluster launch");
  return true;
}

struct XRec {
  int nc = 0, nm = 0, L = 0, ncolV = 0, ncolP = 0, velSweeps = 0, stabSweeps = 0, posSweeps = 0;
  bool stab = false;
  size_t oCab = 0, oSlot = 0, oCOrd = 0, oCOff = 0, oCPl = 0, oMab = 0, oMOrd = 0, oMOff = 0, oMC0 = 0, oMCn = 0;
  DBuf<int> ints;
  DBuf<uint8_t> sf;
  DBuf<D4> st;
  DBuf<u64> lkeys;
  DBuf<D4> lval;
  DBuf<double> lpos;
  size_t bytes() const {
    return ints.n * sizeof(int) + sf.n + st.n * sizeof(D4) + lkeys.n * sizeof(u64) + lval.n * sizeof(D4) +
           lpos.n * sizeof(double);
  }
};

struct XAdj {
  std::vector<std::unique_ptr<XRec>> recs;
  bool open = false;
  int n = 0;
  double dt = 0, mat[3] = {0, 0, 0}, grav[3] = {0, 0, 0};
  // workspace: two sets of replay buffers (the replay of a substep runs beside the reverse of the
  // next one, on the side stream) and one set of adjoint buffers
  DBuf<D4> rbody[2], rcont[2], rman[2], tv[2], tp[2];
  DBuf<double> rcdbl[2], rmdbl[2];
  DBuf<int> rmint[2];
  DBuf<D4> abody, acont, aman, alLB;
  DBuf<double> acdbl, amdbl, ldbl, small;
  DBuf<u64> hashBuf;
  cudaStream_t side = nullptr;
  cudaEvent_t evStart = nullptr, evRep[2] = {nullptr, nullptr}, evRev[2] = {nullptr, nullptr};
  ~XAdj() {
    for (cudaEvent_t e : {evStart, evRep[0], evRep[1], evRev[0], evRev[1]})
      if (e)
        cudaEventDestroy(e);
    if (side)
      cudaStreamDestroy(side);
  }
  double err[2] = {0, 0};
  size_t workBytes = 0;
  // PDEM_XADJ_DUAL=1: the PGS, warm-start, approach-velocity and position updates reversed through
  // forward-mode local Jacobians instead of the hand-written reverses (the cross-check of the hand
  // derivations; slower)
  int dualCheck = [] {
    const char* e = std::getenv("PDEM_XADJ_DUAL");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  int maxSweeps = 0;
};

struct XAdjAccess {
  using S = Sim<double>;
  static XAdj& get(S& s) {
    if (!s.xadj_)
      s.xadj_ = std::shared_ptr<void>(new XAdj, [](void* p) { delete static_cast<XAdj*>(p); });
    return *static_cast<XAdj*>(s.xadj_.get());
  }
  static void checkScope(S& s) {
    auto bad = [](const char* why) { throw std::invalid_argument(std::string("XPBD adjoint: ") + why); };
    if (s.batch_)
      bad("one scene only (not the batched form)");
    if (s.mixed_)
      bad("the FP64 plain path only");
    if (s.shape_.type != SHAPE_SPHERE || s.shape_.numPoints != 0)
      bad("sphere shapes without point shells only");
    if (s.per_[0] || s.per_[1] || s.per_[2])
      bad("no periodic domains");
    if (s.gr_ != 0.0 || s.gf_ > 0.0)
      bad("no growth");
    if (s.thTau_ > 0.0)
      bad("no thermostat");
    if (!s.wallsHost_.empty())
      bad("planes are the only walls (no SDF walls)");
    if (!s.pairMatHost_.empty())
      bad("no pair materials");
    if (!s.useGS_ || (s.g_[0] == 0.0 && s.g_[1] == 0.0 && s.g_[2] == 0.0))
      bad("the PGS path (gravity on, Gauss-Seidel velocity solve)");
    if (s.stabMode_ != 0 && s.stabMode_ != 1 && s.stabMode_ != 3)
      bad("stabilization off, one-sided or escalate");
  }
  static void isotropic(S& s) {
    std::vector<D4> ii(s.numReal_);
    cudaCheck(cudaMemcpyAsync(ii.data(), s.invI_.p, ii.size() * sizeof(D4), cudaMemcpyDeviceToHost, s.stream_), "D2H");
    s.sync();
    for (const D4& v : ii)
      if (!(v.x == v.y && v.y == v.z))
        throw std::invalid_argument("XPBD adjoint: isotropic inverse inertia only (spheres)");
  }
  static XScene scene(S& s, const XAdj& A) {
    XScene c;
    c.n = s.numReal_;
    c.dt = A.dt;
    c.gs = s.gs_;
    c.par = s.shape_.par[0];
    c.eps = 1e-4;
    c.eN = A.mat[0];  // the rollout's own material and gravity (recorded by its first substep)
    c.eT = A.mat[1];
    c.mu = A.mat[2];
    c.g = V3<double>{A.grav[0], A.grav[1], A.grav[2]};
    c.invMass = s.invMass_.p;
    c.invI = s.invI_.p;
    c.scale = s.scale_.p;
    c.extF = s.extF_.p;
    c.planes = s.planesD_.p;
    return c;
  }

  // the rows the caller passes must be device memory (a host pointer would be read by a kernel)
  static void deviceRows(std::initializer_list<const void*> ps) {
    for (const void* p : ps) {
      cudaPointerAttributes a{};
      if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess ||
          (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        throw std::invalid_argument("XPBD adjoint: state rows must be device memory");
      }
    }
  }
  static void begin(S& s, const double* x, const double* q, const double* v, const double* w, int n) {
    checkScope(s);
    if (n > 0)
      deviceRows({x, q, v, w});
    if (n != s.numReal_)
      throw std::invalid_argument("XPBD adjoint: the state rows must cover every particle");
    isotropic(s);
    XAdj& A = get(s);
    A.recs.clear();
    A.open = true;
    A.n = n;
    cudaStream_t st = s.stream_;
    if (n > 0) {
      kxPack<<<gridFor(n), kB, 0, st>>>(n, x, 3, s.pos_.p);
      kxPack<<<gridFor(n), kB, 0, st>>>(n, q, 4, s.quat_.p);
      kxPack<<<gridFor(n), kB, 0, st>>>(n, v, 3, s.vel_.p);
      kxPack<<<gridFor(n), kB, 0, st>>>(n, w, 3, s.angVel_.p);
      cudaCheck(cudaGetLastError(), "xadj pack");
    }
    // a rollout is a function of its start state and parameters only: no warm start from before
    // it, support levels from zero, topology caches rebuilt
    s.ensureGrounded();
    if (s.grounded_.p)
      s.grounded_.zero(st);
    s.prevPairCount_ = 0;
    s.topoValid_ = false;
    s.vValid_ = false;
    s.bvhValid_ = false;
    s.sync();
  }

  static void step(S& s, double dt, int substeps) {
    XAdj& A = get(s);
    if (!A.open)
      throw std::invalid_argument("XPBD adjoint: xa_begin first");
    checkScope(s);
    if (s.numReal_ != A.n)
      throw std::invalid_argument("XPBD adjoint: the particle set changed during the rollout");
    if (!(dt > 0.0))
      dt = s.dt_;
    if (!A.recs.empty() && dt != A.dt)
      throw std::invalid_argument("XPBD adjoint: one substep length per rollout");
    A.dt = dt;
    // the material and gravity the rollout runs with: the backward uses these, not later settings
    const double mat[3] = {s.eN_, s.eT_, s.mu_}, grav[3] = {s.g_[0], s.g_[1], s.g_[2]};
    if (!A.recs.empty() && (std::memcmp(mat, A.mat, sizeof mat) || std::memcmp(grav, A.grav, sizeof grav)))
      throw std::invalid_argument("XPBD adjoint: the material or gravity changed during the rollout");
    std::memcpy(A.mat, mat, sizeof mat);
    std::memcpy(A.grav, grav, sizeof grav);
    cudaStream_t st = s.stream_;
    for (int it = 0; it < substeps; ++it) {
      auto R = std::make_unique<XRec>();
      const int n = A.n;
      // start state and the ledger the step reads
      R->st.ensure(4 * (size_t)std::max(n, 1), false, st);
      auto d2d = [&](void* dst, const void* src, size_t bytes) {
        if (bytes)
          cudaCheck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st), "xadj record");
      };
      d2d(R->st.p, s.pos_.p, n * sizeof(D4));
      d2d(R->st.p + n, s.quat_.p, n * sizeof(D4));
      d2d(R->st.p + 2 * n, s.vel_.p, n * sizeof(D4));
      d2d(R->st.p + 3 * n, s.angVel_.p, n * sizeof(D4));
      const int L = s.prevPairCount_;
      R->L = L;
      R->lkeys.ensure(std::max(L, 1), false, st);
      R->lval.ensure(std::max(L, 1), false, st);
      R->lpos.ensure(std::max(L, 1), false, st);
      if (L > 0) {
        d2d(R->lkeys.p, s.prevKeys_.p, L * sizeof(u64));
        kxLedgerVals<<<gridFor(L), kB, 0, st>>>(L, s.prevLambda_.p, s.prevLambdaT_.p, R->lval.p);
        d2d(R->lpos.p, s.prevPosImp_.p, L * sizeof(double));
      }
      s.step(dt);
      // the frozen decisions
      const Counters<double> c = s.readCounters();
      R->nc = c.contactCount;
      R->nm = c.manifoldCount;
      R->ncolV = s.ncolVLast_;
      R->ncolP = s.ncolPLast_;
      if (R->ncolV > kMaxColours || R->ncolP > kMaxColours)
        throw std::runtime_error("XPBD adjoint: a colouring saturated its 62 colours");
      R->velSweeps = c.velSweeps;
      // the one-sided pass sweeps with its side flags, escalate with none (they stay cleared)
      R->stab = c.stabRun != 0 && (s.stabMode_ == 1 || s.stabMode_ == 3);
      R->stabSweeps = R->stab ? c.stabSweeps : 0;
      R->posSweeps = c.posSweeps;
      const int nc = R->nc, nm = R->nm;
      size_t o = 0;
      R->oCab = o, o += 2 * (size_t)nc;
      R->oSlot = o, o += nc;
      R->oCOrd = o, o += nc;
      R->oCOff = o, o += R->ncolP + 1;
      R->oCPl = o, o += nc;
      o = (o + 1) & ~(size_t)1;  // int2 records start on 8 bytes
      R->oMab = o, o += 2 * (size_t)nm;
      R->oMOrd = o, o += nm;
      R->oMOff = o, o += R->ncolV + 1;
      R->oMC0 = o, o += nm;
      R->oMCn = o, o += nm;
      R->ints.ensure(o + 4, false, st);
      int* I = R->ints.p;
      d2d(I + R->oCab, s.cab_.p, nc * sizeof(int2));
      d2d(I + R->oSlot, s.cSlot_.p, nc * sizeof(int));
      if (R->ncolP > 0) {
        d2d(I + R->oCOrd, s.cOrder_.p, nc * sizeof(int));
        d2d(I + R->oCOff, s.cOff_.p, (R->ncolP + 1) * sizeof(int));
      }
      d2d(I + R->oMab, s.mab_.p, nm * sizeof(int2));
      if (R->ncolV > 0) {
        d2d(I + R->oMOrd, s.mOrder_.p, nm * sizeof(int));
        d2d(I + R->oMOff, s.mOff_.p, (R->ncolV + 1) * sizeof(int));
      }
      R->sf.ensure(std::max(nm, 1), false, st);
      if (R->stab && nm > 0)
        d2d(R->sf.p, s.sideFlags_.p, nm);
      int* bad = I + o;  // four counters after the layout (zeroed by ensure)
      if (nc > 0) {
        kxRanges<<<gridFor(nc), kB, 0, st>>>(nc, nm, I + R->oSlot, I + R->oMC0, I + R->oMCn, bad);
        kxRangesCheck<<<gridFor(nm), kB, 0, st>>>(nc, nm, I + R->oSlot, I + R->oMC0, I + R->oMCn, bad);
        kxPlanes<double><<<gridFor(nc), kB, 0, st>>>(nc, s.cab_.p, s.cn_.p, s.crB_.p, s.planesD_.p,
                                                    (int)s.planesHost_.size(), I + R->oCPl, bad);
        kxLeftover<<<gridFor(std::max(nc, nm)), kB, 0, st>>>(nm, s.mColor_.p, nc, s.cColor_.p, bad);
        cudaCheck(cudaGetLastError(), "xadj record");
      }
      int hb[4] = {0, 0, 0, 0};
      cudaCheck(cudaMemcpyAsync(hb, bad, sizeof hb, cudaMemcpyDeviceToHost, st), "D2H");
      s.sync();
      if (hb[0] || hb[1])
        throw std::runtime_error("XPBD adjoint: a manifold's contacts are not contiguous, or a wall contact has no plane");
      // every entry in a colour class: the Jacobi fallback for uncoloured entries is not reversed
      if (hb[2] || hb[3])
        throw std::runtime_error("XPBD adjoint: uncoloured entries (Jacobi fallback) in the rollout");
      A.recs.push_back(std::move(R));
    }
  }

  static XView view(const XRec& R) {
    XView v;
    v.nc = R.nc, v.nm = R.nm, v.L = R.L, v.ncolV = R.ncolV, v.ncolP = R.ncolP;
    const int* I = R.ints.p;
    v.cab = reinterpret_cast<const int2*>(I + R.oCab);
    v.cSlot = I + R.oSlot;
    v.cOrder = I + R.oCOrd;
    v.cOff = I + R.oCOff;
    v.cPlane = I + R.oCPl;
    v.mab = reinterpret_cast<const int2*>(I + R.oMab);
    v.mOrder = I + R.oMOrd;
    v.mOff = I + R.oMOff;
    v.mC0 = I + R.oMC0;
    v.mCn = I + R.oMCn;
    v.sf = R.sf.p;
    v.st = R.st.p;
    v.lkeys = R.lkeys.p;
    v.lval = R.lval.p;
    v.lpos = R.lpos.p;
    return v;
  }

  // carve the workspace for the largest substep of the record
  // carve the workspace for the largest substep of the record: W[0] and W[1] have their own replay
  // buffers and share the adjoint ones
  static void work(S& s, XAdj& A, XWork* W) {
    int n = std::max(A.n, 1), nc = 1, nm = 1, L = 1, sv = 1, sp = 1;
    for (auto& r : A.recs) {
      nc = std::max(nc, r->nc);
      nm = std::max(nm, r->nm);
      L = std::max(L, r->L);
      sv = std::max(sv, r->velSweeps + r->stabSweeps);
      sp = std::max(sp, r->posSweeps);
    }
    A.maxSweeps = std::max(sv, sp);
    cudaStream_t st = s.stream_;
    size_t bytes = 0;
    for (int k = 0; k < 2; ++k) {
      A.rbody[k].ensure(9 * (size_t)n, false, st);
      A.rcont[k].ensure(3 * (size_t)nc, false, st);
      A.rman[k].ensure(8 * (size_t)nm, false, st);
      A.tv[k].ensure(4 * (size_t)sv * nm, false, st);
      A.tp[k].ensure(2 * (size_t)sp * nc, false, st);
      A.rcdbl[k].ensure((size_t)nc, false, st);
      A.rmdbl[k].ensure((size_t)nm, false, st);
      A.rmint[k].ensure(2 * (size_t)nm, false, st);
      bytes += (A.rbody[k].n + A.rcont[k].n + A.rman[k].n + A.tv[k].n + A.tp[k].n) * sizeof(D4) +
               (A.rcdbl[k].n + A.rmdbl[k].n) * sizeof(double) + A.rmint[k].n * sizeof(int);
    }
    A.abody.ensure(13 * (size_t)n, false, st);
    A.acont.ensure(3 * (size_t)nc, false, st);
    A.aman.ensure(10 * (size_t)nm, false, st);
    A.alLB.ensure((size_t)L, false, st);
    A.acdbl.ensure((size_t)nc, false, st);
    A.amdbl.ensure(3 * (size_t)nm, false, st);
    A.ldbl.ensure((size_t)L, false, st);
    A.small.ensure(8, false, st);
    A.workBytes = bytes + (A.abody.n + A.acont.n + A.aman.n + A.alLB.n) * sizeof(D4) +
                  (A.acdbl.n + A.amdbl.n + A.ldbl.n + A.small.n) * sizeof(double);
    for (int k = 0; k < 2; ++k) {
      XWork& w = W[k];
      D4* b = A.rbody[k].p;
      w.vP0 = b, w.wP0 = b + n, w.xP0 = b + 2 * n, w.vP = b + 3 * n, w.wP = b + 4 * n, w.vF = b + 5 * n,
      w.wF = b + 6 * n, w.xP = b + 7 * n, w.qP = b + 8 * n;
      D4* a = A.abody.p;
      w.gx = a, w.gq = a + n, w.gv = a + 2 * n, w.gw = a + 3 * n;
      w.ax = a + 4 * n, w.aq = a + 5 * n, w.av = a + 6 * n, w.aw = a + 7 * n;
      w.axP = a + 8 * n, w.aqP = a + 9 * n, w.avP = a + 10 * n, w.awP = a + 11 * n, w.axP0 = a + 12 * n;
      D4* c = A.rcont[k].p;
      w.cgN = c, w.cgA = c + nc, w.cgB = c + 2 * nc;
      D4* ac = A.acont.p;
      w.acgN = ac, w.acgA = ac + nc, w.acgB = ac + 2 * nc;
      w.posLam = A.rcdbl[k].p, w.aposLam = A.acdbl.p;
      D4* m = A.rman[k].p;
      w.geo = m, w.lam0 = m + 5 * (size_t)nm, w.lam = m + 6 * (size_t)nm, w.vn = m + 7 * (size_t)nm;
      D4* am = A.aman.p;
      w.ageo = am, w.alam = am + 5 * (size_t)nm, w.avn = am + 6 * (size_t)nm, w.ath = am + 7 * (size_t)nm;
      w.alamOut = am + 8 * (size_t)nm, w.alamPrev = am + 9 * (size_t)nm;
      w.np = A.rmint[k].p, w.src = A.rmint[k].p + nm;
      w.posIn = A.rmdbl[k].p;
      w.aposIn = A.amdbl.p, w.aposOut = A.amdbl.p + nm, w.aposPrev = A.amdbl.p + 2 * nm;
      w.alL = A.alLB.p, w.apL = A.ldbl.p;
      w.tv = A.tv[k].p, w.tp = A.tp[k].p;
      w.theta = A.small.p, w.err = A.small.p + 4;
      w.hash = nullptr;
    }
  }

  static void replay(cudaStream_t st, const XScene& sc, const XRec& R, const XView& r, const XWork& w,
                     const XRec* next, int tag) {
    const int n = sc.n;
    const int gn = gridFor(n), gc = gridFor(std::max(R.nc, 1)), gm = gridFor(std::max(R.nm, 1));
    const double gMag = std::sqrt(sc.g.x * sc.g.x + sc.g.y * sc.g.y + sc.g.z * sc.g.z);
    const double vRest = 2.0 * sc.dt * gMag;  // src/sim.hpp:206, :282 (both loops)
    kxPredict<<<gn, kB, 0, st>>>(sc, r, w);
    if (R.nc > 0)
      kxContacts<<<gc, kB, 0, st>>>(sc, r, w);
    if (R.nm > 0) {
      kxManifolds<<<gm, kB, 0, st>>>(sc, r, w);
      kxGather<<<gm, kB, 0, st>>>(sc, r, w);
      kxVn0<<<gm, kB, 0, st>>>(sc, r, w);
      for (int c = 0; c < R.ncolV; ++c)
        kxWarm<<<gm, kB, 0, st>>>(sc, r, w, c);
      if (!(R.nm <= kClusterEntries && R.ncolV > 0 &&
            launchOneCluster(kxPgsCluster, kClusterBlocks, kB, st, sc, r, w, R.velSweeps, R.stabSweeps, vRest, tag))) {
        for (int it = 0; it < R.velSweeps; ++it)
          for (int c = 0; c < R.ncolV; ++c)
            kxPgs<<<gm, kB, 0, st>>>(sc, r, w, c, it, vRest, 0, tag);
        for (int it = 0; it < R.stabSweeps; ++it)
          for (int c = 0; c < R.ncolV; ++c)
            kxPgs<<<gm, kB, 0, st>>>(sc, r, w, c, R.velSweeps + it, vRest, 1, tag);
      }
    }
    kxIntegrate<<<gn, kB, 0, st>>>(sc, r, w);
    if (R.nc > 0) {
      cudaCheck(cudaMemsetAsync(w.posLam, 0, R.nc * sizeof(double), st), "memset");
      for (int it = 0; it < R.posSweeps; ++it)
        for (int c = 0; c < R.ncolP; ++c)
          kxPos<<<gc, kB, 0, st>>>(sc, r, w, c, it, tag);
    }
    if (next)
      kxCheck<<<gn, kB, 0, st>>>(sc, view(*next), w);
    cudaCheck(cudaGetLastError(), "xadj replay");
  }

  static void pgsRevLaunch(const XAdj& A, int grid, cudaStream_t st, const XScene& sc, const XView& r, const XWork& w,
                           int c, int sweep, double vRest, int stab) {
    if (A.dualCheck)
      kxPgsRev<1><<<grid, kBR, 0, st>>>(sc, r, w, c, sweep, vRest, stab);
    else
      kxPgsRev<0><<<gridFor(std::max(r.nm, 1), kBPgs), kBPgs, 0, st>>>(sc, r, w, c, sweep, vRest, stab);
  }
  static void reverse(S& s, const XAdj& A, const XScene& sc, const XRec& R, const XView& r, const XWork& w) {
    cudaStream_t st = s.stream_;
    const int n = sc.n;
    const int gn = gridFor(n), gc = gridFor(std::max(R.nc, 1)), gm = gridFor(std::max(R.nm, 1));
    const double gMag = std::sqrt(sc.g.x * sc.g.x + sc.g.y * sc.g.y + sc.g.z * sc.g.z);
    const double vRest = 2.0 * sc.dt * gMag;
    // the grouped reverse kernels: kGroup threads an entry
    const int gnG = gridFor((long)kGroup * n, kBR), gcG = gridFor((long)kGroup * std::max(R.nc, 1), kBR),
              gmG = gridFor((long)kGroup * std::max(R.nm, 1), kBR);
    kxRevInit<<<gridFor(std::max(n, std::max(R.nc, R.nm))), kB, 0, st>>>(sc, r, w);
    if (R.nc > 0)
      for (int it = R.posSweeps - 1; it >= 0; --it)
        for (int c = R.ncolP - 1; c >= 0; --c)
          if (A.dualCheck)
            kxPosRev<<<gcG, kBR, 0, st>>>(sc, r, w, c, it);
          else
            kxPosRevH<<<gridFor(std::max(R.nc, 1), kBPgs), kBPgs, 0, st>>>(sc, r, w, c, it);
    kxIntegrateRev<<<gnG, kBR, 0, st>>>(sc, r, w);
    if (R.nm > 0) {
      if (!(!A.dualCheck && R.nm <= kClusterEntries && R.ncolV > 0 &&
            launchOneCluster(kxPgsRevCluster, kClusterBlocks, kB, st, sc, r, w, R.velSweeps, R.stabSweeps, vRest))) {
        for (int it = R.stabSweeps - 1; it >= 0; --it)
          for (int c = R.ncolV - 1; c >= 0; --c)
            pgsRevLaunch(A, gm, st, sc, r, w, c, R.velSweeps + it, vRest, 1);
        for (int it = R.velSweeps - 1; it >= 0; --it)
          for (int c = R.ncolV - 1; c >= 0; --c)
            pgsRevLaunch(A, gm, st, sc, r, w, c, it, vRest, 0);
      }
      if (A.dualCheck) {
        for (int c = 0; c < R.ncolV; ++c)
          kxWarmRev<<<gmG, kBR, 0, st>>>(sc, r, w, c);
        for (int c = 0; c < R.ncolV; ++c)
          kxVn0Rev<<<gmG, kBR, 0, st>>>(sc, r, w, c);
      } else {
        kxWarmRevH<<<gridFor(std::max(R.nm, 1), kBPgs), kBPgs, 0, st>>>(sc, r, w);
        kxVn0RevH<<<gridFor(std::max(R.nm, 1), kBPgs), kBPgs, 0, st>>>(sc, r, w);
      }
      if (R.L > 0) {
        cudaCheck(cudaMemsetAsync(w.alL, 0, R.L * sizeof(D4), st), "memset");
        cudaCheck(cudaMemsetAsync(w.apL, 0, R.L * sizeof(double), st), "memset");
      }
      kxGatherRev<<<gm, kB, 0, st>>>(sc, r, w);
      kxThetaSum<<<std::min(gm, 64), kB, 0, st>>>(r, w);
    }
    if (R.nc > 0) {
      kxManifoldRev<<<gcG, kBR, 0, st>>>(sc, r, w);
      kxContactRev<<<gcG, kBR, 0, st>>>(sc, r, w);
    }
    kxPredictRev<<<gnG, kBR, 0, st>>>(sc, r, w);
    cudaCheck(cudaGetLastError(), "xadj reverse");
  }

  static void backward(S& s, const double* gx, const double* gq, const double* gv, const double* gw, double* dx,
                       double* dq, double* dv, double* dw, double* dtheta) {
    XAdj& A = get(s);
    if (A.recs.empty())
      throw std::invalid_argument("XPBD adjoint: nothing recorded (xa_begin, then xa_step)");
    checkScope(s);
    if (A.n > 0)
      deviceRows({gx, gq, gv, gw, dx, dq, dv, dw});
    cudaStream_t st = s.stream_;
    const XScene sc = scene(s, A);
    XWork W[2];
    work(s, A, W);
    if (!A.side) {
      cudaCheck(cudaStreamCreateWithFlags(&A.side, cudaStreamNonBlocking), "xadj stream");
      for (cudaEvent_t* e : {&A.evStart, &A.evRep[0], &A.evRep[1], &A.evRev[0], &A.evRev[1]})
        cudaCheck(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "xadj event");
    }
    cudaStream_t sb = A.side;
    XWork& w0 = W[0];
    const int n = A.n;
    if (n > 0) {
      kxPack<<<gridFor(n), kB, 0, st>>>(n, gx, 3, w0.gx);
      kxPack<<<gridFor(n), kB, 0, st>>>(n, gq, 4, w0.gq);
      kxPack<<<gridFor(n), kB, 0, st>>>(n, gv, 3, w0.gv);
      kxPack<<<gridFor(n), kB, 0, st>>>(n, gw, 3, w0.gw);
    }
    cudaCheck(cudaMemsetAsync(A.small.p, 0, 8 * sizeof(double), st), "memset");
    // the last substep's ledger output feeds nothing
    const int T = (int)A.recs.size();
    cudaCheck(cudaMemsetAsync(w0.alamOut, 0, std::max(A.recs[T - 1]->nm, 1) * sizeof(D4), st), "memset");
    cudaCheck(cudaMemsetAsync(w0.aposOut, 0, std::max(A.recs[T - 1]->nm, 1) * sizeof(double), st), "memset");
    // the replay of substep t - 1 runs on the side stream beside the reverse of substep t: a replay
    // reads only the record, and replay buffer set t % 2 serves substep t; the side stream waits
    // until the reverse that last used a set is done before it replays into it
    cudaCheck(cudaEventRecord(A.evStart, st), "event");
    cudaCheck(cudaStreamWaitEvent(sb, A.evStart, 0), "event");
    auto replayOn = [&](int t) {
      const XRec& R = *A.recs[t];
      replay(sb, sc, R, view(R), W[t & 1], t + 1 < T ? A.recs[t + 1].get() : nullptr, t);
      cudaCheck(cudaEventRecord(A.evRep[t & 1], sb), "event");
    };
    replayOn(T - 1);
    for (int t = T - 1; t >= 0; --t) {
      const int k = t & 1;
      XWork& w = W[k];
      if (t >= 1) {
        if (t + 1 <= T - 1)
          cudaCheck(cudaStreamWaitEvent(sb, A.evRev[k ^ 1], 0), "event");
        replayOn(t - 1);
      }
      cudaCheck(cudaStreamWaitEvent(st, A.evRep[k], 0), "event");
      const XRec& R = *A.recs[t];
      const XView r = view(R);
      reverse(s, A, sc, R, r, w);
      if (t > 0) {
        const XRec& P = *A.recs[t - 1];
        const size_t pm = std::max(P.nm, 1);
        cudaCheck(cudaMemsetAsync(w.alamPrev, 0, pm * sizeof(D4), st), "memset");
        cudaCheck(cudaMemsetAsync(w.aposPrev, 0, pm * sizeof(double), st), "memset");
        if (R.L > 0)
          kxLedgerMap<<<gridFor(R.L), kB, 0, st>>>(r, view(P), w);
        std::swap(w.alamOut, w.alamPrev);
        std::swap(w.aposOut, w.aposPrev);
      }
      // the start adjoint of this substep is the end adjoint of the previous one
      std::swap(w.gx, w.ax);
      std::swap(w.gq, w.aq);
      std::swap(w.gv, w.av);
      std::swap(w.gw, w.aw);
      // both sets share the adjoint buffers
      XWork& o = W[k ^ 1];
      o.gx = w.gx, o.gq = w.gq, o.gv = w.gv, o.gw = w.gw, o.ax = w.ax, o.aq = w.aq, o.av = w.av, o.aw = w.aw;
      o.alamOut = w.alamOut, o.alamPrev = w.alamPrev, o.aposOut = w.aposOut, o.aposPrev = w.aposPrev;
      cudaCheck(cudaEventRecord(A.evRev[k], st), "event");
      cudaCheck(cudaGetLastError(), "xadj backward");
    }
    XWork& w = W[0];
    if (n > 0) {
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, w.gx, 3, dx);
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, w.gq, 4, dq);
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, w.gv, 3, dv);
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, w.gw, 3, dw);
    }
    double h[8];
    cudaCheck(cudaMemcpyAsync(h, A.small.p, sizeof h, cudaMemcpyDeviceToHost, st), "D2H");
    cudaCheck(cudaStreamSynchronize(sb), "xadj side stream");
    s.sync();
    dtheta[0] = h[0], dtheta[1] = h[1], dtheta[2] = h[2];
    A.err[0] = h[4], A.err[1] = h[5];
  }

  static void state(S& s, double* x, double* q, double* v, double* w) {
    cudaStream_t st = s.stream_;
    const int n = s.numReal_;
    if (n > 0)
      deviceRows({x, q, v, w});
    if (n > 0) {
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, s.pos_.p, 3, x);
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, s.quat_.p, 4, q);
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, s.vel_.p, 3, v);
      kxUnpack<<<gridFor(n), kB, 0, st>>>(n, s.angVel_.p, 3, w);
      cudaCheck(cudaGetLastError(), "xadj state");
    }
    s.sync();
  }

  // the branch signature of the recorded rollout: every substep replayed (no reverse), the branch
  // decisions of every sweep update hashed
  static unsigned long long branches(S& s) {
    XAdj& A = get(s);
    if (A.recs.empty())
      throw std::invalid_argument("XPBD adjoint: nothing recorded (xa_begin, then xa_step)");
    checkScope(s);
    cudaStream_t st = s.stream_;
    const XScene sc = scene(s, A);
    XWork W[2];
    work(s, A, W);
    XWork& w = W[0];
    A.hashBuf.ensure(1, false, st);
    cudaCheck(cudaMemsetAsync(A.hashBuf.p, 0, sizeof(u64), st), "memset");
    w.hash = A.hashBuf.p;
    const int T = (int)A.recs.size();
    for (int t = 0; t < T; ++t) {
      const XRec& R = *A.recs[t];
      replay(st, sc, R, view(R), w, nullptr, t);
    }
    u64 h = 0;
    cudaCheck(cudaMemcpyAsync(&h, A.hashBuf.p, sizeof h, cudaMemcpyDeviceToHost, st), "D2H");
    s.sync();
    return h;
  }
  static long signature(S& s, long* out, long cap) {
    XAdj& A = get(s);
    long k = 0;
    for (auto& r : A.recs) {
      const long v[7] = {r->nc, r->nm, r->ncolV, r->ncolP, r->velSweeps, r->stabSweeps, r->posSweeps};
      for (long j = 0; j < 7; ++j, ++k)
        if (k < cap)
          out[k] = v[j];
    }
    return (long)A.recs.size();
  }
  static void info(S& s, long* out, double* err) {
    XAdj& A = get(s);
    size_t bytes = 0;
    for (auto& r : A.recs)
      bytes += r->bytes();
    out[0] = (long)A.recs.size();
    out[1] = (long)bytes;
    out[2] = (long)A.workBytes;
    out[3] = A.maxSweeps;
    err[0] = A.err[0];
    err[1] = A.err[1];
  }
};

void xadjBegin(Sim<double>& S, const double* x, const double* q, const double* v, const double* w, int n) {
  XAdjAccess::begin(S, x, q, v, w, n);
}
void xadjStep(Sim<double>& S, double dt, int substeps) { XAdjAccess::step(S, dt, substeps); }
void xadjState(Sim<double>& S, double* x, double* q, double* v, double* w) { XAdjAccess::state(S, x, q, v, w); }
void xadjBackward(Sim<double>& S, const double* gx, const double* gq, const double* gv, const double* gw, double* dx,
                  double* dq, double* dv, double* dw, double* dtheta) {
  XAdjAccess::backward(S, gx, gq, gv, gw, dx, dq, dv, dw, dtheta);
}
void xadjInfo(Sim<double>& S, long* out, double* err) { XAdjAccess::info(S, out, err); }
long xadjSignature(Sim<double>& S, long* out, long cap) { return XAdjAccess::signature(S, out, cap); }
unsigned long long xadjBranches(Sim<double>& S) { return XAdjAccess::branches(S); }

}  // namespace pdem
