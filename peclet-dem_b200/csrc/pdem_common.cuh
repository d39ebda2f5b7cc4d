// Shared device-side definitions of the B200 substep: the device view of the simulation state
// (`Dev<R>`), counters, launch geometry and order-preserving atomics.
//
// Layout in HBM (structure of arrays, one aligned 4-wide record per particle field so one field
// of one body is one 16 B / 32 B load):
//   particles [capacity]:   pos, vel, angVel, invI, posPred, velPred, angVelPred, quat, quatPred,
//                           extForce, dVel, dAngVel, dPos (Q4<R>); invMass, scale, targetScale, rad
//                           (R); shapeId, realIdx, counts (int); planeFric (2 R); grounded, matId (u8)
//   pairs [maxPairs]:       int2 (i, j), sorted by (i, j)
//   contacts [maxContacts]: cab int2 (bodyA, bodyB); cn = normal|dist, crA = rA|lambdaN,
//                           crB = rB|restitution, cbv = wall velocity|friction (Q4<R>)
//   manifolds [maxContacts]: mab int2; mnp int; mN = Nsum|restitution_sum, mTA = TauA|friction_sum,
//                           mTB, mrA, mrB, mwv (Q4<R>)
// Every cross-thread accumulation that the reference performs with atomics is done here in the
// canonical order (ascending source index) with prefix sums and owner-computes gathers, so the
// result is deterministic and matches the serial reference; only order-free reductions (max of
// non-negative values, integer counts) use atomics.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "pdem_math.cuh"

namespace pdem {

using u64 = unsigned long long;

constexpr int kMaxMaterials = 8;
constexpr int kHertzMaxWalls = 4;
constexpr int kMaxPlanes = 8;
constexpr int kNumSMs = 148;
constexpr int kBlock = 256;

// device-resident counters and loop-control flags of one substep
template <class R>
struct Counters {
  int pairCount;      // candidate pairs found (may exceed capacity: host grows and re-runs)
  int contactTotal;   // contacts wanted (before the capacity clamp)
  int contactCount;   // contacts stored
  int manifoldCount;
  int topGhost;       // numReal + ghosts stored
  int ghostWanted;
  int remaining;      // colouring: entries still uncoloured after the last round
  int maxColor;       // colouring: max colour (INT_MIN identity)
  int leftover;       // colouring: entries left uncoloured
  int velDone;        // adaptive stop reached in the main velocity loop
  int stabRun;        // stabilization pass triggered
  int stabDone;       // adaptive stop reached in the stabilization loop
  int posDone;        // adaptive stop reached in the position loop
  int hzCand;         // Hertz wall candidates wanted
  int hzRebuild;      // Hertz: displacement check asks for a pair-list rebuild
  int err;            // bit flags: a bounded loop hit its iteration limit (1 = BVH traversal/build)
  int velSweeps;      // sweeps executed this substep (main velocity loop)
  int stabSweeps;     // sweeps executed this substep (stabilization loop)
  int posSweeps;      // sweeps executed this substep (position loop)
  int pad2;
  R maxOverlap;
  R maxApproach;
  R hzMaxDisp2;
  R pad1;
};

// Batched form: several independent scenes in one body array (scene s = bodies
// [sceneFirst[s], sceneFirst[s + 1])). Each scene keeps the reference's own loop state and
// parameters, so it steps exactly as it would alone; this record holds them per scene.
template <class R>
struct SceneCtl {
  R maxOverlap, maxApproach;  // as the Counters fields, per scene
  R margin, eN, mu, pad;      // contact margin (0.1 x the scene's largest radius), restitution, friction
  int velDone, stabRun, stabDone, posDone;
  int velSweeps, stabSweeps, posSweeps, pad2;
};

// polls before a grid-barrier wait of a persistent loop gives up (seconds at any back-off: each
// poll is an L2 round trip)
constexpr long kBarrierSpins = 1L << 26;

// colour-ordered records of the coloured velocity sweeps (layout and packing in pdem_solve.cuh,
// kPackPgs): kPgsSlots slots of 4 values per entry, slot-major, and the entry's ids
constexpr int kPgsSlots = 11;
template <class R>
struct PgsRecs {
  Q4<R>* q;
  int4* ids;
  long cap;
};

template <class R>
struct Dev {
  int cap = 0, maxPairs = 0, maxContacts = 0;
  Q4<R> *pos = nullptr, *vel = nullptr, *angVel = nullptr, *invI = nullptr, *posPred = nullptr,
        *velPred = nullptr, *angVelPred = nullptr, *quat = nullptr, *quatPred = nullptr,
        *extForce = nullptr, *dVel = nullptr, *dAngVel = nullptr, *dPos = nullptr;
  R *invMass = nullptr, *scale = nullptr, *targetScale = nullptr, *rad = nullptr, *planeFric = nullptr;
  int *shapeId = nullptr, *realIdx = nullptr, *counts = nullptr;
  uint8_t *grounded = nullptr, *matId = nullptr;
  long long* winner = nullptr;
  u64* mask = nullptr;
  int2* pairs = nullptr;
  // contacts
  int2* cab = nullptr;
  Q4<R> *cn = nullptr, *crA = nullptr, *crB = nullptr, *cbv = nullptr;
  int *cColor = nullptr, *cSlot = nullptr;
  R* posLamC = nullptr;
  // manifolds
  int2* mab = nullptr;
  int* mnp = nullptr;
  Q4<R> *mN = nullptr, *mTA = nullptr, *mTB = nullptr, *mrA = nullptr, *mrB = nullptr, *mwv = nullptr;
  int* mColor = nullptr;
  u64 *pairKeys = nullptr, *prevKeys = nullptr;
  uint8_t *persistent = nullptr, *sideFlags = nullptr;
  R *lambda = nullptr, *prevLambda = nullptr, *vn0 = nullptr, *posImp = nullptr, *prevPosImp = nullptr;
  Q4<R> *lambdaT = nullptr, *prevLambdaT = nullptr, *vt0 = nullptr;
  // static geometry
  const ShapeDesc<R>* shapes = nullptr;
  const Q4<R>* shell = nullptr;
  const R* sdfGrid = nullptr;
  const PlaneDesc<R>* planes = nullptr;
  const WallDesc<R>* walls = nullptr;
  const R* wallGrid = nullptr;
  const R* pairMat = nullptr;  // null = feature off
  const R *hzE = nullptr, *hzNu = nullptr;
  Counters<R>* ctr = nullptr;
  // batched form (all null / 1 for a single scene)
  int numScenes = 1;
  const int* sceneOf = nullptr;        // [real bodies] scene of each body
  SceneCtl<R>* scn = nullptr;          // [numScenes]
  const int* sceneWallOff = nullptr;   // [numScenes + 1] walls of scene s: sceneWallIdx[off[s] .. off[s + 1])
  const int* sceneWallIdx = nullptr;
  const int* sceneManFirst = nullptr;  // [numScenes + 1] first manifold of each scene
  const int* sceneConFirst = nullptr;  // [3 (numScenes + 1)] first pair / plane / wall contact of each scene
  const int* sceneLeafFirst = nullptr; // [numScenes + 1] first BVH leaf (sorted position) of each scene
};

// scene of body i (0 for a single scene)
template <class R>
__device__ __forceinline__ int sceneOfBody(const Dev<R>& d, int i) {
  return d.sceneOf ? d.sceneOf[i] : 0;
}
// scene-local index of manifold m / contact c (the index the scene would have alone): the colour
// priorities of the batched form are those of each scene stepped alone
template <class R>
__device__ __forceinline__ int localManifold(const Dev<R>& d, int m, int s) {
  return d.sceneManFirst ? m - d.sceneManFirst[s] : m;
}
template <class R>
__device__ __forceinline__ int localContact(const Dev<R>& d, int c, int s) {
  if (!d.sceneConFirst)
    return c;
  const int S = d.numScenes;
  const int* P = d.sceneConFirst;               // pair contacts: P[0..S], region end P[S]
  const int* Q = d.sceneConFirst + (S + 1);     // plane contacts: Q[0..S]
  const int* W = d.sceneConFirst + 2 * (S + 1); // wall contacts: W[0..S]
  if (c < P[S])
    return c - P[s];
  if (c < Q[S])
    return (P[s + 1] - P[s]) + (c - Q[s]);
  return (P[s + 1] - P[s]) + (Q[s + 1] - Q[s]) + (c - W[s]);
}

// ---- launch geometry: grid-stride loops over a device-resident count ----
inline int gridFor(long n, int block = kBlock) {
  long b = (n + block - 1) / block;
  if (b < 1)
    b = 1;
  if (b > kNumSMs * 32)
    b = kNumSMs * 32;
  return (int)b;
}
#define GRID_STRIDE(i, n) \
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (long)(n); i += (long)gridDim.x * blockDim.x)

// ---- max of non-negative values via ordered integer bits (order-free, NaN ignored) ----
__device__ __forceinline__ void atomicMaxNonNeg(double* p, double v) {
  if (v > 0.0)
    atomicMax(reinterpret_cast<unsigned long long*>(p), (unsigned long long)__double_as_longlong(v));
}
__device__ __forceinline__ void atomicMaxNonNeg(float* p, float v) {
  if (v > 0.0f)
    atomicMax(reinterpret_cast<unsigned int*>(p), (unsigned int)__float_as_int(v));
}

// Order-free max of non-negative values with one atomic per warp: every lane of the warp must
// call it (after its grid-stride loop). Lanes carry their own running max (0 when nothing).
template <class R>
__device__ __forceinline__ void warpMaxAtomic(R* p, R v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const R w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  if ((threadIdx.x & 31) == 0)
    atomicMaxNonNeg(p, v);
}
// the same, reduced over the block first: one atomic per block instead of one per warp, for maxima
// that every warp contributes to (thousands of same-address atomics serialise at L2). Every thread
// of the block must call it.
template <class R>
__device__ __forceinline__ void blockMaxAtomic(R* p, R v) {
  __shared__ R sMax[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const R w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  __syncthreads();  // a previous call's reads of sMax are done
  if ((threadIdx.x & 31) == 0)
    sMax[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    R m = sMax[0];
    for (int k = 1; k < (int)((blockDim.x + 31) >> 5); ++k)
      m = sMax[k] > m ? sMax[k] : m;
    atomicMaxNonNeg(p, m);
  }
}
// running max that ignores NaN (the reference's atomic max never stores NaN)
template <class R>
__device__ __forceinline__ void runMax(R& acc, R v) {
  if (v > acc)
    acc = v;
}

}  // namespace pdem
