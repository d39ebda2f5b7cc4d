// Persistent loops: the Jones-Plassmann colouring rounds and the coloured Gauss-Seidel sweep loops
// of the substep, each run as ONE cooperative launch whose blocks are all resident and step
// through rounds / colours / sweeps together behind a grid-wide barrier. Per-colour and per-round
// launches (and the host read-back after every colouring round) become barrier crossings of a
// microsecond or two. The work done per colour, per sweep and per round, and its order, is exactly
// that of the per-colour kernels (pdem_solve.cuh) and per-round kernels (pdem_contact.cuh).
#pragma once
#include "pdem_contact.cuh"
#include "pdem_solve.cuh"

namespace pdem {

// polls before a barrier wait gives up (seconds at any back-off: each poll is an L2 round trip)
constexpr long kBarrierSpins = 1L << 26;
constexpr int kErrBarrier = 2;  // Counters::err bit: a grid barrier timed out

// word[0] = arrivals, word[1] = generation; both zero before the launch; sleepNs = the back-off
// of a waiting block between polls of the generation
struct GridBar {
  unsigned* word;
  int* err;
  unsigned sleepNs;
};

// Grid-wide barrier of a cooperative launch (all blocks co-resident). Thread 0 of each block
// arrives; the last arrival resets the counter and advances the generation; the others wait for
// the generation to move, bounded. Fences on both sides order every block's writes before the
// barrier with every block's reads after it. Returns false (and sets the error bit) on time-out;
// the caller then returns.
__device__ __forceinline__ bool gridBarrier(const GridBar& gb) {
  __shared__ int sOk;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = gb.word + 1;
    const unsigned g = *gen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(gb.word, 1u) == gridDim.x - 1) {
      atomicExch(gb.word, 0u);
      __threadfence();
      atomicAdd(gb.word + 1, 1u);
    } else {
      long spins = 0;
      while (*gen == g) {
        if (++spins > kBarrierSpins) {
          atomicOr(gb.err, kErrBarrier);
          ok = 0;
          break;
        }
        if (gb.sleepNs)
          __nanosleep(gb.sleepNs);
      }
    }
    __threadfence();
    sOk = ok;
  }
  __syncthreads();
  return sOk != 0;
}

// ---------------------------------------------------------------------------------------------
// Coloured sweep loop. KIND 0: projected GS velocity sweep (pgsOne), 1: one-shot GS velocity
// sweep (gsOne), 2: position sweep (posGSOne). LOOP selects the control flags: 1 main velocity
// loop, 2 stabilization loop, 3 position loop. The host has already run the first sweep's BEGIN
// (kCtl): each END here is fused with the next sweep's BEGIN.
template <class R, int KIND, int LOOP>
__global__ void __launch_bounds__(kBlock) kSweepLoop(Dev<R> d, const int* order, const int* coff, int ncol, int iters,
                                                     SolveP<R> P, R thr, GridBar gb) {
  Counters<R>* c = d.ctr;
  volatile int* done = LOOP == 1 ? &c->velDone : LOOP == 2 ? &c->stabDone : &c->posDone;
  int* sweeps = LOOP == 1 ? &c->velSweeps : LOOP == 2 ? &c->stabSweeps : &c->posSweeps;
  R* mxp = KIND == 2 ? &c->maxOverlap : &c->maxApproach;
  const bool lead = (blockIdx.x | threadIdx.x) == 0;
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x, gstride = (long)gridDim.x * blockDim.x;
  if (*done)
    return;
  for (int it = 0; it < iters; ++it) {
    R mx = R(0);
    for (int col = 0; col < ncol; ++col) {
      const int b = coff[col], n = coff[col + 1] - b;
      // colour 62 is where the 62-colour mask saturates: not an independent set, so one thread
      // runs it in manifold order, as the reference's serial sweep does
      const bool serial = col >= kSaturatedColor;
      if (!serial || lead)
        for (long t = serial ? 0 : gtid; t < n; t += serial ? 1 : gstride) {
          if (KIND == 0)
            pgsOne(d, order[b + t], P, mx, LOOP);
          else if (KIND == 1)
            gsOne(d, order[b + t], P, mx);
          else
            posGSOne(d, order[b + t], mx);
        }
      if (col == ncol - 1)
        warpMaxAtomic(mxp, mx);
      if (!gridBarrier(gb))
        return;
    }
    // END of this sweep, then BEGIN of the next one
    if (d.scn) {  // batched form: every scene's own END/BEGIN; done when all scenes are
      if (blockIdx.x == 0) {
        int notDone = 0;
        for (int s = threadIdx.x; s < d.numScenes; s += blockDim.x) {
          SceneCtl<R>& q = d.scn[s];
          volatile int* dn = LOOP == 1 ? &q.velDone : LOOP == 2 ? &q.stabDone : &q.posDone;
          volatile R* m = KIND == 2 ? &q.maxOverlap : &q.maxApproach;
          if (!*dn) {
            const R mv = *m;
            if (KIND == 2 ? (mv < thr) : (mv <= thr)) {
              *dn = 1;
            } else if (it + 1 < iters) {
              *m = R(0);
              (LOOP == 1 ? q.velSweeps : LOOP == 2 ? q.stabSweeps : q.posSweeps) += 1;
            }
          }
          notDone |= !*dn;
        }
        notDone = __syncthreads_or(notDone);
        if (threadIdx.x == 0 && !notDone)
          *done = 1;
      }
    } else if (lead) {
      const R m = *reinterpret_cast<volatile R*>(mxp);
      const bool stop = KIND == 2 ? (m < thr) : (m <= thr);
      if (stop) {
        *done = 1;
      } else if (it + 1 < iters) {
        *reinterpret_cast<volatile R*>(mxp) = R(0);
        *sweeps += 1;
      }
    }
    if (!gridBarrier(gb))
      return;
    if (*done)
      break;
  }
}

// ---------------------------------------------------------------------------------------------
// Batched form: the same sweep loop with ONE BLOCK PER SCENE. A scene's colour classes are
// contiguous in the (scene, colour)-sorted order (off[s * 64 + c] .. off[s * 64 + c + 1]); its
// blocks-worth of threads sweeps them in colour order with block barriers, and the block ends its
// own loop at the scene's adaptive stop. No grid-wide barrier and no cooperative launch: scenes are
// independent. The host has run the first sweep's BEGIN for every scene (kCtlScenes).
constexpr int kSceneBlock = 128;      // default block of the per-scene sweep loops
constexpr int kSceneBlockMax = 512;   // largest block the launch shape autotuner tries

template <class R, int KIND, int LOOP>
__global__ void __launch_bounds__(kSceneBlockMax) kSweepScenes(Dev<R> d, const int* order, const int* off, int iters,
                                                            SolveP<R> P, R thr) {
  const int s = blockIdx.x;
  SceneCtl<R>& q = d.scn[s];
  volatile int* done = LOOP == 1 ? &q.velDone : LOOP == 2 ? &q.stabDone : &q.posDone;
  volatile R* mxp = KIND == 2 ? &q.maxOverlap : &q.maxApproach;
  if (*done)
    return;
  const int* so = off + (long)s * 64;
  for (int it = 0; it < iters; ++it) {
    R mx = R(0);  // unused: batched entries take their scene's max atomically (loopMax)
    for (int col = 0; col < 63; ++col) {
      const int b = so[col], n = so[col + 1] - b;
      if (n == 0)
        continue;  // uniform over the block
      const bool serial = col >= kSaturatedColor;
      if (!serial || threadIdx.x == 0)
        for (int t = serial ? 0 : threadIdx.x; t < n; t += serial ? 1 : blockDim.x) {
          if (KIND == 0)
            pgsOne(d, order[b + t], P, mx, LOOP);
          else if (KIND == 1)
            gsOne(d, order[b + t], P, mx);
          else
            posGSOne(d, order[b + t], mx);
        }
      __syncthreads();
    }
    // END of this sweep, then BEGIN of the next one (kCtlScenes' rule for this scene)
    if (threadIdx.x == 0) {
      const R m = *mxp;
      if (KIND == 2 ? (m < thr) : (m <= thr)) {
        *done = 1;
      } else if (it + 1 < iters) {
        *mxp = R(0);
        (LOOP == 1 ? q.velSweeps : LOOP == 2 ? q.stabSweeps : q.posSweeps) += 1;
      }
    }
    __syncthreads();
    if (*done)
      break;
  }
}

constexpr int kColorBlock = 1024;  // one large block per SM: fewer arrivals per grid barrier

// ---------------------------------------------------------------------------------------------
// Both colourings of a substep in ONE cooperative launch: the manifold graph (velocity solve) and
// the contact graph (position solve) are independent, so their Jones-Plassmann rounds run in
// lockstep behind the same grid barriers, each graph stopping on its own. The initialisation
// (masks, colours, first winner array, counters) is the kernel's first phase. Per graph the
// rounds, the winners and the statistics are exactly those of kColorLoop.
struct ColorJob {
  int ne, nb;          // entries, bodies
  int* col;            // [ne] colours out
  long long *winA, *winB;
  u64* mask;           // [nb]
  int* aux;            // [0..2] remaining counts by round % 3, [3] max colour, [4] left uncoloured
};

template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorInit(const Dev<R>& d, const ColorJob& J, long gtid, long gstride) {
  if (J.ne <= 0)
    return;  // a kept (or empty) graph: its colours and statistics stay as they are
  for (long b = gtid; b < J.nb; b += gstride) {
    J.mask[b] = 0ull;
    J.winA[b] = -1ll;
  }
  for (long i = gtid; i < J.ne; i += gstride) {
    if (MANIFOLD) {
      const int2 ab = d.mab[i];
      J.col[i] = (d.mnp[i] <= 0 || (ab.y >= 0 && d.realIdx[ab.x] > d.realIdx[ab.y])) ? -2 : -1;
    } else {
      J.col[i] = -1;
    }
  }
  if (gtid == 0) {
    J.aux[0] = J.aux[1] = J.aux[2] = 0;
    J.aux[3] = INT_MIN;
    J.aux[4] = 0;
  }
}
template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorContend(const Dev<R>& d, const ColorJob& J, int round, long gtid,
                                             long gstride) {
  long long* win = (round & 1) ? J.winB : J.winA;
  if (gtid == 0)
    J.aux[(round + 1) % 3] = 0;
  for (long i = gtid; i < J.ne; i += gstride) {
    if (J.col[i] != -1)
      continue;
    int ea, eb;
    colorEnds<R, MANIFOLD>(d, (int)i, ea, eb);
    const long long k = entryKey<R, MANIFOLD>(d, (int)i, ea);
    atomicMax(&win[ea], k);
    if (eb >= 0)
      atomicMax(&win[eb], k);
  }
}
template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorCommit(const Dev<R>& d, const ColorJob& J, int round, long gtid,
                                            long gstride) {
  long long* win = (round & 1) ? J.winB : J.winA;
  long long* nxt = (round & 1) ? J.winA : J.winB;
  int lost = 0;
  for (long i = gtid; i < J.ne; i += gstride) {
    if (J.col[i] != -1)
      continue;
    int ea, eb;
    colorEnds<R, MANIFOLD>(d, (int)i, ea, eb);
    const long long k = entryKey<R, MANIFOLD>(d, (int)i, ea);
    if (win[ea] != k || (eb >= 0 && win[eb] != k)) {
      ++lost;
      nxt[ea] = -1;
      if (eb >= 0)
        nxt[eb] = -1;
      continue;
    }
    u64 forb = J.mask[ea];
    if (eb >= 0)
      forb |= J.mask[eb];
    int cc = 0;
    while (cc < 62 && (forb & (1ull << cc)))
      ++cc;
    J.col[i] = cc;
    J.mask[ea] |= 1ull << cc;
    if (eb >= 0)
      J.mask[eb] |= 1ull << cc;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    lost += __shfl_xor_sync(0xffffffffu, lost, o);
  if ((threadIdx.x & 31) == 0 && lost)
    atomicAdd(&J.aux[round % 3], lost);
}
__device__ __forceinline__ void colorStats(const ColorJob& J, long gtid, long gstride) {
  int mxc = INT_MIN, left = 0;
  for (long i = gtid; i < J.ne; i += gstride) {
    const int v = J.col[i];
    mxc = v > mxc ? v : mxc;
    left += (v == -1) ? 1 : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int w = __shfl_xor_sync(0xffffffffu, mxc, o);
    mxc = w > mxc ? w : mxc;
    left += __shfl_xor_sync(0xffffffffu, left, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (mxc != INT_MIN)
      atomicMax(&J.aux[3], mxc);
    if (left)
      atomicAdd(&J.aux[4], left);
  }
}

// job 0: manifolds over real bodies (skipped when ne = 0), job 1: contacts over body slots
// reuse: a graph equal to the previous substep's keeps its colours and statistics (differ[0]: the
// contact list changed, differ[1]: the manifold list changed; reuse = 0 forces both colourings)
template <class R>
__global__ void __launch_bounds__(kColorBlock) kColorBoth(Dev<R> d, ColorJob jm, ColorJob jc, int maxRounds,
                                                          GridBar gb, const int* differ, int reuse) {
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x, gstride = (long)gridDim.x * blockDim.x;
  if (reuse && !differ[1])
    jm.ne = 0;  // uniform over the grid: the flags are written before the launch
  if (reuse && !differ[0])
    jc.ne = 0;
  if (jm.ne <= 0 && jc.ne <= 0)
    return;
  colorInit<R, true>(d, jm, gtid, gstride);
  colorInit<R, false>(d, jc, gtid, gstride);
  if (!gridBarrier(gb))
    return;
  int prevM = -1, prevC = -1;
  bool doneM = jm.ne <= 0, doneC = jc.ne <= 0;
  for (int round = 0; round < maxRounds && !(doneM && doneC); ++round) {
    if (!doneM)
      colorContend<R, true>(d, jm, round, gtid, gstride);
    if (!doneC)
      colorContend<R, false>(d, jc, round, gtid, gstride);
    if (!gridBarrier(gb))
      return;
    if (!doneM)
      colorCommit<R, true>(d, jm, round, gtid, gstride);
    if (!doneC)
      colorCommit<R, false>(d, jc, round, gtid, gstride);
    if (!gridBarrier(gb))
      return;
    if (!doneM) {
      const int rem = *reinterpret_cast<volatile int*>(&jm.aux[round % 3]);
      doneM = rem == 0 || rem == prevM;
      prevM = rem;
    }
    if (!doneC) {
      const int rem = *reinterpret_cast<volatile int*>(&jc.aux[round % 3]);
      doneC = rem == 0 || rem == prevC;
      prevC = rem;
    }
  }
  colorStats(jm, gtid, gstride);
  colorStats(jc, gtid, gstride);
}

}  // namespace pdem
