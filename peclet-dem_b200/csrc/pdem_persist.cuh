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

// back-off iterations before a barrier wait gives up (a few seconds with __nanosleep(64))
constexpr long kBarrierSpins = 1L << 26;
constexpr int kErrBarrier = 2;  // Counters::err bit: a grid barrier timed out

// word[0] = arrivals, word[1] = generation; both zero before the launch
struct GridBar {
  unsigned* word;
  int* err;
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
        __nanosleep(64);
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
// Jones-Plassmann colouring rounds (src/solver_velocity.hpp:277-374, src/solver_position.hpp:
// 155-241) until no entry is left or a round colours nothing. Preconditions set by the host:
// mask[0..nb) = 0, col initialised (-1 = to colour, -2 = skipped), winA[0..nb) = -1,
// remCnt[0..3) = 0. Two winner arrays alternate by round: the losers of round r, the only entries
// of round r + 1, reset their bodies in the other array during round r. The remaining-entry count
// of round r lives in remCnt[r % 3]; the lead zeroes the slot of round r + 1 during round r.
// At the end the colour statistics (largest colour, entries left uncoloured) are accumulated into
// stats[0] (atomic max, preset to INT_MIN) and stats[1] (preset to 0).
constexpr int kColorBlock = 1024;  // one large block per SM: fewer arrivals per grid barrier

template <class R, bool MANIFOLD>
__global__ void __launch_bounds__(kColorBlock) kColorLoop(Dev<R> d, int ne, int maxRounds, int* col, long long* winA,
                                                     long long* winB, int* remCnt, int* stats, GridBar gb) {
  const bool lead = (blockIdx.x | threadIdx.x) == 0;
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x, gstride = (long)gridDim.x * blockDim.x;
  int prev = -1;
  for (int round = 0; round < maxRounds; ++round) {
    long long* win = (round & 1) ? winB : winA;
    long long* nxt = (round & 1) ? winA : winB;
    if (lead)
      remCnt[(round + 1) % 3] = 0;
    for (long i = gtid; i < ne; i += gstride) {
      if (col[i] != -1)
        continue;
      int ea, eb;
      colorEnds<R, MANIFOLD>(d, (int)i, ea, eb);
      const long long k = entryKey<R, MANIFOLD>(d, (int)i, ea);
      atomicMax(&win[ea], k);
      if (eb >= 0)
        atomicMax(&win[eb], k);
    }
    if (!gridBarrier(gb))
      return;
    int lost = 0;
    for (long i = gtid; i < ne; i += gstride) {
      if (col[i] != -1)
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
      u64 forb = d.mask[ea];
      if (eb >= 0)
        forb |= d.mask[eb];
      int cc = 0;
      while (cc < 62 && (forb & (1ull << cc)))
        ++cc;
      col[i] = cc;
      d.mask[ea] |= 1ull << cc;
      if (eb >= 0)
        d.mask[eb] |= 1ull << cc;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      lost += __shfl_xor_sync(0xffffffffu, lost, o);
    if ((threadIdx.x & 31) == 0 && lost)
      atomicAdd(&remCnt[round % 3], lost);
    if (!gridBarrier(gb))
      return;
    const int rem = *reinterpret_cast<volatile int*>(&remCnt[round % 3]);
    if (rem == 0 || rem == prev)
      break;
    prev = rem;
  }
  int mxc = INT_MIN, left = 0;
  for (long i = gtid; i < ne; i += gstride) {
    const int v = col[i];
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
      atomicMax(&stats[0], mxc);
    if (left)
      atomicAdd(&stats[1], left);
  }
}

}  // namespace pdem
