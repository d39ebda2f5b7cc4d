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

constexpr int kErrBarrier = 2;  // Counters::err bit: a grid barrier timed out

// word[0] = arrivals, word[1] = generation; both zero before the launch; sleepNs = the back-off
// of a waiting block between polls of the generation; spins = the polls before a wait gives up
// (kBarrierSpins unless a test shortens it to make the wait run out)
struct GridBar {
  unsigned* word;
  int* err;
  unsigned sleepNs;
  long spins;
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
        if (++spins > gb.spins) {
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
// (kCtl): each END here is fused with the next sweep's BEGIN. CLUSTER: the launch is one thread-block
// cluster (a small graph), and the hardware cluster barrier (arrive with release, wait with acquire
// semantics at cluster scope) replaces the grid-wide one.
constexpr int kSweepCluster = 8;                                  // blocks of the portable cluster
constexpr int kSweepClusterEntries = 4 * kSweepCluster * kBlock;  // default largest graph it takes
template <bool CLUSTER>
__device__ __forceinline__ bool loopBarrier(const GridBar& gb) {
  if (CLUSTER) {
    cg::this_cluster().sync();
    return true;
  }
  return gridBarrier(gb);
}
// KIND 3: the projected GS velocity sweep of KIND 0 from the colour-ordered records of kPackPgs
// (entry t of the order is record t), the same arithmetic with fewer dependent loads. The colour
// offsets (at most 63 colours) are read once into shared memory.
template <class R, int KIND, int LOOP, bool CLUSTER = false>
__global__ void __launch_bounds__(kBlock) kSweepLoop(Dev<R> d, const int* order, const int* coff, int ncol, int iters,
                                                     SolveP<R> P, R thr, GridBar gb, PgsRecs<R> recs) {
  __shared__ int sOff[kSaturatedColor + 2];
  Counters<R>* c = d.ctr;
  volatile int* done = LOOP == 1 ? &c->velDone : LOOP == 2 ? &c->stabDone : &c->posDone;
  int* sweeps = LOOP == 1 ? &c->velSweeps : LOOP == 2 ? &c->stabSweeps : &c->posSweeps;
  R* mxp = KIND == 2 ? &c->maxOverlap : &c->maxApproach;
  const bool lead = (blockIdx.x | threadIdx.x) == 0;
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x, gstride = (long)gridDim.x * blockDim.x;
  if (*done)
    return;
  for (int k = threadIdx.x; k <= ncol && k < kSaturatedColor + 2; k += blockDim.x)
    sOff[k] = coff[k];
  __syncthreads();
  for (int it = 0; it < iters; ++it) {
    R mx = R(0);
    for (int col = 0; col < ncol; ++col) {
      const int b = sOff[col], n = sOff[col + 1] - b;
      // colour 62 is where the 62-colour mask saturates: not an independent set, so one thread
      // runs it in manifold order, as the reference's serial sweep does
      const bool serial = col >= kSaturatedColor;
      if (!serial || lead)
        for (long t = serial ? 0 : gtid; t < n; t += serial ? 1 : gstride) {
          if (KIND == 0) {
            pgsOne(d, order[b + t], P, mx, LOOP);
          } else if (KIND == 1) {
            gsOne(d, order[b + t], P, mx);
          } else if (KIND == 3) {
            int idx;
            const PgsStatic<R> st = pgsRecord(recs, b + t, idx);
            pgsCore<R>(d, idx, st, P.eN, P.mu, 0, P, mx);
          } else {
            posGSOne(d, order[b + t], mx);
          }
        }
      if (col == ncol - 1)
        warpMaxAtomic(mxp, mx);
      if (!loopBarrier<CLUSTER>(gb))
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
    if (!loopBarrier<CLUSTER>(gb))
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
// independent. Block b runs scene sceneOrder[b] (largest scenes first, so none is left to the last
// wave). The host has run the first sweep's BEGIN for every scene (kCtlScenes).
constexpr int kSceneBlock = 128;      // default block of the per-scene sweep loops
constexpr int kSceneBlockMax = 512;   // largest block the launch shape autotuner tries

template <class R, int KIND, int LOOP>
__global__ void __launch_bounds__(kSceneBlockMax) kSweepScenes(Dev<R> d, const int* sceneOrder, const int* order,
                                                            const int* off, int iters, SolveP<R> P, R thr) {
  const int s = sceneOrder[blockIdx.x];
  SceneCtl<R>& q = d.scn[s];
  volatile int* done = LOOP == 1 ? &q.velDone : LOOP == 2 ? &q.stabDone : &q.posDone;
  volatile R* mxp = KIND == 2 ? &q.maxOverlap : &q.maxApproach;
  if (*done)
    return;
  const int* so = off + (long)s * 64;
  __shared__ R sMax[kSceneBlockMax / 32];
  for (int it = 0; it < iters; ++it) {
    R mx = R(0);  // this thread's running max of the sweep; the block reduces it at the END
    for (int col = 0; col < 63; ++col) {
      const int b = so[col], n = so[col + 1] - b;
      if (n == 0)
        continue;  // uniform over the block
      const bool serial = col >= kSaturatedColor;
      if (!serial || threadIdx.x == 0)
        for (int t = serial ? 0 : threadIdx.x; t < n; t += serial ? 1 : blockDim.x) {
          if (KIND == 0)
            pgsOne<R, true>(d, order[b + t], P, mx, LOOP);
          else if (KIND == 1)
            gsOne<R, true>(d, order[b + t], P, mx);
          else
            posGSOne<R, true>(d, order[b + t], mx);
        }
      __syncthreads();
    }
    // the sweep's max over the block (the scene): no atomics on the scene's one max word
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const R w = __shfl_xor_sync(0xffffffffu, mx, o);
      mx = w > mx ? w : mx;
    }
    if ((threadIdx.x & 31) == 0)
      sMax[threadIdx.x >> 5] = mx;
    __syncthreads();
    // END of this sweep, then BEGIN of the next one (kCtlScenes' rule for this scene)
    if (threadIdx.x == 0) {
      R m = sMax[0];
      for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
        m = sMax[k] > m ? sMax[k] : m;
      *mxp = m;  // BEGIN left it 0 and only this block writes it during the loop
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
  int* aux;            // [0..2] remaining counts by round % 3, [3] max colour, [4] left uncoloured,
                       // [5] rounds run
  int *listA, *listB;  // [ne] each: every block's still-uncoloured entries, in its own chunk
  int* blockCount;     // [gridDim] the blocks' list lengths, published for the tail
  int *tailA, *tailB;  // [kColorTailMax] each: the tail's worklists (block 0 alone)
  int tailAt;          // block 0 takes over once at most this many entries (both graphs) are left
  int tailShared;      // the launch has the shared-memory tail's tables (dynamic shared memory)
  // stable order by colour, built in the same launch when order is set: order[ne] (entry indices,
  // colour-major, index order within a colour), off[65] (first position of each colour key, then
  // ne), hist[64 * gridDim] (scratch)
  int *order = nullptr, *off = nullptr, *hist = nullptr;
};
// once at most ColorJob::tailAt entries (both colourings together) are left, block 0 alone runs the
// remaining rounds with block barriers (in shared memory when they fit its tables), and the other
// blocks wait at one grid barrier
constexpr int kColorMaxChunks = 20;    // histogram row chunks of 32 blocks (grids up to 640 blocks)
constexpr int kColorTailMax = 65536;  // largest tail hand-over the worklists are sized for

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
// Worklists. Block b owns the entries [b chunk, (b + 1) chunk). Round 0 walks them all (skipping
// the coloured ones); every later round walks only the block's losers of the round before, kept
// in its own segment of listA / listB (ping-pong) and counted in shared memory. A round's outcome
// does not depend on the order its entries are visited in: the winners at one end are unique,
// winners never share an end, and losers only reset the next round's slots.
struct ColorRange {
  const int* list;  // nullptr: round 0, the whole chunk
  long first, count;
};
__device__ __forceinline__ ColorRange colorRange(const ColorJob& J, int round, int inCount) {
  const long chunk = (J.ne + gridDim.x - 1) / gridDim.x;
  const long first = (long)blockIdx.x * chunk;
  if (round == 0) {
    const long last = first + chunk < J.ne ? first + chunk : J.ne;
    return ColorRange{nullptr, first, last > first ? last - first : 0};
  }
  return ColorRange{((round & 1) ? J.listB : J.listA) + first, first, inCount};
}
template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorContend(const Dev<R>& d, const ColorJob& J, int round, const ColorRange& rg) {
  long long* win = (round & 1) ? J.winB : J.winA;
  if ((blockIdx.x | threadIdx.x) == 0)
    J.aux[(round + 1) % 3] = 0;
  for (long t = threadIdx.x; t < rg.count; t += blockDim.x) {
    const long i = rg.list ? rg.list[t] : rg.first + t;
    if (!rg.list && J.col[i] != -1)
      continue;
    int ea, eb;
    colorEnds<R, MANIFOLD>(d, (int)i, ea, eb);
    const long long k = entryKey<R, MANIFOLD>(d, (int)i, ea);
    atomicMax(&win[ea], k);
    if (eb >= 0)
      atomicMax(&win[eb], k);
  }
}
// losers go to the block's next list (shared-memory counter *outCount); the grid's loser count
// for the round's stop test is added once per block by the caller
template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorCommitTo(const Dev<R>& d, const ColorJob& J, int round, const ColorRange& rg,
                                              int* out, int* outCount) {
  long long* win = (round & 1) ? J.winB : J.winA;
  long long* nxt = (round & 1) ? J.winA : J.winB;
  for (long t = threadIdx.x; t < rg.count; t += blockDim.x) {
    const long i = rg.list ? rg.list[t] : rg.first + t;
    if (!rg.list && J.col[i] != -1)
      continue;
    int ea, eb;
    colorEnds<R, MANIFOLD>(d, (int)i, ea, eb);
    const long long k = entryKey<R, MANIFOLD>(d, (int)i, ea);
    if (__ldcg(&win[ea]) != k || (eb >= 0 && __ldcg(&win[eb]) != k)) {
      out[atomicAdd(outCount, 1)] = (int)i;
      nxt[ea] = -1;
      if (eb >= 0)
        nxt[eb] = -1;
      continue;
    }
    u64 forb = __ldcg(&J.mask[ea]);
    if (eb >= 0)
      forb |= __ldcg(&J.mask[eb]);
    int cc = 0;
    while (cc < 62 && (forb & (1ull << cc)))
      ++cc;
    J.col[i] = cc;
    J.mask[ea] |= 1ull << cc;
    if (eb >= 0)
      J.mask[eb] |= 1ull << cc;
  }
}
template <class R, bool MANIFOLD>
__device__ __forceinline__ void colorCommit(const Dev<R>& d, const ColorJob& J, int round, const ColorRange& rg,
                                            int* outCount) {
  colorCommitTo<R, MANIFOLD>(d, J, round, rg, (((round + 1) & 1) ? J.listB : J.listA) + rg.first, outCount);
}
// ---- stable order by colour (counting sort over 64 keys: colours 0..62, 63 for uncoloured, the
// order of the reference's stable sort by colour). Block b owns the contiguous chunk
// [b * chunk, (b + 1) * chunk) of the entries; the colour-major histogram H[key * gridDim + b]
// scanned exclusively gives each (key, block) its first position. Colours are read through L2
// (__ldcg): other SMs wrote them in this launch.
__device__ __forceinline__ int colorSortKey(int c) { return c >= 0 ? c : 63; }
__device__ __forceinline__ void colorChunk(const ColorJob& J, long& b0, long& b1) {
  const long chunk = ((long)J.ne + gridDim.x - 1) / gridDim.x;
  b0 = min((long)J.ne, (long)blockIdx.x * chunk);
  b1 = min((long)J.ne, b0 + chunk);
}
__device__ __forceinline__ void colorOrderCount(const ColorJob& J) {
  __shared__ int h[64];
  if (!J.order || J.ne <= 0)
    return;  // uniform over the grid
  long b0, b1;
  colorChunk(J, b0, b1);
  __syncthreads();
  if (threadIdx.x < 64)
    h[threadIdx.x] = 0;
  __syncthreads();
  for (long i = b0 + threadIdx.x; i < b1; i += blockDim.x)
    atomicAdd(&h[colorSortKey(__ldcg(&J.col[i]))], 1);
  __syncthreads();
  if (threadIdx.x < 64)
    J.hist[(long)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}
// one block: exclusive scan of the colour-major histogram in place, and the colour offsets. Each
// warp scans whole rows (colours) with shuffles over coalesced loads, then one warp scans the 64
// row totals, and each row gets its offset.
__device__ __forceinline__ void colorOrderScan(const ColorJob& J) {
  __shared__ int rowTot[64], rowOff[64];
  if (!J.order || J.ne <= 0)
    return;
  const int G = gridDim.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();  // rowTot / rowOff free (a previous call's reads are done)
  for (int c = w; c < 64; c += nw) {
    int* row = J.hist + (long)c * G;
    int run = 0;
    int vals[kColorMaxChunks];  // the row's loads, issued together (G <= 32 * kColorMaxChunks)
#pragma unroll
    for (int k = 0; k < kColorMaxChunks; ++k)
      vals[k] = (32 * k + lane < G) ? __ldcg(&row[32 * k + lane]) : 0;
#pragma unroll
    for (int k = 0; k < kColorMaxChunks; ++k) {
      const int b0 = 32 * k;
      if (b0 >= G)
        break;
      const int b = b0 + lane;
      const int v = vals[k];
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
          x += y;
      }
      if (b < G)
        row[b] = run + x - v;
      run += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0)
      rowTot[c] = run;
  }
  __syncthreads();
  if (w == 0) {
    const int a = rowTot[lane], b = rowTot[lane + 32];
    int xa = a, xb = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ya = __shfl_up_sync(0xffffffffu, xa, o), yb = __shfl_up_sync(0xffffffffu, xb, o);
      if (lane >= o) {
        xa += ya;
        xb += yb;
      }
    }
    const int totA = __shfl_sync(0xffffffffu, xa, 31);
    rowOff[lane] = xa - a;
    rowOff[lane + 32] = totA + xb - b;
  }
  __syncthreads();
  for (int c = w; c < 64; c += nw) {  // the same thread wrote these entries above
    int* row = J.hist + (long)c * G;
    for (int b = lane; b < G; b += 32)
      row[b] += rowOff[c];
  }
  if (threadIdx.x < 64)
    J.off[threadIdx.x] = rowOff[threadIdx.x];
  if (threadIdx.x == 0)
    J.off[64] = J.ne;
}
// every block: its chunk in tiles of blockDim entries; within a tile, the rank among equal keys is
// the lanes below in the warp with that key plus the earlier warps' counts of it
__device__ __forceinline__ void colorOrderScatter(const ColorJob& J) {
  __shared__ int run[64];
  __shared__ int cnt[kColorBlock / 32][64];
  if (!J.order || J.ne <= 0)
    return;
  long b0, b1;
  colorChunk(J, b0, b1);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (threadIdx.x < 64)
    run[threadIdx.x] = __ldcg(&J.hist[(long)threadIdx.x * gridDim.x + blockIdx.x]);
  for (long t0 = b0; t0 < b1; t0 += blockDim.x) {
    for (int k = threadIdx.x; k < nw * 64; k += blockDim.x)
      (&cnt[0][0])[k] = 0;
    __syncthreads();
    const long i = t0 + threadIdx.x;
    const int key = i < b1 ? colorSortKey(__ldcg(&J.col[i])) : 64;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int below = __popc(peers & ((1u << lane) - 1u));
    if (key < 64 && below == 0)
      cnt[w][key] = __popc(peers);
    __syncthreads();
    if (key < 64) {
      int pos = run[key] + below;
      for (int v = 0; v < w; ++v)
        pos += cnt[v][key];
      J.order[pos] = (int)i;
    }
    __syncthreads();
    if (threadIdx.x < 64) {
      int tot = 0;
      for (int v = 0; v < nw; ++v)
        tot += cnt[v][threadIdx.x];
      run[threadIdx.x] += tot;
    }
    __syncthreads();
  }
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

// The tail, in block 0 alone: gather every block's remaining entries into one list, then run the
// remaining rounds as the grid does (same contend / commit / stop rule), with block barriers.
// Global writes of one round are seen by the next through the barrier (and the L2 reads of win and
// mask in colorCommit).
template <class R, bool MANIFOLD>
__device__ __forceinline__ int colorTailGather(const ColorJob& J, int round, int* dst) {
  // thread b copies block b's list to its offset (an exclusive scan of the list lengths; the
  // grid has at most blockDim blocks)
  __shared__ int sWarp[kColorBlock / 32];
  __shared__ int sTotal;
  const long chunk = (J.ne + gridDim.x - 1) / gridDim.x;
  const int* src = (round & 1) ? J.listB : J.listA;  // the lists this round reads
  const int b = threadIdx.x, lane = b & 31, w = b >> 5;
  const int n = b < (int)gridDim.x ? J.blockCount[b] : 0;
  int incl = n;
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o)
      incl += u;
  }
  if (lane == 31)
    sWarp[w] = incl;
  __syncthreads();
  if (b == 0) {
    int run = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      const int c = sWarp[q];
      sWarp[q] = run;
      run += c;
    }
    sTotal = run;
  }
  __syncthreads();
  const int off = sWarp[w] + incl - n;
  for (int t = 0; t < n; ++t)
    dst[off + t] = src[(long)b * chunk + t];
  __threadfence_block();
  __syncthreads();
  return sTotal;
}
template <class R>
__device__ void colorTail(const Dev<R>& d, const ColorJob& jm, const ColorJob& jc, int round, int maxRounds,
                          bool doneM, bool doneC, int prevM, int prevC) {
  __shared__ int sOut[2];
  int nM = doneM ? 0 : colorTailGather<R, true>(jm, round, jm.tailA);
  int nC = doneC ? 0 : colorTailGather<R, false>(jc, round, jc.tailA);
  for (int k = 0; round < maxRounds && !(doneM && doneC); ++round, ++k) {
    const int* inM = (k & 1) ? jm.tailB : jm.tailA;
    const int* inC = (k & 1) ? jc.tailB : jc.tailA;
    int* outM = (k & 1) ? jm.tailA : jm.tailB;
    int* outC = (k & 1) ? jc.tailA : jc.tailB;
    if (threadIdx.x == 0)
      sOut[0] = sOut[1] = 0;
    const ColorRange rm{inM, 0, nM}, rc{inC, 0, nC};
    if (!doneM)
      colorContend<R, true>(d, jm, round, rm);
    if (!doneC)
      colorContend<R, false>(d, jc, round, rc);
    __syncthreads();  // block 0 alone: the block barrier orders its global accesses
    if (!doneM)
      colorCommitTo<R, true>(d, jm, round, rm, outM, &sOut[0]);
    if (!doneC)
      colorCommitTo<R, false>(d, jc, round, rc, outC, &sOut[1]);
    __syncthreads();  // block 0 alone: the block barrier orders its global accesses
    const int remM = sOut[0], remC = sOut[1];
    if (threadIdx.x == 0) {
      if (!doneM)
        jm.aux[round % 3] = remM;
      if (!doneC)
        jc.aux[round % 3] = remC;
    }
    if (!doneM) {
      doneM = remM == 0 || remM == prevM;
      prevM = remM;
      nM = remM;
    }
    if (!doneC) {
      doneC = remC == 0 || remC == prevC;
      prevC = remC;
      nC = remC;
    }
    __syncthreads();
  }
}

// The tail in shared memory (block 0 alone, at most kTailShEntries entries of both graphs): every
// body the remaining entries touch gets a slot of a hash table (code body * 2 + graph), holding its
// winner word and colour mask, so a round touches no global memory but the final colours. The
// rounds, winners and colours are those of colorTail: contend (max of the keys at both ends), win
// with the maximum at both ends, take the lowest colour free at both ends; the losers contend
// again. One winner word per slot suffices: after each commit the words of every end touched that
// round go back to -1, and the next round's contenders are that round's losers.
constexpr int kTailShEntries = 1024;
constexpr int kTailShSlots = 4096;  // a power of two, at least 2 ends x entries x 2
struct TailShared {
  u64 mask[kTailShSlots];
  long long win[kTailShSlots];
  long long key[kTailShEntries];
  int body[kTailShSlots];  // code of the slot's body, -1 free
  int ent[kTailShEntries];
  short la[kTailShEntries], lb[kTailShEntries];  // slots of the ends (lb -1: no second body)
  short list[2][kTailShEntries];                 // entries of this round and the next
  unsigned char g[kTailShEntries];               // 0 manifold graph, 1 contact graph
};
__device__ __forceinline__ int tailSlot(TailShared& S, int code) {
  const unsigned h = (unsigned)code * 2654435761u;
  for (int probe = 0; probe < kTailShSlots; ++probe) {  // at most 2 x kTailShEntries codes: a slot is free
    const int s = (int)((h + (unsigned)probe) & (kTailShSlots - 1));
    const int prev = atomicCAS(&S.body[s], -1, code);
    if (prev == -1 || prev == code)
      return s;
  }
  return 0;
}
template <class R, bool MANIFOLD>
__device__ __forceinline__ void tailEntry(const Dev<R>& d, TailShared& S, int t, int i, int g) {
  int ea, eb;
  colorEnds<R, MANIFOLD>(d, i, ea, eb);
  S.ent[t] = i;
  S.g[t] = (unsigned char)g;
  S.key[t] = entryKey<R, MANIFOLD>(d, i, ea);
  S.la[t] = (short)tailSlot(S, 2 * ea + g);
  S.lb[t] = (short)(eb >= 0 ? tailSlot(S, 2 * eb + g) : -1);
  S.list[0][t] = (short)t;
}
template <class R>
__device__ void colorTailShared(const Dev<R>& d, const ColorJob& jm, const ColorJob& jc, int round, int maxRounds,
                                bool doneM, bool doneC, int prevM, int prevC) {
  extern __shared__ __align__(16) unsigned char tailSmem[];
  TailShared& S = *reinterpret_cast<TailShared*>(tailSmem);
  __shared__ int sLose[2], sNext;
  const int nM = doneM ? 0 : colorTailGather<R, true>(jm, round, jm.tailA);
  const int nC = doneC ? 0 : colorTailGather<R, false>(jc, round, jc.tailA);
  for (int s = threadIdx.x; s < kTailShSlots; s += blockDim.x)
    S.body[s] = -1;
  __syncthreads();
  for (int t = threadIdx.x; t < nM + nC; t += blockDim.x) {
    if (t < nM)
      tailEntry<R, true>(d, S, t, jm.tailA[t], 0);
    else
      tailEntry<R, false>(d, S, t, jc.tailA[t - nM], 1);
  }
  __syncthreads();
  for (int s = threadIdx.x; s < kTailShSlots; s += blockDim.x) {
    const int code = S.body[s];
    if (code >= 0)
      S.mask[s] = __ldcg(&((code & 1) ? jc.mask : jm.mask)[code >> 1]);
    S.win[s] = -1;
  }
  int cnt = nM + nC;
  for (int k = 0; round < maxRounds && !(doneM && doneC); ++round, ++k) {
    const short* in = S.list[k & 1];
    short* out = S.list[(k + 1) & 1];
    if (threadIdx.x == 0)
      sLose[0] = sLose[1] = sNext = 0;
    __syncthreads();  // the slots' words and masks, and the counters, are set
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int t = in[j];
      if (S.g[t] ? doneC : doneM)
        continue;
      atomicMax(&S.win[S.la[t]], S.key[t]);
      if (S.lb[t] >= 0)
        atomicMax(&S.win[S.lb[t]], S.key[t]);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int t = in[j];
      const int g = S.g[t];
      if (g ? doneC : doneM)
        continue;
      const int la = S.la[t], lb = S.lb[t];
      const long long key = S.key[t];
      if (S.win[la] != key || (lb >= 0 && S.win[lb] != key)) {
        out[atomicAdd(&sNext, 1)] = (short)t;
        atomicAdd(&sLose[g], 1);
        continue;
      }
      const u64 forb = S.mask[la] | (lb >= 0 ? S.mask[lb] : 0ull);
      int cc = 0;
      while (cc < 62 && (forb & (1ull << cc)))
        ++cc;
      (g ? jc : jm).col[S.ent[t]] = cc;
      S.mask[la] |= 1ull << cc;  // the round's winners share no end
      if (lb >= 0)
        S.mask[lb] |= 1ull << cc;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
      const int t = in[j];
      if (S.g[t] ? doneC : doneM)
        continue;
      S.win[S.la[t]] = -1;
      if (S.lb[t] >= 0)
        S.win[S.lb[t]] = -1;
    }
    const int remM = sLose[0], remC = sLose[1];
    cnt = sNext;
    if (threadIdx.x == 0) {
      if (!doneM)
        jm.aux[round % 3] = remM;
      if (!doneC)
        jc.aux[round % 3] = remC;
    }
    if (!doneM) {
      doneM = remM == 0 || remM == prevM;
      prevM = remM;
    }
    if (!doneC) {
      doneC = remC == 0 || remC == prevC;
      prevC = remC;
    }
    __syncthreads();  // the counters are read before the next round resets them
  }
}

// job 0: manifolds over real bodies (skipped when ne = 0), job 1: contacts over body slots.
// CLUSTER: the launch is one thread-block cluster (graphs of a few tens of thousands of entries)
// and the hardware cluster barrier replaces the grid-wide one, as in kSweepLoop.
// reuse: a graph equal to the previous substep's keeps its colours and statistics (differ[0]: the
// contact list changed, differ[1]: the manifold list changed; reuse = 0 forces both colourings)
template <class R, bool CLUSTER = false>
__global__ void __launch_bounds__(kColorBlock) kColorBoth(Dev<R> d, ColorJob jm, ColorJob jc, int maxRounds,
                                                          GridBar gb, const int* differ, int reuse) {
  __shared__ int sCount[2][2];  // per job: this block's loser counts, ping-pong by round
  const long gtid = (long)blockIdx.x * blockDim.x + threadIdx.x, gstride = (long)gridDim.x * blockDim.x;
  if (reuse && !differ[1])
    jm.ne = 0;  // uniform over the grid: the flags are written before the launch
  if (reuse && !differ[0])
    jc.ne = 0;
  if (jm.ne <= 0 && jc.ne <= 0)
    return;
  colorInit<R, true>(d, jm, gtid, gstride);
  colorInit<R, false>(d, jc, gtid, gstride);
  if (threadIdx.x < 4)
    sCount[threadIdx.x >> 1][threadIdx.x & 1] = 0;
  if (!loopBarrier<CLUSTER>(gb))
    return;
  int prevM = -1, prevC = -1;
  bool doneM = jm.ne <= 0, doneC = jc.ne <= 0;
  int round = 0;
  bool tail = false;
  for (; round < maxRounds && !(doneM && doneC); ++round) {
    const int in = round & 1, outS = in ^ 1;  // shared counter slots: this round's list, the next
    const ColorRange rm = colorRange(jm, round, sCount[0][in]), rc = colorRange(jc, round, sCount[1][in]);
    if (!doneM)
      colorContend<R, true>(d, jm, round, rm);
    if (!doneC)
      colorContend<R, false>(d, jc, round, rc);
    if (!loopBarrier<CLUSTER>(gb))
      return;
    if (!doneM)
      colorCommit<R, true>(d, jm, round, rm, &sCount[0][outS]);
    if (!doneC)
      colorCommit<R, false>(d, jc, round, rc, &sCount[1][outS]);
    __syncthreads();
    if (threadIdx.x == 0) {  // this block's losers into the grid's count; its consumed slot reset
      if (!doneM && sCount[0][outS])
        atomicAdd(&jm.aux[round % 3], sCount[0][outS]);
      if (!doneC && sCount[1][outS])
        atomicAdd(&jc.aux[round % 3], sCount[1][outS]);
      sCount[0][in] = sCount[1][in] = 0;
    }
    if (!loopBarrier<CLUSTER>(gb))
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
    // few entries left: publish this block's lists, and block 0 takes over (uniform decision)
    if (!(doneM && doneC) && round + 1 < maxRounds && gridDim.x <= blockDim.x &&
        (doneM ? 0 : prevM) + (doneC ? 0 : prevC) <= jm.tailAt) {
      if (threadIdx.x == 0) {
        jm.blockCount[blockIdx.x] = doneM ? 0 : sCount[0][(round + 1) & 1];
        jc.blockCount[blockIdx.x] = doneC ? 0 : sCount[1][(round + 1) & 1];
      }
      tail = true;
      ++round;
      break;
    }
  }
  if (tail) {
    if (!loopBarrier<CLUSTER>(gb))  // the published lists are complete
      return;
    if (blockIdx.x == 0) {
      if (jm.tailShared)
        colorTailShared(d, jm, jc, round, maxRounds, doneM, doneC, prevM, prevC);
      else
        colorTail(d, jm, jc, round, maxRounds, doneM, doneC, prevM, prevC);
    }
    if (!loopBarrier<CLUSTER>(gb))  // the tail's colours are visible to every block
      return;
  }
  if (gtid == 0) {
    if (jm.ne > 0)
      jm.aux[5] = round;
    if (jc.ne > 0)
      jc.aux[5] = round;
  }
  colorStats(jm, gtid, gstride);
  colorStats(jc, gtid, gstride);
  // both colour orders (unless kept or batched: then the host orders them)
  if (!jm.order && !jc.order)
    return;
  colorOrderCount(jm);
  colorOrderCount(jc);
  if (!loopBarrier<CLUSTER>(gb))
    return;
  if (blockIdx.x == 0)
    colorOrderScan(jm);
  if (blockIdx.x == (gridDim.x > 1 ? 1 : 0))
    colorOrderScan(jc);
  if (!loopBarrier<CLUSTER>(gb))
    return;
  colorOrderScatter(jm);
  colorOrderScatter(jc);
}

}  // namespace pdem
