// The broadphase's own sort: a stable least-significant-digit radix sort of (64-bit key, int
// value) pairs, 8-bit digits, for the Morton codes of the LBVH build (the leaf order of the tree).
//
// One pass per digit of the key's low `endBit` bits (the last digit masked to the bits below
// endBit), three launches a pass:
//   kRadixCount   each block counts the digits of its tile (2,048 keys) in shared memory and writes
//                 its 256 counts digit-major (count of digit d in block b at d * blocks + b);
//   kRadixScan    one block turns the digit-major counts into exclusive offsets: the keys of digit
//                 d from block b start after every smaller digit and after digit d of the blocks
//                 before b;
//   kRadixScatter each block walks its tile in the original order, 256 keys a round: equal digits
//                 in a warp rank among themselves by __match_any_sync, the warps of the round by a
//                 per-digit prefix over the warps' counts, and the rounds by a running offset per
//                 digit, so equal digits keep their input order (the sort is stable).
// No pass waits on another block (no spin), so the sort needs nothing but stream order. The passes
// ping-pong between the output and a scratch pair so that the last one writes the output.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace pdem {

constexpr int kRadixBlock = 256;                          // 8 warps
constexpr int kRadixItems = 8;                            // keys a thread per tile
constexpr int kRadixTile = kRadixBlock * kRadixItems;     // 2,048 keys a block
constexpr int kRadixScanBlock = 1024;

inline int radixBlocks(long n) { return (int)((n + kRadixTile - 1) / kRadixTile); }

// (templates on the key type: each translation unit that includes this header instantiates them once)
template <class K>
__global__ void __launch_bounds__(kRadixBlock) kRadixCount(const K* keys, int n, int shift, K mask, int* hist) {
  __shared__ int h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long base = (long)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixItems; ++r) {
    const long i = base + (long)r * kRadixBlock + threadIdx.x;
    if (i < n)
      atomicAdd(&h[(int)((keys[i] >> shift) & mask)], 1);
  }
  __syncthreads();
  hist[(long)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of m counts in place, one block: each thread sums a contiguous chunk, the block
// scans the chunk sums, each thread rewrites its chunk
template <class K>
__global__ void __launch_bounds__(kRadixScanBlock) kRadixScan(int* hist, int m) {
  __shared__ int s[kRadixScanBlock];
  const int chunk = (m + kRadixScanBlock - 1) / kRadixScanBlock;
  const long lo = (long)threadIdx.x * chunk, hi = min((long)m, lo + chunk);
  int sum = 0;
  for (long i = lo; i < hi; ++i)
    sum += hist[i];
  s[threadIdx.x] = sum;
  __syncthreads();
  for (int o = 1; o < kRadixScanBlock; o <<= 1) {  // inclusive Hillis-Steele scan of the sums
    const int v = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
    __syncthreads();
    s[threadIdx.x] += v;
    __syncthreads();
  }
  int run = s[threadIdx.x] - sum;
  for (long i = lo; i < hi; ++i) {
    const int c = hist[i];
    hist[i] = run;
    run += c;
  }
}

template <class K>
__global__ void __launch_bounds__(kRadixBlock) kRadixScatter(const K* kin, const int* vin, K* kout, int* vout, int n,
                                                             int shift, K mask, const int* off) {
  __shared__ int base[256];                        // where this block's next key of each digit goes
  __shared__ int cnt[kRadixBlock / 32][257];       // per warp: digit counts, then their warp prefix
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  base[threadIdx.x] = off[(long)threadIdx.x * gridDim.x + blockIdx.x];
  const long b0 = (long)blockIdx.x * kRadixTile;
  for (int r = 0; r < kRadixItems; ++r) {
    for (int k = threadIdx.x; k < (kRadixBlock / 32) * 257; k += kRadixBlock)
      (&cnt[0][0])[k] = 0;
    __syncthreads();
    const long i = b0 + (long)r * kRadixBlock + threadIdx.x;
    const bool ok = i < n;
    const K key = ok ? kin[i] : K(0);
    const int val = ok ? vin[i] : 0;
    const int dg = ok ? (int)((key >> shift) & mask) : 256;  // 256: no key
    const unsigned peers = __match_any_sync(0xffffffffu, dg);
    const int below = __popc(peers & ((1u << lane) - 1u));
    if (below == 0)
      cnt[w][dg] = __popc(peers);
    __syncthreads();
    // thread d: the exclusive prefix of digit d over the warps, and the round's count of d
    int tot = 0;
    {
      const int d = threadIdx.x;
      for (int k = 0; k < kRadixBlock / 32; ++k) {
        const int c = cnt[k][d];
        cnt[k][d] = tot;
        tot += c;
      }
    }
    __syncthreads();
    if (ok) {
      const int pos = base[dg] + cnt[w][dg] + below;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
    base[threadIdx.x] += tot;
  }
}

// Stable sort of n (key, value) pairs by the low endBit bits of the key into (kout, vout). tmpK /
// tmpV hold n pairs, hist 256 x radixBlocks(n) ints. kin / vin are not modified.
inline cudaError_t radixSortPairs(const unsigned long long* kin, unsigned long long* kout, const int* vin, int* vout,
                                  int n, int endBit, unsigned long long* tmpK, int* tmpV, int* hist,
                                  cudaStream_t st) {
  if (n <= 0)
    return cudaSuccess;
  const int passes = (endBit + 7) / 8;
  if (passes == 0) {
    cudaError_t e = cudaMemcpyAsync(kout, kin, n * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(vout, vin, n * sizeof(int), cudaMemcpyDeviceToDevice, st);
    return e;
  }
  const int nb = radixBlocks(n);
  const unsigned long long* sk = kin;
  const int* sv = vin;
  for (int p = 0; p < passes; ++p) {
    const bool toOut = ((passes - 1 - p) & 1) == 0;  // the last pass writes the output
    unsigned long long* dk = toOut ? kout : tmpK;
    int* dv = toOut ? vout : tmpV;
    // the last digit may be narrower: bits at or above endBit take no part
    const int bits = endBit - 8 * p < 8 ? endBit - 8 * p : 8;
    const unsigned long long mask = (1ull << bits) - 1ull;
    kRadixCount<unsigned long long><<<nb, kRadixBlock, 0, st>>>(sk, n, 8 * p, mask, hist);
    kRadixScan<unsigned long long><<<1, kRadixScanBlock, 0, st>>>(hist, 256 * nb);
    kRadixScatter<unsigned long long><<<nb, kRadixBlock, 0, st>>>(sk, sv, dk, dv, n, 8 * p, mask, hist);
    sk = dk;
    sv = dv;
  }
  return cudaGetLastError();
}

}  // namespace pdem
