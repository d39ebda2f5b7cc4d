// Candidate-pair search that allocates nothing: the LBVH broadphase of the substep
// (pdem_broad.cuh: boxes, Morton codes, radix sort, Karras tree, refit, ropes, two-pass query,
// per-query sort) run over caller-owned device arrays, with every scratch array carved out of one
// file-scope __device__ buffer of fixed size instead of cudaMalloc'd memory.
//
// Who needs it: a host code that couples the particle step to its own solver and owns the whole
// device memory budget (a CFD code that reserves HBM at start-up and forbids allocation inside its
// time loop), or a code that cannot afford the implicit device-wide synchronisation of
// cudaMalloc/cudaFree between its streams. Such a caller supplies positions and radii already on
// the device and a device output buffer, and gets the same canonical (i, j)-sorted pair list as the
// simulation's own broadphase, with no allocation by this library, by CUB or by anything else.
//
// Limits and rules:
//  * at most kStaticMaxBodies (16384) bodies per call; larger calls are rejected with
//    PDEM_ERR_INVALID before anything is launched;
//  * the first call on a device does the set-up (cudaGetSymbolAddress of the scratch buffer and the
//    CUB temporary-size queries, neither of which allocates), so make it before any stream capture;
//  * the scratch buffer is shared by every call on a device: calls that overlap in time (two host
//    threads, or two streams without ordering between them) race on it and corrupt each other;
//  * arrays that must start at zero (tree arrival counters, per-query counts, the error flag) and
//    the scene bounds are reset inside every call on the caller's stream; nothing is assumed from a
//    previous call. The call returns after synchronising that stream (the pair count is read back).
#include <cstring>
#include <mutex>
#include <string>

#include <cub/cub.cuh>

#include "../../include/pdem.h"
#include "pdem_broad.cuh"

namespace pdem {
void setLastError(const std::string& msg);  // pdem_capi.cu
}

namespace {

using pdem::BvhBuffers;
using pdem::BvhNodes;
using pdem::Box;
using pdem::Q4;
using pdem::u64;

constexpr int kStaticMaxBodies = 16384;
constexpr int kMaxDevices = 64;

// scratch layout in bytes, every array 256-byte aligned
constexpr size_t al(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t kN = kStaticMaxBodies;
constexpr size_t kOffPos = 0;                                          // Q4<double>[n]
constexpr size_t kOffPrim = kOffPos + al(sizeof(Q4<double>) * kN);     // Box<double>[n]
constexpr size_t kOffNode = kOffPrim + al(sizeof(Box<double>) * kN);   // Box<double>[n]
constexpr size_t kOffCodes = kOffNode + al(sizeof(Box<double>) * kN);  // u64[n]
constexpr size_t kOffCodesAlt = kOffCodes + al(8 * kN);                // u64[n]
constexpr size_t kOffIdx = kOffCodesAlt + al(8 * kN);                  // int[n]
constexpr size_t kOffIdxAlt = kOffIdx + al(4 * kN);                    // int[n]
constexpr size_t kOffLeft = kOffIdxAlt + al(4 * kN);                   // int[n]
constexpr size_t kOffRight = kOffLeft + al(4 * kN);                    // int[n]
constexpr size_t kOffParent = kOffRight + al(4 * kN);                  // int[2n]
constexpr size_t kOffRope = kOffParent + al(8 * kN);                   // int[2n]
constexpr size_t kOffFlag = kOffRope + al(8 * kN);                     // int[n]     zeroed per call
constexpr size_t kOffCnt = kOffFlag + al(4 * kN);                      // int[n+1]   zeroed per call
constexpr size_t kOffOff = kOffCnt + al(4 * (kN + 1));                 // int[n+1]
constexpr size_t kOffBounds = kOffOff + al(4 * (kN + 1));              // u64[6]     set per call
constexpr size_t kOffErr = kOffBounds + al(48);                        // int        zeroed per call
constexpr size_t kOffCub = kOffErr + al(sizeof(int));                  // CUB temporary storage
constexpr size_t kCubBytes = size_t(2) << 20;
constexpr size_t kScratchBytes = kOffCub + kCubBytes;  // 5,178,368 bytes

}  // namespace

// the whole scratch of a call, sized for kStaticMaxBodies bodies
static __device__ __align__(256) unsigned char gScratch[kScratchBytes];

namespace {

struct DeviceSetup {
  bool done = false;
  unsigned char* base = nullptr;
};
DeviceSetup gSetup[kMaxDevices];
std::mutex gSetupMutex;

struct Fail {
  int status;
  std::string msg;
};
void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw Fail{PDEM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

// per-call reset of the scene bounds (min = all ones, max = zero in the ordered encoding) and error flag
__global__ void kResetStatic(u64* bounds, int* err) {
  if (threadIdx.x < 6)
    bounds[threadIdx.x] = threadIdx.x < 3 ? ~0ull : 0ull;
  if (threadIdx.x == 0)
    *err = 0;
}

// (x, y, z) rows -> aligned 4-wide records in scratch
__global__ void kPackPositions(const double* xyz, int n, Q4<double>* out) {
  GRID_STRIDE(i, n) {
    Q4<double> q;
    q.x = xyz[3 * i];
    q.y = xyz[3 * i + 1];
    q.z = xyz[3 * i + 2];
    q.w = 0.0;
    out[i] = q;
  }
}

// once per device, with that device current: resolve the scratch address and check that CUB's
// temporaries for the largest allowed call fit in the space reserved for them
unsigned char* setupDevice(int dev) {
  std::lock_guard<std::mutex> lock(gSetupMutex);
  DeviceSetup& s = gSetup[dev];
  if (s.done)
    return s.base;
  void* p = nullptr;
  check(cudaGetSymbolAddress(&p, gScratch), "cudaGetSymbolAddress(scratch)");
  size_t sortBytes = 0, scanBytes = 0;
  check(cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, (const u64*)nullptr, (u64*)nullptr, (const int*)nullptr,
                                        (int*)nullptr, kStaticMaxBodies, 0, 63),
        "CUB sort size query");
  check(cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, (const int*)nullptr, (int*)nullptr, kStaticMaxBodies + 1),
        "CUB scan size query");
  if (sortBytes > kCubBytes || scanBytes > kCubBytes)
    throw Fail{PDEM_ERR_RUNTIME, "static broadphase: CUB temporary storage exceeds the reserved scratch"};
  s.base = static_cast<unsigned char*>(p);
  s.done = true;
  return s.base;
}

}  // namespace

extern "C" int pdem_find_pairs_static(const double* d_xyz, const double* d_radius, int n, double margin,
                                      double box_cap, int* d_pairs, long pair_cap, long* out_count,
                                      void* stream) {
  try {
    if (n < 0 || n > kStaticMaxBodies)
      throw Fail{PDEM_ERR_INVALID, "pdem_find_pairs_static: n = " + std::to_string(n) + " outside [0, " +
                                       std::to_string(kStaticMaxBodies) + "]"};
    if (!out_count || pair_cap < 0 || (n > 0 && (!d_xyz || !d_radius)) || (pair_cap > 0 && !d_pairs))
      throw Fail{PDEM_ERR_INVALID, "pdem_find_pairs_static: null pointer or negative capacity"};
    *out_count = 0;
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices)
      throw Fail{PDEM_ERR_RUNTIME, "pdem_find_pairs_static: device index out of range"};
    unsigned char* base = setupDevice(dev);
    if (n < 2)
      return PDEM_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    Q4<double>* pos = reinterpret_cast<Q4<double>*>(base + kOffPos);
    BvhNodes<double> bn{reinterpret_cast<Box<double>*>(base + kOffPrim), reinterpret_cast<Box<double>*>(base + kOffNode)};
    BvhBuffers bb;
    bb.n = n;
    bb.codes = reinterpret_cast<u64*>(base + kOffCodes);
    bb.codesAlt = reinterpret_cast<u64*>(base + kOffCodesAlt);
    bb.idx = reinterpret_cast<int*>(base + kOffIdx);
    bb.idxAlt = reinterpret_cast<int*>(base + kOffIdxAlt);
    bb.left = reinterpret_cast<int*>(base + kOffLeft);
    bb.right = reinterpret_cast<int*>(base + kOffRight);
    bb.parent = reinterpret_cast<int*>(base + kOffParent);
    bb.rope = reinterpret_cast<int*>(base + kOffRope);
    bb.flag = reinterpret_cast<int*>(base + kOffFlag);
    bb.bounds = reinterpret_cast<u64*>(base + kOffBounds);
    bb.err = reinterpret_cast<int*>(base + kOffErr);
    int* cnt = reinterpret_cast<int*>(base + kOffCnt);
    int* off = reinterpret_cast<int*>(base + kOffOff);
    void* cubTmp = base + kOffCub;

    // the boxes read positions and radii through the simulation's device view
    pdem::Dev<double> d{};
    d.posPred = pos;
    d.rad = const_cast<double*>(d_radius);

    const int B = pdem::kBlock;
    kResetStatic<<<1, 32, 0, st>>>(bb.bounds, bb.err);
    check(cudaMemsetAsync(bb.flag, 0, sizeof(int) * n, st), "arrival counter reset");
    check(cudaMemsetAsync(cnt, 0, sizeof(int) * (n + 1), st), "query count reset");
    kPackPositions<<<pdem::gridFor(n), B, 0, st>>>(d_xyz, n, pos);
    pdem::kBoxes<double><<<pdem::gridFor(n), B, 0, st>>>(d, n, margin, box_cap, bn, bb);
    pdem::kMorton<double><<<pdem::gridFor(n), B, 0, st>>>(n, bn, bb);
    size_t bytes = kCubBytes;
    check(cub::DeviceRadixSort::SortPairs(cubTmp, bytes, bb.codes, bb.codesAlt, bb.idx, bb.idxAlt, n, 0, 63, st),
          "CUB sort");
    std::swap(bb.codes, bb.codesAlt);
    std::swap(bb.idx, bb.idxAlt);
    pdem::kKarras<<<pdem::gridFor(n - 1), B, 0, st>>>(bb);
    pdem::kRefit<double><<<pdem::gridFor(n), B, 0, st>>>(bb, bn);
    pdem::kRopes<<<pdem::gridFor(2 * n - 1), B, 0, st>>>(bb);
    pdem::kQuery<double, 0><<<pdem::gridFor(n, 128), 128, 0, st>>>(d, n, bb, bn, cnt, nullptr, nullptr, 0);
    bytes = kCubBytes;
    check(cub::DeviceScan::ExclusiveSum(cubTmp, bytes, cnt, off, n + 1, st), "CUB scan");
    check(cudaGetLastError(), "broadphase launch");
    int total = 0, err = 0;
    check(cudaMemcpyAsync(&total, off + n, sizeof(int), cudaMemcpyDeviceToHost, st), "count read-back");
    check(cudaMemcpyAsync(&err, bb.err, sizeof(int), cudaMemcpyDeviceToHost, st), "error read-back");
    check(cudaStreamSynchronize(st), "stream synchronize");
    if (err)
      throw Fail{PDEM_ERR_RUNTIME, "pdem_find_pairs_static: BVH traversal exceeded its iteration bound"};
    *out_count = total;
    if (total <= pair_cap) {
      int2* out = reinterpret_cast<int2*>(d_pairs);
      const int cap = (int)std::min<long>(pair_cap, 0x7fffffff);
      pdem::kQuery<double, 1><<<pdem::gridFor(n, 128), 128, 0, st>>>(d, n, bb, bn, nullptr, off, out, cap);
      pdem::kSortPairLists<<<pdem::gridFor(n), B, 0, st>>>(n, off, out, cap);
      check(cudaGetLastError(), "broadphase write launch");
      check(cudaStreamSynchronize(st), "stream synchronize");
    }
    return PDEM_OK;
  } catch (const Fail& f) {
    pdem::setLastError(f.msg);
    return f.status;
  } catch (const std::exception& e) {
    pdem::setLastError(e.what());
    return PDEM_ERR_RUNTIME;
  }
}
