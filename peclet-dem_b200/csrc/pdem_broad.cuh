// LBVH broadphase (replaces src/broadphase_arborx.hpp:36-107, the ArborX BVH query).
//
// Candidate predicate (identical to the reference): box_i = [x_i - b_i, x_i + b_i] per axis with
// b_i = rad_i + margin (non-finite or oversized boxes parked at -1e30 with b = 0, SANE_BOX), and
// (i, j) is a candidate iff i is real, j > i and the two closed boxes overlap on every axis.
// Build: 63-bit Morton codes of the box centres (21 bits per axis, quantised in double), a stable
// radix sort of (code, index), a Karras binary radix tree (duplicate codes split by index), a
// bottom-up refit with arrival counters (no waiting), and escape ("rope") links for a stackless
// depth-first traversal. Emission: per-query count, exclusive scan, write, then each query's list
// is sorted by j, so the pair list is sorted by (i, j) — the canonical order.
#pragma once
#include "pdem_common.cuh"

namespace pdem {

template <class R>
struct Box {
  R lo[3], hi[3];
};

template <class R>
__device__ __forceinline__ Box<R> saneBox(const Dev<R>& d, int i, const Q4<R>* P, R margin, R boxCap) {
  const Q4<R> p = P[i];
  R x = p.x, y = p.y, z = p.z, b = d.rad[i] + margin;
  if (!(b == b) || !(x == x) || !(y == y) || !(z == z) || (boxCap > R(0) && b > boxCap)) {
    x = y = z = R(-1.0e30);
    b = R(0);
  }
  Box<R> bx;
  bx.lo[0] = x - b;
  bx.lo[1] = y - b;
  bx.lo[2] = z - b;
  bx.hi[0] = x + b;
  bx.hi[1] = y + b;
  bx.hi[2] = z + b;
  return bx;
}
template <class R>
__device__ __forceinline__ bool boxOverlap(const Box<R>& a, const Box<R>& b) {
  return !(a.lo[0] > b.hi[0] || a.hi[0] < b.lo[0] || a.lo[1] > b.hi[1] || a.hi[1] < b.lo[1] ||
           a.lo[2] > b.hi[2] || a.hi[2] < b.lo[2]);
}

// order-preserving encoding of a double for atomic min/max of signed values
__device__ __forceinline__ u64 orderedBits(double v) {
  const u64 b = (u64)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double fromOrderedBits(u64 o) {
  const u64 b = (o & 0x8000000000000000ull) ? (o & 0x7fffffffffffffffull) : ~o;
  return __longlong_as_double((long long)b);
}

struct BvhBuffers {
  int n = 0;             // primitives (all particles incl. ghosts)
  u64* codes = nullptr;  // [n] then sorted in place via the alt buffers
  u64* codesAlt = nullptr;
  int* idx = nullptr;    // [n] sorted primitive index
  int* idxAlt = nullptr;
  int *left = nullptr, *right = nullptr, *parent = nullptr, *rope = nullptr, *flag = nullptr;
  u64* bounds = nullptr;  // [6] ordered bits: min xyz, max xyz
  int* err = nullptr;     // error flags (Counters::err)
  // batched form: each scene's leaves are one contiguous sorted range (its id leads the key), so
  // each scene is one subtree; first/last leaf of every internal node bound a query to its scene
  const int* sceneOf = nullptr;    // [n] scene of each primitive (null: one scene)
  const int* leafFirst = nullptr;  // [scenes + 1] first sorted position of each scene
  int *first = nullptr, *last = nullptr;  // [n - 1] leaf range of each internal node
};
constexpr int kSceneShift = 54;  // batched Morton key: scene << 54 | the top 54 bits of the 63-bit code

// first / last sorted leaf under node v
__device__ __forceinline__ int nodeFirst(const BvhBuffers& bb, int v) {
  return v >= bb.n - 1 ? v - (bb.n - 1) : bb.first[v];
}
__device__ __forceinline__ int nodeLast(const BvhBuffers& bb, int v) {
  return v >= bb.n - 1 ? v - (bb.n - 1) : bb.last[v];
}

template <class R>
struct BvhNodes {
  Box<R>* prim = nullptr;  // [n] primitive boxes in ORIGINAL index order
  Box<R>* node = nullptr;  // [n-1] internal node boxes
};

template <class R>
__global__ void kBoxes(Dev<R> d, int n, R margin, R boxCap, BvhNodes<R> bn, BvhBuffers bb, R extra = R(0)) {
  u64 lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
  GRID_STRIDE(i, n) {
    const R mg = (d.scn ? d.scn[d.sceneOf[i]].margin : margin) + extra;
    const Box<R> b = saneBox(d, (int)i, d.posPred, mg, boxCap);
    bn.prim[i] = b;
    bool ok = true;
    double c[3];
    for (int a = 0; a < 3; ++a) {
      c[a] = 0.5 * ((double)b.lo[a] + (double)b.hi[a]);
      ok = ok && isfinite(c[a]) && fabs(c[a]) < 1e29;
    }
    if (ok)
      for (int a = 0; a < 3; ++a) {
        const u64 o = orderedBits(c[a]);
        lo[a] = o < lo[a] ? o : lo[a];
        hi[a] = o > hi[a] ? o : hi[a];
      }
  }
  // scene bounds: warp then block reduction, one atomic per block and bound (every warp has
  // boxes, and same-address atomics from all of them would serialise at L2)
  __shared__ u64 sLo[3][32], sHi[3][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      const u64 l = __shfl_xor_sync(0xffffffffu, lo[a], o), h = __shfl_xor_sync(0xffffffffu, hi[a], o);
      lo[a] = l < lo[a] ? l : lo[a];
      hi[a] = h > hi[a] ? h : hi[a];
    }
    if (lane == 0)
      sLo[a][w] = lo[a], sHi[a][w] = hi[a];
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    const int a = threadIdx.x % 3;
    const bool isLo = threadIdx.x < 3;
    u64 v = isLo ? ~0ull : 0ull;
    for (int k = 0; k < nw; ++k) {
      const u64 x = isLo ? sLo[a][k] : sHi[a][k];
      v = isLo ? (x < v ? x : v) : (x > v ? x : v);
    }
    if (isLo && v != ~0ull)
      atomicMin(&bb.bounds[a], v);
    if (!isLo && v != 0ull)
      atomicMax(&bb.bounds[3 + a], v);
  }
}

__device__ __forceinline__ u64 spread21(u64 v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

template <class R>
__global__ void kMorton(int n, BvhNodes<R> bn, BvhBuffers bb) {
  GRID_STRIDE(i, n) {
    const Box<R> b = bn.prim[i];
    double lo[3], ext[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = fromOrderedBits(bb.bounds[a]);
      ext[a] = fromOrderedBits(bb.bounds[3 + a]) - lo[a];
    }
    u64 code = 0x7fffffffffffffffull;
    bool ok = true;
    u64 q[3];
    for (int a = 0; a < 3; ++a) {
      const double c = 0.5 * ((double)b.lo[a] + (double)b.hi[a]);
      if (!(isfinite(c) && fabs(c) < 1e29)) {
        ok = false;
        break;
      }
      double t = ext[a] > 0.0 ? (c - lo[a]) / ext[a] : 0.0;
      t = fmin(fmax(t, 0.0), 1.0);
      q[a] = (u64)(t * 2097151.0);
    }
    if (ok)
      code = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
    if (bb.sceneOf)
      code = ((u64)bb.sceneOf[i] << kSceneShift) | (code >> (63 - kSceneShift));
    bb.codes[i] = code;
    bb.idx[i] = (int)i;
  }
}

// common-prefix length of sorted keys i and j (duplicates split by position)
__device__ __forceinline__ int deltaKey(const u64* k, int n, int i, int j) {
  if (j < 0 || j >= n)
    return -1;
  const u64 a = k[i], b = k[j];
  if (a == b)
    return 64 + __clz(i ^ j);
  return __clzll(a ^ b);
}

// Karras 2012: internal node i of n-1; leaves are nodes n-1 .. 2n-2
static __global__ void kKarras(BvhBuffers bb) {
  const int n = bb.n;
  GRID_STRIDE(ii, n - 1) {
    const int i = (int)ii;
    const u64* k = bb.codes;
    const int dir = (deltaKey(k, n, i, i + 1) - deltaKey(k, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = deltaKey(k, n, i, i - dir);
    int lmax = 2;
    while (deltaKey(k, n, i, i + lmax * dir) > dmin)
      lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
      if (deltaKey(k, n, i, i + (l + t) * dir) > dmin)
        l += t;
    const int j = i + l * dir;
    const int dnode = deltaKey(k, n, i, j);
    int s = 0, t = l;
    while (true) {
      t = (t + 1) >> 1;
      if (deltaKey(k, n, i, i + (s + t) * dir) > dnode)
        s += t;
      if (t <= 1)
        break;
    }
    const int gamma = i + s * dir + (dir < 0 ? -1 : 0);
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const int L = (lo == gamma) ? (n - 1 + gamma) : gamma;
    const int Rn = (hi == gamma + 1) ? (n - 1 + gamma + 1) : (gamma + 1);
    if (bb.first) {
      bb.first[i] = lo;
      bb.last[i] = hi;
    }
    bb.left[i] = L;
    bb.right[i] = Rn;
    bb.parent[L] = i;
    bb.parent[Rn] = i;
  }
}

template <class R>
__device__ __forceinline__ Box<R> loadBoxCG(const Box<R>* p) {
  Box<R> b;
  const R* s = reinterpret_cast<const R*>(p);
  R* o = reinterpret_cast<R*>(&b);
#pragma unroll
  for (int a = 0; a < 6; ++a)
    o[a] = __ldcg(s + a);
  return b;
}

// bottom-up box refit: the second child to arrive at a node computes its union
template <class R>
__global__ void kRefit(BvhBuffers bb, BvhNodes<R> bn) {
  const int n = bb.n;
  GRID_STRIDE(k, n) {
    int node = bb.parent[n - 1 + (int)k];
    for (int guard = 0;; ++guard) {
      if (guard > n) {  // deeper than the number of primitives: corrupt tree, stop
        atomicOr(&bb.err[0], 1);
        break;
      }
      __threadfence();
      if (atomicAdd(&bb.flag[node], 1) == 0)
        break;
      __threadfence();
      Box<R> u;
      const int c[2] = {bb.left[node], bb.right[node]};
      for (int s = 0; s < 2; ++s) {
        const Box<R> b = (c[s] >= n - 1) ? bn.prim[bb.idx[c[s] - (n - 1)]] : loadBoxCG(&bn.node[c[s]]);
        for (int a = 0; a < 3; ++a) {
          u.lo[a] = (s == 0) ? b.lo[a] : fmin(u.lo[a], b.lo[a]);
          u.hi[a] = (s == 0) ? b.hi[a] : fmax(u.hi[a], b.hi[a]);
        }
      }
      R* dst = reinterpret_cast<R*>(&bn.node[node]);
      const R* src = reinterpret_cast<const R*>(&u);
      for (int a = 0; a < 6; ++a)
        __stcg(dst + a, src[a]);
      if (node == 0)
        break;
      node = bb.parent[node];
    }
  }
}

// escape link of every node: the right sibling of the nearest ancestor-or-self that is a left
// child (-1 past the last leaf)
static __global__ void kRopes(BvhBuffers bb) {
  const int n = bb.n;
  GRID_STRIDE(v, 2 * n - 1) {
    int cur = (int)v, r = -1;
    for (int guard = 0; cur != 0; ++guard) {
      if (guard > n) {
        atomicOr(&bb.err[0], 1);
        break;
      }
      const int p = bb.parent[cur];
      if (bb.left[p] == cur) {
        r = bb.right[p];
        break;
      }
      cur = p;
    }
    bb.rope[v] = r;
  }
}

// stackless traversal for real particle i; mode 0 counts j > i, mode 1 writes them
template <class R, int MODE>
__global__ void kQuery(Dev<R> d, int numReal, BvhBuffers bb, BvhNodes<R> bn, int* cnt, const int* off,
                       int2* out, int outCap) {
  const int n = bb.n;
  // threads take the primitives in Morton order, so a warp's queries are spatial neighbours and
  // walk nearly the same nodes; each real particle's results go to its own (i-ordered) segment
  GRID_STRIDE(kk, n) {
    const int i = bb.idx[kk];
    if (i >= numReal)
      continue;
    const Box<R> q = bn.prim[i];
    int c = 0;
    int base = MODE ? off[i] : 0;
    int node = (n > 1) ? 0 : -1;
    for (long guard = 0; node != -1; ++guard) {
      if (guard > 4L * n + 8) {  // every node is visited at most once per query
        atomicOr(&bb.err[0], 1);
        break;
      }
      if (node >= n - 1) {
        const int j = bb.idx[node - (n - 1)];
        if (j > i && boxOverlap(q, bn.prim[j])) {
          if (MODE) {
            const int s = base + c;
            if (s < outCap)
              out[s] = make_int2(i, j);
          }
          ++c;
        }
        node = bb.rope[node];
      } else {
        if (boxOverlap(q, bn.node[node]))
          node = bb.left[node];
        else
          node = bb.rope[node];
      }
    }
    if (!MODE)
      cnt[i] = c;
  }
}

// sort each query's list by j (insertion sort; lists are short)
static __global__ void kSortPairLists(int numReal, const int* off, int2* pairs, int cap) {
  GRID_STRIDE(ii, numReal) {
    const int b = off[ii], e = min(off[ii + 1], cap);
    for (int x = b + 1; x < e; ++x) {
      const int2 v = pairs[x];
      int y = x - 1;
      while (y >= b && pairs[y].y > v.y) {
        pairs[y + 1] = pairs[y];
        --y;
      }
      pairs[y + 1] = v;
    }
  }
}

}  // namespace pdem

namespace pdem {

// =============================================================================================
// Packed tree for the single-pass query. Every node (internal 0..n-2, leaf n-1+k for sorted
// position k) is one 32-byte record: a float box rounded outward (it contains the exact box, so a
// miss on it is a miss on the exact box), the first child (internal) or -(j + 1) for the primitive
// j (leaf), and the escape link. The traversal tests the float box; a leaf hit is confirmed on the
// primitive's exact box in R, so the candidate set is exactly the reference predicate.
// =============================================================================================
struct __align__(16) PNode {
  float lo[3], hi[3];
  int a;     // internal: left child; leaf: -(primitive + 1)
  int rope;  // escape link (-1 past the last leaf)
};

__device__ __forceinline__ float roundDown(double v) { return __double2float_rd(v); }
__device__ __forceinline__ float roundUp(double v) { return __double2float_ru(v); }
__device__ __forceinline__ float roundDown(float v) { return v; }
__device__ __forceinline__ float roundUp(float v) { return v; }

template <class R>
__device__ __forceinline__ void outwardBox(const Box<R>& b, float lo[3], float hi[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = roundDown(b.lo[a]);
    hi[a] = roundUp(b.hi[a]);
  }
}
__device__ __forceinline__ bool overlapF(const float qlo[3], const float qhi[3], const PNode& n) {
  return !(qlo[0] > n.hi[0] || qhi[0] < n.lo[0] || qlo[1] > n.hi[1] || qhi[1] < n.lo[1] || qlo[2] > n.hi[2] ||
           qhi[2] < n.lo[2]);
}
__device__ __forceinline__ PNode loadNode(const PNode* p) {
  const float4* s = reinterpret_cast<const float4*>(p);
  const float4 u = __ldg(s), v = __ldg(s + 1);
  PNode n;
  n.lo[0] = u.x, n.lo[1] = u.y, n.lo[2] = u.z, n.hi[0] = u.w;
  n.hi[1] = v.x, n.hi[2] = v.y;
  n.a = __float_as_int(v.z);
  n.rope = __float_as_int(v.w);
  return n;
}

// leaves in sorted order: outward float box of the primitive and its index
template <class R>
__global__ void kPackLeaves(BvhBuffers bb, const Box<R>* prim, PNode* nodes) {
  const int n = bb.n;
  GRID_STRIDE(k, n) {
    const int j = bb.idx[k];
    PNode p;
    outwardBox(prim[j], p.lo, p.hi);
    p.a = -(j + 1);
    p.rope = -1;
    nodes[n - 1 + k] = p;
  }
}

// arrival counter with acquire-release ordering at device scope: the child's box stores before it
// are visible to the thread that sees the count, and that thread's loads come after it
__device__ __forceinline__ int arriveAcqRel(int* p) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

// refit-only substeps: the leaves keep their place in the last build's order (and their links);
// only their boxes are refreshed from the current primitive boxes
template <class R>
__global__ void kRefreshLeaves(BvhBuffers bb, const Box<R>* prim, PNode* nodes) {
  const int n = bb.n;
  GRID_STRIDE(k, n) {
    float lo[3], hi[3];
    outwardBox(prim[bb.idx[k]], lo, hi);
    float* dst = reinterpret_cast<float*>(&nodes[n - 1 + k]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dst[a] = lo[a];
      dst[3 + a] = hi[a];
    }
  }
}

// bottom-up union of the float boxes; the second child to arrive at a node computes it
static __global__ void kRefitPacked(BvhBuffers bb, PNode* nodes) {
  const int n = bb.n;
  GRID_STRIDE(k, n) {
    int node = bb.parent[n - 1 + (int)k];
    for (int guard = 0;; ++guard) {
      if (guard > n) {  // deeper than the number of primitives: corrupt tree, stop
        atomicOr(&bb.err[0], 1);
        break;
      }
      if (arriveAcqRel(&bb.flag[node]) == 0)
        break;
      const int c0 = bb.left[node], c1 = bb.right[node];
      float lo[3], hi[3];
      const float* b0 = reinterpret_cast<const float*>(&nodes[c0]);
      const float* b1 = reinterpret_cast<const float*>(&nodes[c1]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(__ldcg(b0 + a), __ldcg(b1 + a));
        hi[a] = fmaxf(__ldcg(b0 + 3 + a), __ldcg(b1 + 3 + a));
      }
      float* dst = reinterpret_cast<float*>(&nodes[node]);
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        __stcg(dst + a, lo[a]);
        __stcg(dst + 3 + a, hi[a]);
      }
      if (node == 0)
        break;
      node = bb.parent[node];
    }
  }
}

// escape links of all nodes, and the first child of internal nodes
static __global__ void kRopesPacked(BvhBuffers bb, PNode* nodes) {
  const int n = bb.n;
  GRID_STRIDE(v, 2 * n - 1) {
    int cur = (int)v, r = -1;
    for (int guard = 0; cur != 0; ++guard) {
      if (guard > n) {
        atomicOr(&bb.err[0], 1);
        break;
      }
      const int p = bb.parent[cur];
      if (bb.left[p] == cur) {
        r = bb.right[p];
        break;
      }
      cur = p;
    }
    nodes[v].rope = r;
    if (v < n - 1)
      nodes[v].a = bb.left[v];
  }
}

// Half traversal: the query at sorted position kk starts at its own leaf's escape link, so it
// visits only subtrees of sorted positions > kk and every overlapping unordered pair is found
// exactly once, by its lower sorted position. A found pair {i, j} belongs to row a = min(i, j)
// (kept when a is real); its rank in the row is taken with an atomic on the row count and kept,
// with the partner, in the query's own slots. The scatter pass places each pair at row offset +
// rank and the per-row sort by j restores the canonical (i, j) order, so the result does not
// depend on the order of the atomics. A query with more than kSlots pairs raises `overflow`; the
// host then runs the full two-pass traversal instead.
constexpr int kSlots = 32;

// first sorted leaf of every scene (the scene id leads each sorted key): leafFirst[s] = number of
// keys whose scene is below s
static __global__ void kSceneLeafFirst(int n, int scenes, const u64* sortedCodes, int* leafFirst) {
  GRID_STRIDE(s, scenes + 1) {
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((long)(sortedCodes[mid] >> kSceneShift) < (long)s)
        lo = mid + 1;
      else
        hi = mid;
    }
    leafFirst[s] = lo;
  }
}

template <class R>
__global__ void kQueryHalf(BvhBuffers bb, const Box<R>* prim, const PNode* nodes, int numReal, int* rowCnt,
                           int* qcnt, int2* slots, int* overflow) {
  const int n = bb.n;
  GRID_STRIDE(kk, n) {
    const PNode self = loadNode(&nodes[n - 1 + kk]);
    const int i = -self.a - 1;
    const Box<R> q = prim[i];
    float qlo[3], qhi[3];
    outwardBox(q, qlo, qhi);
    int c = 0;
    int node = self.rope;
    // batched form: the walk leaves this scene's subtree at the first node past its last leaf
    const int sceneEnd = bb.sceneOf ? bb.leafFirst[bb.sceneOf[i] + 1] : n;
    for (long guard = 0; node != -1; ++guard) {
      if (guard > 2L * n + 8) {  // each node is visited at most once
        atomicOr(&bb.err[0], 1);
        break;
      }
      if (bb.sceneOf && nodeFirst(bb, node) >= sceneEnd)
        break;
      const PNode nd = loadNode(&nodes[node]);
      if (overlapF(qlo, qhi, nd)) {
        if (nd.a >= 0) {
          node = nd.a;
          continue;
        }
        const int j = -nd.a - 1;
        if (boxOverlap(q, prim[j])) {
          const int lo = i < j ? i : j;
          if (lo < numReal) {
            if (c < kSlots)
              slots[(long)kk * kSlots + c] = make_int2(j, atomicAdd(&rowCnt[lo], 1));
            ++c;
          }
        }
      }
      node = nd.rope;
    }
    qcnt[kk] = c;
    if (c > kSlots)
      *overflow = 1;
  }
}

// place every found pair at its row offset + rank
static __global__ void kScatterHalf(BvhBuffers bb, const int* qcnt, const int2* slots, const int* rowOff, int2* out,
                             int outCap) {
  GRID_STRIDE(kk, bb.n) {
    const int c = min(qcnt[kk], kSlots);
    if (c == 0)
      continue;
    const int i = bb.idx[kk];
    for (int t = 0; t < c; ++t) {
      const int2 s = slots[(long)kk * kSlots + t];
      const int lo = i < s.x ? i : s.x, hi = i < s.x ? s.x : i;
      const int p = rowOff[lo] + s.y;
      if (p < outCap)
        out[p] = make_int2(lo, hi);
    }
  }
}

// Full traversal from the root for real particle i = idx[kk] (used when a half-traversal query
// overflowed its slots): MODE 0 counts the partners j > i, MODE 1 writes them at off[i].
template <class R, int MODE>
__global__ void kQueryFull(BvhBuffers bb, const Box<R>* prim, const PNode* nodes, int numReal, int* cnt,
                           const int* off, int2* out, int outCap) {
  const int n = bb.n;
  GRID_STRIDE(kk, n) {
    const int i = bb.idx[kk];
    if (i >= numReal)
      continue;
    const Box<R> q = prim[i];
    float qlo[3], qhi[3];
    outwardBox(q, qlo, qhi);
    int c = 0;
    const int base = MODE ? off[i] : 0;
    int node = 0;
    const int s0 = bb.sceneOf ? bb.leafFirst[bb.sceneOf[i]] : 0;
    const int s1 = bb.sceneOf ? bb.leafFirst[bb.sceneOf[i] + 1] : n;
    for (long guard = 0; node != -1; ++guard) {
      if (guard > 2L * n + 8) {
        atomicOr(&bb.err[0], 1);
        break;
      }
      const PNode nd = loadNode(&nodes[node]);
      if (bb.sceneOf && (nodeLast(bb, node) < s0 || nodeFirst(bb, node) >= s1)) {  // other scenes only
        node = nd.rope;
        continue;
      }
      if (overlapF(qlo, qhi, nd)) {
        if (nd.a >= 0) {
          node = nd.a;
          continue;
        }
        const int j = -nd.a - 1;
        if (j > i && boxOverlap(q, prim[j])) {
          if (MODE && base + c < outCap)
            out[base + c] = make_int2(i, j);
          ++c;
        }
      }
      node = nd.rope;
    }
    if (!MODE)
      cnt[i] = c;
  }
}

// ---------------------------------------------------------------------------------------------
// Verlet superset. A candidate list built with every box widened by half a skin contains every
// pair whose exact boxes overlap later, as long as no body moved more than half the skin (per
// axis) since the build and no box size changed. Between rebuilds each substep filters that list
// by the exact predicate on the current boxes; the filter keeps the list's canonical (i, j) order.

// largest per-axis displacement since the build over all primitives; a primitive whose slot now
// holds another body's image (or whose position is not finite) counts as infinitely far
template <class R>
__global__ void kVerletDisplacement(Dev<R> d, int n, const Q4<R>* ref, const int* refReal, R* out) {
  R m = R(0);
  GRID_STRIDE(i, n) {
    const Q4<R> a = d.posPred[i], b = ref[i];
    R v = fmax(fmax(fabs(a.x - b.x), fabs(a.y - b.y)), fabs(a.z - b.z));
    if (!(v <= R(1e30)) || d.realIdx[i] != refReal[i])
      v = R(1e30);
    runMax(m, v);
  }
  blockMaxAtomic(out, m);
}
template <class R>
__global__ void kFilterPairs(const int2* cand, int nc, const Box<R>* prim, int* keep) {
  GRID_STRIDE(k, nc) {
    const int2 p = cand[k];
    keep[k] = boxOverlap(prim[p.x], prim[p.y]) ? 1 : 0;
  }
}
static __global__ void kCompactPairs(const int2* cand, int nc, const int* keep, const int* off, int2* out, int cap) {
  GRID_STRIDE(k, nc) {
    if (keep[k] && off[k] < cap)
      out[off[k]] = cand[k];
  }
}

}  // namespace pdem
