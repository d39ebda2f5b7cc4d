// Minimal ArborX API shim (test infrastructure, not product code).
//
// The reference broadphase (src/broadphase_arborx.hpp:36-107) builds ArborX::Box<3> AABBs, a
// BoundingVolumeHierarchy over all particles and one `intersects(box)` query per real particle.
// ArborX is not available here, so this shim answers the SAME query exactly: primitive j matches
// query q iff the two closed boxes overlap on every axis (ArborX's box-box `intersects`, the
// corner predicate the reference relies on). Acceleration is a uniform cell list over box centres
// (cell edge >= the largest box width, candidates from the neighbouring cells, exact predicate on
// each candidate); boxes that are not finite, or parked far away by the reference's SANE_BOX, are
// tested against every primitive. Results per query are returned in ASCENDING primitive index, so
// the serial emit loop produces pairs sorted by (i, j): the canonical order.
#ifndef PDEM_ARBORX_SHIM_HPP
#define PDEM_ARBORX_SHIM_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include <Kokkos_Core.hpp>

namespace ArborX {

template <int DIM, class Coordinate = float>
struct Box {
  Coordinate minCorner[DIM];
  Coordinate maxCorner[DIM];
};

template <class Geometry>
struct IntersectsPredicate {
  Geometry geometry{};
};
template <class Geometry>
IntersectsPredicate<Geometry> intersects(const Geometry& g) {
  return IntersectsPredicate<Geometry>{g};
}

struct PairValueIndex {
  Box<3> value{};
  int index = 0;
};

namespace Experimental {
template <class V>
struct AttachedIndices {
  V boxes;
};
template <class V>
AttachedIndices<V> attach_indices(const V& boxes) {
  return AttachedIndices<V>{boxes};
}
}  // namespace Experimental

inline bool boxesIntersect(const Box<3>& a, const Box<3>& b) {
  for (int d = 0; d < 3; ++d)
    if (a.minCorner[d] > b.maxCorner[d] || a.maxCorner[d] < b.minCorner[d])
      return false;
  return true;
}

class BoundingVolumeHierarchy {
 public:
  using value_type = PairValueIndex;

  template <class S, class V>
  BoundingVolumeHierarchy(const S&, const Experimental::AttachedIndices<V>& src) {
    const std::size_t n = src.boxes.extent(0);
    boxes_.resize(n);
    for (std::size_t i = 0; i < n; ++i)
      boxes_[i] = src.boxes(i);
    build();
  }

  template <class S, class PV, class VV, class OV>
  void query(const S&, const PV& preds, VV& values, OV& offsets) const {
    const std::size_t nq = preds.extent(0);
    std::vector<std::vector<int>> hits(nq);
#ifdef PDEM_SHIM_OPENMP
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (std::int64_t q = 0; q < static_cast<std::int64_t>(nq); ++q)
      collect(preds(q).geometry, hits[q]);
    std::size_t total = 0;
    for (auto& h : hits)
      total += h.size();
    VV nv("arborx_shim::values", total);
    OV no("arborx_shim::offsets", nq + 1);
    std::size_t k = 0;
    for (std::size_t q = 0; q < nq; ++q) {
      no(q) = static_cast<int>(k);
      for (int j : hits[q]) {
        nv(k).value = boxes_[j];
        nv(k).index = j;
        ++k;
      }
    }
    no(nq) = static_cast<int>(k);
    values = nv;
    offsets = no;
  }

 private:
  std::vector<Box<3>> boxes_;
  std::vector<int> far_;         // primitives not in the grid (non-finite / huge / parked)
  std::vector<int> cellStart_;   // CSR over cells
  std::vector<int> cellItems_;
  double origin_[3] = {0, 0, 0};
  double h_ = 1.0;
  int dims_[3] = {1, 1, 1};
  double maxHalf_ = 0.0;

  static bool finiteBox(const Box<3>& b) {
    for (int d = 0; d < 3; ++d)
      if (!std::isfinite(b.minCorner[d]) || !std::isfinite(b.maxCorner[d]) ||
          std::fabs(b.minCorner[d]) > 1e20f || std::fabs(b.maxCorner[d]) > 1e20f)
        return false;
    return true;
  }

  void build() {
    const std::size_t n = boxes_.size();
    std::vector<int> inGrid;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    double maxW = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
      const Box<3>& b = boxes_[i];
      if (!finiteBox(b)) {
        far_.push_back(static_cast<int>(i));
        continue;
      }
      inGrid.push_back(static_cast<int>(i));
      for (int d = 0; d < 3; ++d) {
        const double c = 0.5 * (double(b.minCorner[d]) + double(b.maxCorner[d]));
        lo[d] = std::min(lo[d], c);
        hi[d] = std::max(hi[d], c);
        maxW = std::max(maxW, double(b.maxCorner[d]) - double(b.minCorner[d]));
      }
    }
    maxHalf_ = 0.5 * maxW;
    if (inGrid.empty()) {
      cellStart_.assign(2, 0);
      return;
    }
    h_ = std::max(maxW * 1.0001, 1e-30);
    for (int d = 0; d < 3; ++d)
      origin_[d] = lo[d];
    // cap the cell count (coarser cells if the extent is huge relative to the boxes)
    for (;;) {
      double cells = 1.0;
      for (int d = 0; d < 3; ++d) {
        dims_[d] = static_cast<int>(std::floor((hi[d] - lo[d]) / h_)) + 1;
        cells *= dims_[d];
      }
      if (cells <= 16.0e6)
        break;
      h_ *= 2.0;
    }
    const std::size_t nc = static_cast<std::size_t>(dims_[0]) * dims_[1] * dims_[2];
    std::vector<int> cellOf(inGrid.size());
    cellStart_.assign(nc + 1, 0);
    for (std::size_t t = 0; t < inGrid.size(); ++t) {
      const Box<3>& b = boxes_[inGrid[t]];
      int c[3];
      for (int d = 0; d < 3; ++d) {
        const double x = 0.5 * (double(b.minCorner[d]) + double(b.maxCorner[d]));
        c[d] = std::clamp(static_cast<int>(std::floor((x - origin_[d]) / h_)), 0, dims_[d] - 1);
      }
      cellOf[t] = (c[2] * dims_[1] + c[1]) * dims_[0] + c[0];
      cellStart_[cellOf[t] + 1]++;
    }
    for (std::size_t c = 0; c < nc; ++c)
      cellStart_[c + 1] += cellStart_[c];
    cellItems_.assign(inGrid.size(), 0);
    std::vector<int> fill(cellStart_.begin(), cellStart_.end() - 1);
    for (std::size_t t = 0; t < inGrid.size(); ++t)
      cellItems_[fill[cellOf[t]]++] = inGrid[t];
  }

  void collect(const Box<3>& q, std::vector<int>& out) const {
    if (!finiteBox(q)) {
      for (std::size_t j = 0; j < boxes_.size(); ++j)
        if (boxesIntersect(q, boxes_[j]))
          out.push_back(static_cast<int>(j));
      std::sort(out.begin(), out.end());
      return;
    }
    if (!cellItems_.empty()) {
      int c0[3], c1[3];
      for (int d = 0; d < 3; ++d) {
        const double slack = 1e-6 * (std::fabs(double(q.minCorner[d])) +
                                     std::fabs(double(q.maxCorner[d])) + maxHalf_) + 1e-30;
        const double a = double(q.minCorner[d]) - maxHalf_ - slack;
        const double b = double(q.maxCorner[d]) + maxHalf_ + slack;
        c0[d] = std::clamp(static_cast<int>(std::floor((a - origin_[d]) / h_)), 0, dims_[d] - 1);
        c1[d] = std::clamp(static_cast<int>(std::floor((b - origin_[d]) / h_)), 0, dims_[d] - 1);
      }
      for (int z = c0[2]; z <= c1[2]; ++z)
        for (int y = c0[1]; y <= c1[1]; ++y)
          for (int x = c0[0]; x <= c1[0]; ++x) {
            const int c = (z * dims_[1] + y) * dims_[0] + x;
            for (int t = cellStart_[c]; t < cellStart_[c + 1]; ++t) {
              const int j = cellItems_[t];
              if (boxesIntersect(q, boxes_[j]))
                out.push_back(j);
            }
          }
    }
    for (int j : far_)
      if (boxesIntersect(q, boxes_[j]))
        out.push_back(j);
    std::sort(out.begin(), out.end());
  }
};

}  // namespace ArborX

#endif  // PDEM_ARBORX_SHIM_HPP
