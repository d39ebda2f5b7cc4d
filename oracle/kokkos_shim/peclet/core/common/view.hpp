// Shim for peclet-core's toVector (test infrastructure): contiguous host copy of a View's elements.
#pragma once
#include <vector>
#include <Kokkos_Core.hpp>
namespace peclet::core {
template <class V>
std::vector<typename V::non_const_value_type> toVector(const V& v) {
  return std::vector<typename V::non_const_value_type>(v.data(), v.data() + v.size());
}
}  // namespace peclet::core
