// Minimal host-only Kokkos API shim (test infrastructure, not product code).
//
// Purpose: compile the peclet-dem reference headers (src/*.hpp) UNMODIFIED with g++ so that the
// reference's own demStep / demStepHertz can be run on the CPU as the parity pin of the oracle, and
// (OpenMP flavour) timed as the CPU baseline. It implements only the API surface those headers use:
// View (rank 0/1/2 with a static trailing extent, const views, shallow reference-counted copies),
// subview/pair/ALL, deep_copy, create_mirror_view (aliasing, as Kokkos does for host spaces),
// resize/realloc/view_alloc/WithoutInitializing, RangePolicy, parallel_for/reduce/scan, atomics,
// Experimental::sort_by_key (stable), sort, math functions, Timer, DefaultExecutionSpace.
//
// Serial flavour (default) executes every parallel construct in ascending index order, so every
// atomic accumulation happens in ascending source index: this is the canonical order the B200
// implementation reproduces with prefix sums and ordered gathers. Define PDEM_SHIM_OPENMP for the
// OpenMP flavour (timing only; its atomic order is non-deterministic like the real backends).
#ifndef PDEM_KOKKOS_SHIM_CORE_HPP
#define PDEM_KOKKOS_SHIM_CORE_HPP

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#ifdef PDEM_SHIM_OPENMP
#include <omp.h>
#endif

#define KOKKOS_LAMBDA [=]
#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_FORCEINLINE_FUNCTION inline

namespace Kokkos {

// ------------------------------------------------------------------------------------------------
// Execution / memory spaces
struct HostSpace {};
struct DefaultExecutionSpace {
  using memory_space = HostSpace;
  using execution_space = DefaultExecutionSpace;
  void fence() const {}
  static const char* name() {
#ifdef PDEM_SHIM_OPENMP
    return "OpenMP";
#else
    return "Serial";
#endif
  }
};
using DefaultHostExecutionSpace = DefaultExecutionSpace;
inline void fence() {}
inline bool& shim_init_flag() {
  static bool f = false;
  return f;
}
inline bool& shim_fin_flag() {
  static bool f = false;
  return f;
}
inline void initialize() { shim_init_flag() = true; }
inline void initialize(int&, char**) { shim_init_flag() = true; }
inline void finalize() { shim_fin_flag() = true; }
inline bool is_initialized() { return shim_init_flag(); }
inline bool is_finalized() { return shim_fin_flag(); }

// ------------------------------------------------------------------------------------------------
// pair / ALL
template <class T1, class T2>
struct pair {
  T1 first;
  T2 second;
  pair() = default;
  pair(T1 a, T2 b) : first(a), second(b) {}
};
template <class T1, class T2>
pair<T1, T2> make_pair(T1 a, T2 b) {
  return pair<T1, T2>(a, b);
}
struct ALL_t {};
inline constexpr ALL_t ALL{};

struct WithoutInitializing_t {};
inline constexpr WithoutInitializing_t WithoutInitializing{};
struct ViewAllocProp {
  std::string label;
};
inline void va_collect(ViewAllocProp&) {}
template <class A, class... R>
void va_collect(ViewAllocProp& p, const A& a, const R&... r) {
  if constexpr (std::is_convertible_v<A, std::string>)
    p.label = std::string(a);
  va_collect(p, r...);
}
template <class... A>
ViewAllocProp view_alloc(const A&... a) {
  ViewAllocProp p;
  va_collect(p, a...);
  return p;
}

// ------------------------------------------------------------------------------------------------
// View
namespace Impl {
template <class D>
struct DataTraits {
  using value_type = D;
  static constexpr int rank = 0;
  static constexpr std::size_t ext1 = 1;
};
template <class T>
struct DataTraits<T*> {
  using value_type = T;
  static constexpr int rank = 1;
  static constexpr std::size_t ext1 = 1;
};
template <class T, std::size_t N>
struct DataTraits<T* [N]> {
  using value_type = T;
  static constexpr int rank = 2;
  static constexpr std::size_t ext1 = N;
};
template <class T>
struct Store {
  std::vector<T> v;
};
}  // namespace Impl

template <class DataType, class... Props>
class View {
 public:
  using traits = Impl::DataTraits<DataType>;
  using value_type = typename traits::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  using data_type = DataType;
  using memory_space = HostSpace;
  using HostMirror = View;
  static constexpr int rank = traits::rank;
  static constexpr std::size_t ext1 = traits::ext1;

  View() = default;
  explicit View(const std::string& label, std::size_t n0 = (rank == 0 ? 1 : 0)) {
    allocate(label, rank == 0 ? 1 : n0);
  }
  explicit View(const char* label, std::size_t n0 = (rank == 0 ? 1 : 0)) {
    allocate(label, rank == 0 ? 1 : n0);
  }
  View(const ViewAllocProp& p, std::size_t n0 = (rank == 0 ? 1 : 0)) {
    allocate(p.label, rank == 0 ? 1 : n0);
  }
  // non-const -> const (and same-type) conversion, sharing storage.
  template <class D2, class... P2,
            class = std::enable_if_t<std::is_convertible_v<
                typename Impl::DataTraits<D2>::value_type*, value_type*>>>
  View(const View<D2, P2...>& o)
      : store_(o.store_), ptr_(o.ptr_), n0_(o.n0_), label_(o.label_) {
    static_assert(Impl::DataTraits<D2>::rank == rank, "rank mismatch");
    static_assert(Impl::DataTraits<D2>::ext1 == ext1, "extent mismatch");
  }
  // unmanaged wrap (used by the shim's own helpers)
  View(value_type* p, std::size_t n0) : ptr_(p), n0_(n0) {}

  value_type& operator()() const { return ptr_[0]; }
  value_type& operator()(std::size_t i) const { return ptr_[i]; }
  value_type& operator()(std::size_t i, std::size_t j) const { return ptr_[i * ext1 + j]; }
  value_type& operator[](std::size_t i) const { return ptr_[i]; }

  std::size_t extent(int r) const { return r == 0 ? n0_ : (r == 1 ? ext1 : 1); }
  int extent_int(int r) const { return static_cast<int>(extent(r)); }
  std::size_t size() const { return n0_ * ext1; }
  std::size_t span() const { return size(); }
  value_type* data() const { return ptr_; }
  const std::string& label() const { return label_; }
  bool is_allocated() const { return ptr_ != nullptr; }

  // shim internals (public so conversions / helpers can reach them)
  std::shared_ptr<Impl::Store<non_const_value_type>> store_;
  value_type* ptr_ = nullptr;
  std::size_t n0_ = 0;
  std::string label_;

  void allocate(const std::string& label, std::size_t n0) {
    label_ = label;
    n0_ = n0;
    store_ = std::make_shared<Impl::Store<non_const_value_type>>();
    store_->v.assign(n0 * ext1, non_const_value_type{});
    ptr_ = store_->v.empty() ? nullptr : store_->v.data();
  }
};

template <class T>
struct is_view : std::false_type {};
template <class D, class... P>
struct is_view<View<D, P...>> : std::true_type {};
template <class T>
inline constexpr bool is_view_v = is_view<std::remove_cv_t<std::remove_reference_t<T>>>::value;

// subview: rank-1 range, or rank-2 row range + ALL
template <class D, class... P, class I1, class I2>
View<D, P...> subview(const View<D, P...>& v, const pair<I1, I2>& r) {
  View<D, P...> s = v;
  s.ptr_ = v.ptr_ + static_cast<std::size_t>(r.first) * View<D, P...>::ext1;
  s.n0_ = static_cast<std::size_t>(r.second - r.first);
  return s;
}
template <class D, class... P, class I1, class I2>
View<D, P...> subview(const View<D, P...>& v, const pair<I1, I2>& r, ALL_t) {
  return subview(v, r);
}
template <class D, class... P, class I1, class I2>
View<D, P...> subview(const View<D, P...>& v, const std::pair<I1, I2>& r) {
  return subview(v, pair<I1, I2>(r.first, r.second));
}

template <class V>
V create_mirror_view(const V& v) {
  return v;  // host memory: the mirror aliases the view (as Kokkos does for host spaces)
}
template <class S, class V>
V create_mirror_view(const S&, const V& v) {
  return v;
}

// deep_copy ------------------------------------------------------------------------------------
template <class D, class... P, class U>
std::enable_if_t<!is_view_v<U>> deep_copy(const View<D, P...>& dst, const U& val) {
  using T = typename View<D, P...>::non_const_value_type;
  const T t = static_cast<T>(val);
  for (std::size_t i = 0; i < dst.size(); ++i)
    dst.ptr_[i] = t;
}
template <class T, class D, class... P>
std::enable_if_t<!is_view_v<T>> deep_copy(T& dst, const View<D, P...>& src) {
  dst = static_cast<T>(src());
}
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.ptr_ == src.ptr_)
    return;
  const std::size_t n = std::min(dst.size(), src.size());
  for (std::size_t i = 0; i < n; ++i)
    dst.ptr_[i] = src.ptr_[i];
}
template <class A, class B>
std::enable_if_t<is_view_v<A> || is_view_v<B>> deep_copy(const DefaultExecutionSpace&, A&& dst,
                                                          B&& src) {
  deep_copy(std::forward<A>(dst), std::forward<B>(src));
}

template <class D, class... P>
void resize(View<D, P...>& v, std::size_t n) {
  using V = View<D, P...>;
  V nv(v.label_, n);
  const std::size_t m = std::min(v.size(), nv.size());
  for (std::size_t i = 0; i < m; ++i)
    nv.ptr_[i] = v.ptr_[i];
  v = nv;
}
template <class D, class... P>
void resize(WithoutInitializing_t, View<D, P...>& v, std::size_t n) {
  resize(v, n);
}
template <class D, class... P>
void realloc(View<D, P...>& v, std::size_t n) {
  v = View<D, P...>(v.label_, n);
}
template <class D, class... P>
void realloc(WithoutInitializing_t, View<D, P...>& v, std::size_t n) {
  realloc(v, n);
}

// ------------------------------------------------------------------------------------------------
// Policies and parallel constructs
template <class... Args>
struct RangePolicy {
  std::int64_t b = 0, e = 0;
  RangePolicy(std::int64_t begin, std::int64_t end) : b(begin), e(end) {}
  template <class S, class = std::enable_if_t<std::is_class_v<S>>>
  RangePolicy(const S&, std::int64_t begin, std::int64_t end) : b(begin), e(end) {}
};

template <class... A, class F>
void parallel_for(const std::string&, const RangePolicy<A...>& p, const F& f) {
#ifdef PDEM_SHIM_OPENMP
#pragma omp parallel for schedule(static)
  for (std::int64_t i = p.b; i < p.e; ++i)
    f(static_cast<int>(i));
#else
  for (std::int64_t i = p.b; i < p.e; ++i)
    f(static_cast<int>(i));
#endif
}
template <class F>
void parallel_for(const std::string& l, std::int64_t n, const F& f) {
  parallel_for(l, RangePolicy<DefaultExecutionSpace>(0, n), f);
}

template <class T>
struct Max {
  using value_type = T;
  T& ref;
  explicit Max(T& r) : ref(r) {}
  static T identity() { return std::numeric_limits<T>::lowest(); }
  static void join(T& a, const T& b) {
    if (b > a)
      a = b;
  }
};
template <class T>
struct Min {
  using value_type = T;
  T& ref;
  explicit Min(T& r) : ref(r) {}
  static T identity() { return std::numeric_limits<T>::max(); }
  static void join(T& a, const T& b) {
    if (b < a)
      a = b;
  }
};
template <class T>
struct Sum {
  using value_type = T;
  T& ref;
  explicit Sum(T& r) : ref(r) {}
  static T identity() { return T{}; }
  static void join(T& a, const T& b) { a += b; }
};

namespace Impl {
template <class R>
struct is_reducer : std::false_type {};
template <class T>
struct is_reducer<Max<T>> : std::true_type {};
template <class T>
struct is_reducer<Min<T>> : std::true_type {};
template <class T>
struct is_reducer<Sum<T>> : std::true_type {};

template <class Red, class... A, class F>
void reduce_impl(const RangePolicy<A...>& p, const F& f, typename Red::value_type& out) {
  using T = typename Red::value_type;
#ifdef PDEM_SHIM_OPENMP
  const int nt = omp_get_max_threads();
  std::vector<T> part(nt, Red::identity());
#pragma omp parallel
  {
    const int t = omp_get_thread_num();
    T acc = Red::identity();
#pragma omp for schedule(static)
    for (std::int64_t i = p.b; i < p.e; ++i)
      f(static_cast<int>(i), acc);
    part[t] = acc;
  }
  T acc = Red::identity();
  for (int t = 0; t < nt; ++t)
    Red::join(acc, part[t]);
  out = acc;
#else
  T acc = Red::identity();
  for (std::int64_t i = p.b; i < p.e; ++i)
    f(static_cast<int>(i), acc);
  out = acc;
#endif
}
}  // namespace Impl

template <class... A, class F, class R>
void parallel_reduce(const std::string&, const RangePolicy<A...>& p, const F& f, R&& r) {
  using RR = std::remove_cv_t<std::remove_reference_t<R>>;
  if constexpr (Impl::is_reducer<RR>::value) {
    Impl::reduce_impl<RR>(p, f, r.ref);
  } else {
    Impl::reduce_impl<Sum<RR>>(p, f, r);
  }
}
template <class F, class R>
void parallel_reduce(const std::string& l, std::int64_t n, const F& f, R&& r) {
  parallel_reduce(l, RangePolicy<DefaultExecutionSpace>(0, n), f, std::forward<R>(r));
}

template <class... A, class F, class T>
void parallel_scan(const std::string&, const RangePolicy<A...>& p, const F& f, T& total) {
  T run{};
  for (std::int64_t i = p.b; i < p.e; ++i)
    f(static_cast<int>(i), run, true);
  total = run;
}
template <class... A, class F>
void parallel_scan(const std::string& l, const RangePolicy<A...>& p, const F& f) {
  using T = int;
  T total;
  parallel_scan(l, p, f, total);
}

// ------------------------------------------------------------------------------------------------
// Atomics
template <class T>
using nd_t = std::type_identity_t<T>;
#ifdef PDEM_SHIM_OPENMP
template <class T>
inline void atomic_add(T* p, nd_t<T> v) {
  std::atomic_ref<T> a(*p);
  if constexpr (std::is_integral_v<T>) {
    a.fetch_add(v, std::memory_order_relaxed);
  } else {
    T old = a.load(std::memory_order_relaxed);
    while (!a.compare_exchange_weak(old, old + v, std::memory_order_relaxed)) {
    }
  }
}
template <class T>
inline T atomic_fetch_add(T* p, nd_t<T> v) {
  std::atomic_ref<T> a(*p);
  if constexpr (std::is_integral_v<T>) {
    return a.fetch_add(v, std::memory_order_relaxed);
  } else {
    T old = a.load(std::memory_order_relaxed);
    while (!a.compare_exchange_weak(old, old + v, std::memory_order_relaxed)) {
    }
    return old;
  }
}
template <class T>
inline T atomic_fetch_max(T* p, nd_t<T> v) {
  std::atomic_ref<T> a(*p);
  T old = a.load(std::memory_order_relaxed);
  while (v > old && !a.compare_exchange_weak(old, v, std::memory_order_relaxed)) {
  }
  return old;
}
template <class T>
inline T atomic_fetch_min(T* p, nd_t<T> v) {
  std::atomic_ref<T> a(*p);
  T old = a.load(std::memory_order_relaxed);
  while (v < old && !a.compare_exchange_weak(old, v, std::memory_order_relaxed)) {
  }
  return old;
}
#else
template <class T>
inline void atomic_add(T* p, nd_t<T> v) {
  *p += v;
}
template <class T>
inline T atomic_fetch_add(T* p, nd_t<T> v) {
  T o = *p;
  *p += v;
  return o;
}
template <class T>
inline T atomic_fetch_max(T* p, nd_t<T> v) {
  T o = *p;
  if (v > o)
    *p = v;
  return o;
}
template <class T>
inline T atomic_fetch_min(T* p, nd_t<T> v) {
  T o = *p;
  if (v < o)
    *p = v;
  return o;
}
#endif
template <class T>
inline void atomic_max(T* p, nd_t<T> v) {
  atomic_fetch_max(p, v);
}
template <class T>
inline void atomic_min(T* p, nd_t<T> v) {
  atomic_fetch_min(p, v);
}
template <class T>
inline void atomic_increment(T* p) {
  atomic_add(p, T(1));
}

// ------------------------------------------------------------------------------------------------
// Math
inline float sqrt(float x) { return std::sqrt(x); }
inline double sqrt(double x) { return std::sqrt(x); }
inline float fabs(float x) { return std::fabs(x); }
inline double fabs(double x) { return std::fabs(x); }
inline float fmin(float a, float b) { return std::fmin(a, b); }
inline double fmin(double a, double b) { return std::fmin(a, b); }
inline float fmax(float a, float b) { return std::fmax(a, b); }
inline double fmax(double a, double b) { return std::fmax(a, b); }
inline float log(float x) { return std::log(x); }
inline double log(double x) { return std::log(x); }
inline float exp(float x) { return std::exp(x); }
inline double exp(double x) { return std::exp(x); }
inline float floor(float x) { return std::floor(x); }
inline double floor(double x) { return std::floor(x); }
inline float ceil(float x) { return std::ceil(x); }
inline double ceil(double x) { return std::ceil(x); }
inline float pow(float a, float b) { return std::pow(a, b); }
inline double pow(double a, double b) { return std::pow(a, b); }
template <class T>
inline T max(const T& a, const T& b) {
  return a < b ? b : a;
}
template <class T>
inline T min(const T& a, const T& b) {
  return b < a ? b : a;
}
inline bool isfinite(float x) { return std::isfinite(x); }
inline bool isfinite(double x) { return std::isfinite(x); }
inline bool isnan(float x) { return std::isnan(x); }
inline bool isnan(double x) { return std::isnan(x); }

// ------------------------------------------------------------------------------------------------
// Sorting (stable: equal keys keep their original relative order)
namespace Experimental {
template <class S, class KV, class VV>
void sort_by_key(const S&, const KV& keys, const VV& values) {
  const std::size_t n = keys.extent(0);
  std::vector<std::size_t> idx(n);
  std::iota(idx.begin(), idx.end(), std::size_t(0));
  std::stable_sort(idx.begin(), idx.end(),
                   [&](std::size_t a, std::size_t b) { return keys(a) < keys(b); });
  std::vector<typename KV::non_const_value_type> k(n);
  std::vector<typename VV::non_const_value_type> v(n);
  for (std::size_t i = 0; i < n; ++i) {
    k[i] = keys(idx[i]);
    v[i] = values(idx[i]);
  }
  for (std::size_t i = 0; i < n; ++i) {
    keys(i) = k[i];
    values(i) = v[i];
  }
}
}  // namespace Experimental
template <class S, class V>
void sort(const S&, const V& v) {
  std::stable_sort(v.data(), v.data() + v.extent(0));
}
template <class V>
void sort(const V& v) {
  std::stable_sort(v.data(), v.data() + v.extent(0));
}

// ------------------------------------------------------------------------------------------------
class Timer {
  std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();

 public:
  void reset() { t0_ = std::chrono::steady_clock::now(); }
  double seconds() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }
};

}  // namespace Kokkos

#endif  // PDEM_KOKKOS_SHIM_CORE_HPP
