// Host-only stand-in for the small part of the Kokkos API that the
// reference's lattice-Boltzmann headers use, so that those headers compile
// unmodified with g++ and OpenMP.  This is test infrastructure for the oracle
// build only: nothing in the product links it.
//
// Semantics follow the Kokkos host backends (Serial / OpenMP):
//   * View<T*> / View<T**>: reference-counted, zero-initialised, LayoutRight
//     (last index fastest), host memory;
//   * create_mirror_view* on a host view returns the same view (shallow);
//   * deep_copy copies element by element when the two views differ;
//   * parallel_for / parallel_reduce run over [begin, end) with OpenMP,
//     parallel_reduce summing per-thread partials in thread order so the
//     result is deterministic for a fixed thread count;
//   * fence / initialize / finalize are no-ops.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct HostSpace {
  using memory_space = HostSpace;
  using execution_space = HostSpace;
};
struct OpenMP {
  using memory_space = HostSpace;
  using execution_space = OpenMP;
  static const char* name() { return "OpenMP"; }
};
using DefaultExecutionSpace = OpenMP;
using DefaultHostExecutionSpace = OpenMP;
struct LayoutRight {};
struct LayoutLeft {};

namespace shim {
template <class T> struct Rank { static constexpr int value = 0; using value_type = T; };
template <class T> struct Rank<T*> { static constexpr int value = 1 + Rank<T>::value; using value_type = typename Rank<T>::value_type; };
}  // namespace shim

template <class DataType, class... Props>
class View {
 public:
  using value_type = typename shim::Rank<DataType>::value_type;
  using non_const_value_type = std::remove_const_t<value_type>;
  static constexpr int rank = shim::Rank<DataType>::value;
  using memory_space = HostSpace;
  using execution_space = OpenMP;

  View() = default;
  explicit View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 0)
      : label_(label), n0_(n0), n1_(rank >= 2 ? n1 : 1) {
    const std::size_t n = n0_ * n1_;
    store_ = std::make_shared<std::vector<non_const_value_type>>(n ? n : 0);
    ptr_ = store_->data();
  }
  // Converting constructor (e.g. View<T*> -> View<const T*>).
  template <class D2, class... P2>
  View(const View<D2, P2...>& o)
      : label_(o.label_), n0_(o.n0_), n1_(o.n1_), store_(o.store_), ptr_(o.ptr_) {}

  KOKKOS_INLINE_FUNCTION value_type& operator()(std::size_t i) const { return ptr_[i]; }
  KOKKOS_INLINE_FUNCTION value_type& operator()(std::size_t i, std::size_t j) const {
    return ptr_[i * n1_ + j];
  }
  KOKKOS_INLINE_FUNCTION value_type& operator[](std::size_t i) const { return ptr_[i]; }
  std::size_t extent(int d) const { return d == 0 ? n0_ : (d == 1 ? (rank >= 2 ? n1_ : 1) : 1); }
  int extent_int(int d) const { return int(extent(d)); }
  std::size_t size() const { return n0_ * n1_; }
  std::size_t span() const { return size(); }
  value_type* data() const { return ptr_; }
  const std::string& label() const { return label_; }
  bool is_allocated() const { return ptr_ != nullptr; }
  long use_count() const { return store_.use_count(); }

  std::string label_;
  std::size_t n0_ = 0, n1_ = 1;
  std::shared_ptr<std::vector<non_const_value_type>> store_;
  value_type* ptr_ = nullptr;
};

template <class V> V create_mirror_view(const V& v) { return v; }
template <class S, class V> V create_mirror_view(const S&, const V& v) { return v; }
template <class S, class V> V create_mirror_view_and_copy(const S&, const V& v) { return v; }
template <class V> V create_mirror(const V& v) {
  V m(v.label(), v.extent(0), v.extent(1));
  return m;
}

template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.data() == src.data()) return;
  const std::size_t n = std::min(dst.size(), src.size());
  for (std::size_t i = 0; i < n; ++i) dst.data()[i] = src.data()[i];
}
template <class D1, class... P1>
void deep_copy(const View<D1, P1...>& dst,
               const typename View<D1, P1...>::non_const_value_type& v) {
  for (std::size_t i = 0; i < dst.size(); ++i) dst.data()[i] = v;
}
template <class D1, class... P1, class D2, class... P2, class E>
void deep_copy(const E&, const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  deep_copy(dst, src);
}

template <class Exec = OpenMP, class... P>
struct RangePolicy {
  std::int64_t b = 0, e = 0;
  RangePolicy() = default;
  RangePolicy(std::int64_t b_, std::int64_t e_) : b(b_), e(e_) {}
  RangePolicy(const Exec&, std::int64_t b_, std::int64_t e_) : b(b_), e(e_) {}
};

namespace shim {
template <class P> inline void bounds(const P& p, std::int64_t& b, std::int64_t& e) { b = p.b; e = p.e; }
inline void bounds(int n, std::int64_t& b, std::int64_t& e) { b = 0; e = n; }
inline void bounds(long n, std::int64_t& b, std::int64_t& e) { b = 0; e = n; }
inline void bounds(unsigned n, std::int64_t& b, std::int64_t& e) { b = 0; e = n; }
inline void bounds(unsigned long n, std::int64_t& b, std::int64_t& e) { b = 0; e = std::int64_t(n); }
}  // namespace shim

template <class P, class F>
void parallel_for(const std::string&, const P& p, const F& f) {
  std::int64_t b, e; shim::bounds(p, b, e);
#pragma omp parallel for schedule(static)
  for (std::int64_t i = b; i < e; ++i) f(i);
}
template <class P, class F>
void parallel_for(const P& p, const F& f) { parallel_for(std::string(), p, f); }

template <class P, class F, class R>
void parallel_reduce(const std::string&, const P& p, const F& f, R& result) {
  std::int64_t b, e; shim::bounds(p, b, e);
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  std::vector<R> part(std::size_t(nt), R(0));
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    R acc = R(0);
#pragma omp for schedule(static)
    for (std::int64_t i = b; i < e; ++i) f(i, acc);
    part[std::size_t(t)] = acc;
  }
  R s = R(0);
  for (const R& v : part) s += v;
  result = s;
}
template <class P, class F, class R>
void parallel_reduce(const P& p, const F& f, R& result) {
  parallel_reduce(std::string(), p, f, result);
}

// Two-dimensional ranges for reductions: rows (first index) split over
// threads in static chunks, the second index fastest.
template <unsigned N> struct Rank {};
template <class RankT>
struct MDRangePolicy {
  std::int64_t b[2] = {0, 0}, e[2] = {0, 0};
  MDRangePolicy(std::initializer_list<std::int64_t> lo, std::initializer_list<std::int64_t> hi) {
    std::size_t k = 0;
    for (auto v : lo) b[k++] = v;
    k = 0;
    for (auto v : hi) e[k++] = v;
  }
};
template <class RankT, class F, class R>
void parallel_reduce(const std::string&, const MDRangePolicy<RankT>& p, const F& f, R& result) {
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  std::vector<R> part(std::size_t(nt), R(0));
#pragma omp parallel num_threads(nt)
  {
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    R acc = R(0);
#pragma omp for schedule(static)
    for (std::int64_t i = p.b[0]; i < p.e[0]; ++i)
      for (std::int64_t j = p.b[1]; j < p.e[1]; ++j) f(i, j, acc);
    part[std::size_t(t)] = acc;
  }
  R s = R(0);
  for (const R& v : part) s += v;
  result = s;
}

inline void fence() {}
inline void fence(const std::string&) {}
inline void initialize() {}
inline void initialize(int&, char**) {}
inline void finalize() {}
inline bool is_initialized() { return true; }

using std::abs; using std::fabs; using std::sqrt; using std::cos; using std::sin;
using std::tanh; using std::atan; using std::acos; using std::pow; using std::exp;
using std::log; using std::fmax; using std::fmin; using std::floor; using std::ceil;
using std::isfinite; using std::isnan; using std::atan2; using std::tan; using std::cbrt;
using std::asin; using std::sinh; using std::cosh; using std::erf; using std::round;
template <class T> KOKKOS_INLINE_FUNCTION constexpr T max(const T& a, const T& b) { return a < b ? b : a; }
template <class T> KOKKOS_INLINE_FUNCTION constexpr T min(const T& a, const T& b) { return b < a ? b : a; }

}  // namespace Kokkos
