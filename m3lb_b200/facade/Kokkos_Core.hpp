// Host side of the B200 drop-in: the handful of Kokkos names that code written
// against M3LB's headers uses around the solver (initialize/finalize, fence,
// host views and their mirrors, parallel loops on the host).
//
// With this facade the time step runs in libm3lb.so on the GPU; what remains
// of Kokkos in user code is host bookkeeping, served here:
//   * View<T*> / View<T**>: reference-counted host arrays (last index fastest);
//   * create_mirror_view* return the view itself (it already lives on the host);
//   * fence() waits for every live solver's queued GPU work;
//   * parallel_for / parallel_reduce run on the host, in order.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "m3lb_facade_device.hpp"

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]

namespace Kokkos {

struct HostSpace {
  using memory_space = HostSpace;
  using execution_space = HostSpace;
  static const char* name() { return "Host"; }
};
// The execution space a solver's time step runs on.
struct Cuda {
  using memory_space = HostSpace;  // results are handed back in host arrays
  using execution_space = Cuda;
  static const char* name() { return "CUDA sm_100a (libm3lb)"; }
};
using DefaultExecutionSpace = Cuda;
using DefaultHostExecutionSpace = HostSpace;

namespace facade {
template <class T> struct Rank { static constexpr int value = 0; using type = T; };
template <class T> struct Rank<T*> { static constexpr int value = 1 + Rank<T>::value; using type = typename Rank<T>::type; };
}  // namespace facade

template <class DataType, class... Props>
class View {
 public:
  using value_type = typename facade::Rank<DataType>::type;
  using non_const_value_type = std::remove_const_t<value_type>;
  static constexpr int rank = facade::Rank<DataType>::value;

  View() = default;
  explicit View(const std::string& label, std::size_t n0 = 0, std::size_t n1 = 1)
      : label_(label), n0_(n0), n1_(rank >= 2 ? n1 : 1),
        data_(std::make_shared<std::vector<non_const_value_type>>(n0 * (rank >= 2 ? n1 : 1))) {}
  template <class D2, class... P2>
  View(const View<D2, P2...>& o)
      : label_(o.label_), n0_(o.n0_), n1_(o.n1_), data_(o.data_), dev_(o.dev_),
        dev_stream_(o.dev_stream_) {}

  value_type& operator()(std::size_t i) const { return (*data_)[i]; }
  value_type& operator()(std::size_t i, std::size_t j) const { return (*data_)[i * n1_ + j]; }
  value_type& operator[](std::size_t i) const { return (*data_)[i]; }
  std::size_t extent(int d) const { return d == 0 ? n0_ : (d == 1 ? n1_ : 1); }
  int extent_int(int d) const { return int(extent(d)); }
  std::size_t size() const { return n0_ * n1_; }
  value_type* data() const { return data_ ? data_->data() : nullptr; }
  const std::string& label() const { return label_; }

  std::string label_;
  std::size_t n0_ = 0, n1_ = 1;
  std::shared_ptr<std::vector<non_const_value_type>> data_;
  // A view a solver hands out for a field it holds on the device: that
  // field's device array (one value per interior node, the solver's
  // arithmetic type) and the stream its writes are queued on.  Another
  // solver given this view reads the device array directly.
  const void* dev_ = nullptr;
  void* dev_stream_ = nullptr;
};

template <class V> V create_mirror_view(const V& v) { return v; }
template <class S, class V> V create_mirror_view(const S&, const V& v) { return v; }
template <class S, class V> V create_mirror_view_and_copy(const S&, const V& v) { return v; }
template <class D1, class... P1, class D2, class... P2>
void deep_copy(const View<D1, P1...>& dst, const View<D2, P2...>& src) {
  if (dst.data() != src.data())
    for (std::size_t i = 0; i < dst.size() && i < src.size(); ++i) dst.data()[i] = src.data()[i];
}

template <class D1, class... P1>
void deep_copy(const View<D1, P1...>& dst, const typename View<D1, P1...>::value_type& v) {
  for (std::size_t i = 0; i < dst.size(); ++i) dst.data()[i] = v;
}

template <class Exec = DefaultExecutionSpace>
struct RangePolicy {
  std::int64_t b = 0, e = 0;
  RangePolicy(std::int64_t b_, std::int64_t e_) : b(b_), e(e_) {}
};
template <class F>
void parallel_for(const std::string&, std::int64_t n, const F& f) {
  for (std::int64_t i = 0; i < n; ++i) f(i);
}
template <class E, class F>
void parallel_for(const std::string&, const RangePolicy<E>& p, const F& f) {
  for (std::int64_t i = p.b; i < p.e; ++i) f(i);
}
template <class E, class F, class R>
void parallel_reduce(const std::string&, const RangePolicy<E>& p, const F& f, R& r) {
  R acc = R(0);
  for (std::int64_t i = p.b; i < p.e; ++i) f(i, acc);
  r = acc;
}

// Wait for the GPU work every live solver has queued.
inline void fence() { m3lb_facade::fence_all(); }
inline void fence(const std::string&) { fence(); }
inline void initialize() {}
inline void initialize(int&, char**) {}
inline void finalize() { fence(); }

using std::abs; using std::fabs; using std::sqrt; using std::cos; using std::sin;
using std::tanh; using std::atan; using std::acos; using std::pow; using std::exp;
using std::log; using std::fmax; using std::fmin; using std::floor; using std::isfinite;
template <class T> inline constexpr T max(const T& a, const T& b) { return a < b ? b : a; }
template <class T> inline constexpr T min(const T& a, const T& b) { return b < a ? b : a; }

}  // namespace Kokkos
