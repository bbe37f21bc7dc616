// Esoteric Pull streaming (src/memory/EsotericPull.hpp): one population array
// updated in place.  On the B200 path it is a policy tag; the streaming runs
// inside the fused kernel of libm3lb.so.
#pragma once
#include <cstddef>

#include "core/Types.hpp"

namespace lbm {
template <class L>
class EsotericPull {
 public:
  using Lattice = L;
  static constexpr int Q = L::Q;
  static constexpr const char* name = "EsotericPull";
  static constexpr bool implicit_bounce_back = true;
  static constexpr int nb_first = 1, nb_stride = 2;
  static constexpr std::size_t bytes_per_node() { return Q * sizeof(Real); }
};
}  // namespace lbm
