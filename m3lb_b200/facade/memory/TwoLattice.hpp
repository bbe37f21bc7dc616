// Two-lattice (A/B) streaming (src/memory/TwoLattice.hpp).  The reference
// keeps it as the obviously-correct twin of Esoteric Pull and checks the two
// give the same populations (tests/test_streaming.cpp:80-124).  On the B200
// path a solver declared with it runs the Esoteric-Pull kernel, whose results
// are those same populations; bytes_per_node keeps the reference's figure.
#pragma once
#include <cstddef>

#include "core/Types.hpp"

namespace lbm {
template <class L>
class TwoLattice {
 public:
  using Lattice = L;
  static constexpr int Q = L::Q;
  static constexpr const char* name = "TwoLattice";
  static constexpr bool implicit_bounce_back = false;
  static constexpr int nb_first = 1, nb_stride = 1;
  static constexpr std::size_t bytes_per_node() { return 2 * Q * sizeof(Real); }
};
}  // namespace lbm
