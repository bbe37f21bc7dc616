// The factorised moment basis {1, C, C^2 - cs2} of src/collision/ProductBasis.hpp
// is evaluated inside the device kernel; this header only keeps the include
// path and the basis size available to code that names it.
#pragma once
#include "lattice/Lattices.hpp"

namespace lbm {
template <class L> struct ProductBasis {
  static constexpr bool enabled = true;
  static constexpr int D = L::D;
  static constexpr int NM = (D == 2) ? 9 : 27;
};
}  // namespace lbm
