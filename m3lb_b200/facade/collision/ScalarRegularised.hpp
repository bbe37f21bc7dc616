// ScalarRegularised (src/collision/ScalarRegularised.hpp): every even moment
// reset to its equilibrium, the flux relaxed at omega.
#pragma once
#include "collision/ScalarBGK.hpp"

namespace lbm {
template <class L>
struct ScalarRegularised : ScalarBGK<L> {
  static_assert(L::Q == 2 * L::D + 1,
                "ScalarRegularised needs a rest-plus-axial-pairs lattice (D2Q5 or D3Q7).");
  using Lattice = L;
  static constexpr const char* name = "ScalarRegularised";
  static constexpr int device_op = 3;
};
}  // namespace lbm
