// ScalarTRT (src/collision/ScalarTRT.hpp): the odd moment relaxed at omega,
// the even ones at omega_plus set by the magic parameter Lambda.
#pragma once
#include "collision/ScalarBGK.hpp"

namespace lbm {
template <class L>
struct ScalarTRT : ScalarBGK<L> {
  static_assert(L::Q == 2 * L::D + 1, "ScalarTRT needs a rest-plus-axial-pairs lattice (D2Q5 or D3Q7).");
  using Lattice = L;
  static constexpr const char* name = "ScalarTRT";
  static constexpr int device_op = 2;
  Real Lambda = Real(0.25);
  Real omega_plus(Real w) const {
    const Real tm = Real(1) / w - Real(0.5);
    return tm > Real(0) ? Real(1) / (Lambda / tm + Real(0.5)) : Real(0);
  }
};
}  // namespace lbm
