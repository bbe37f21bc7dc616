// TRT collision policy (names, members and defaults of src/collision/TRT.hpp).
#pragma once
#include "collision/BGK.hpp"

namespace lbm {

template <class L, class Eq = SecondOrderEquilibrium<L>, class Forcing = NoForcing,
          class Store = RawPopulations>
struct TRT {
  using Lattice = L;
  using Equilibrium = Eq;
  using Storage = Store;
  using ForcingPolicy = Forcing;
  static constexpr const char* name = "TRT";
  static constexpr int device_op = M3LB_OP_TRT;
  static constexpr Real magic_3_16 = Real(3) / Real(16);

  Real omega_p = Real(1);
  Real omega_m = Real(1);
  Forcing forcing{};

  static Real omega_from_viscosity(Real nu) { return Real(1) / (nu * inv_cs2<L, Real>() + Real(0.5)); }
  static Real viscosity_from_omega(Real w) { return (Real(1) / w - Real(0.5)) * cs2<L, Real>(); }
  static Real omega_minus_for(Real omega_plus, Real lambda) {
    return Real(1) / (lambda / (Real(1) / omega_plus - Real(0.5)) + Real(0.5));
  }
  static Real magic_parameter(Real omega_plus, Real omega_minus) {
    return (Real(1) / omega_plus - Real(0.5)) * (Real(1) / omega_minus - Real(0.5));
  }
  static Real density(const Macro& m) { return Store::shifted ? Real(1) + m.dens : m.dens; }
  void device_rates(double& w1, double& w2) const { w1 = omega_p; w2 = omega_m; }
};

}  // namespace lbm
