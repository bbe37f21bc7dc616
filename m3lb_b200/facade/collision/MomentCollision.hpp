// Moment-space collision policy: central moments (Central = true) or raw MRT
// (names, members and defaults of src/collision/MomentCollision.hpp).
#pragma once
#include "collision/BGK.hpp"
#include "collision/ProductBasis.hpp"

namespace lbm {

template <class L, class Forcing = NoForcing, class Store = RawPopulations, bool Central = true>
struct MomentCollision {
  using Lattice = L;
  using Storage = Store;
  using ForcingPolicy = Forcing;
  using Equilibrium = SecondOrderEquilibrium<L>;  // unused: the equilibrium is closed-form
  static constexpr const char* name = Central ? "CentralMoments" : "MRT";
  static constexpr int device_op = Central ? M3LB_OP_CM : M3LB_OP_MRT;
  static constexpr int D = L::D;
  static constexpr int NM = ProductBasis<L>::NM;

  Real omega = Real(1);
  Real omega_bulk = Real(-1);
  Forcing forcing{};

  static Real omega_from_viscosity(Real nu) { return Real(1) / (nu * inv_cs2<L, Real>() + Real(0.5)); }
  static Real viscosity_from_omega(Real w) { return (Real(1) / w - Real(0.5)) * cs2<L, Real>(); }
  Real bulk() const { return omega_bulk < Real(0) ? omega : omega_bulk; }
  static Real density(const Macro& m) { return Store::shifted ? Real(1) + m.dens : m.dens; }
  void device_rates(double& w1, double& w2) const { w1 = omega; w2 = omega_bulk; }
};

template <class L, class F = NoForcing, class S = RawPopulations>
using CentralMoments = MomentCollision<L, F, S, true>;
template <class L, class F = NoForcing, class S = RawPopulations>
using MRT = MomentCollision<L, F, S, false>;

}  // namespace lbm
