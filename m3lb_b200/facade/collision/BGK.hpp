// BGK collision policy (names, members and defaults of
// src/collision/BGK.hpp): the relaxation itself runs in the fused kernel of
// libm3lb.so; this type carries its parameters and selects the kernel.
#pragma once
#include "core/Types.hpp"
#include "equilibrium/Equilibrium.hpp"
#include "forcing/Forcing.hpp"
#include "lattice/Lattices.hpp"
#include "memory/Storage.hpp"

namespace lbm {

struct Macro {
  Real dens;
  Real ux, uy, uz;
};

template <class L, class Eq = SecondOrderEquilibrium<L>, class Forcing = NoForcing,
          class Store = RawPopulations>
struct BGK {
  using Lattice = L;
  using Equilibrium = Eq;
  using Storage = Store;
  using ForcingPolicy = Forcing;
  static constexpr const char* name = "BGK";
  static constexpr int device_op = M3LB_OP_BGK;

  Real omega = Real(1);
  Forcing forcing{};

  static Real omega_from_viscosity(Real nu) { return Real(1) / (nu * inv_cs2<L, Real>() + Real(0.5)); }
  static Real viscosity_from_omega(Real w) { return (Real(1) / w - Real(0.5)) * cs2<L, Real>(); }
  static Real density(const Macro& m) { return Store::shifted ? Real(1) + m.dens : m.dens; }
  void device_rates(double& w1, double& w2) const { w1 = omega; w2 = -1.0; }
};

}  // namespace lbm
