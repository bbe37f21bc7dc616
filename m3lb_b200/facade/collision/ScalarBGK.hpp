// Scalar (advection-diffusion) collision policies and cell types: the names
// of src/collision/ScalarBGK.hpp.  The operator itself runs on the device in
// ScalarSolver's step; the members here are its parameters, and eq /
// deviation / temperature evaluate the same formulas on the host.
#pragma once
#include <cstdint>

#include "core/Types.hpp"
#include "lattice/Lattices.hpp"
#include "memory/Storage.hpp"

namespace lbm {

template <class L>
struct ScalarBGK {
  using Lattice = L;
  using Storage = RawPopulations;
  static constexpr const char* name = "ScalarBGK";
  static constexpr int device_op = 1;

  Real omega = Real(1);
  Real T_ref = Real(0);      // storage reference: populations hold g - w T_ref
  View1D<Real> omega_of;     // optional rate per padded node; empty means uniform

  // D = cs2 (1/omega - 1/2)
  static Real omega_from_diffusivity(Real d) { return Real(1) / (d * inv_cs2<L, Real>() + Real(0.5)); }
  static Real diffusivity_from_omega(Real w) { return (Real(1) / w - Real(0.5)) * cs2<L, Real>(); }

  static Real deviation(const Real h[L::Q]) {
    Real t = Real(0);
    for (int i = 0; i < L::Q; ++i) t += h[i];
    return t;
  }
  Real temperature(const Real h[L::Q]) const { return T_ref + deviation(h); }
  // w_i (dT + (T_ref + dT) c_i.u / cs2)
  Real eq(int i, Real dT, Real ux, Real uy, Real uz) const {
    const Real cu = Real(cvel<L>(i, 0)) * ux + Real(cvel<L>(i, 1)) * uy + Real(cvel<L>(i, 2)) * uz;
    return weight<L, Real>(i) * (dT + (T_ref + dT) * inv_cs2<L, Real>() * cu);
  }
  Real omega_at(Index n) const { return omega_of.data() ? omega_of(n) : omega; }
};

enum ScalarCell : std::uint8_t {
  ScalarBulk = 0,
  ScalarAdiabatic = 1,
  ScalarDirichlet = 2,
  ScalarExcluded = 3,
  ScalarMoment = 4,
  ScalarOutflow = 5,
  ScalarSpecular = 6,
};

}  // namespace lbm
