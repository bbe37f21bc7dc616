// Equilibrium policies (names of src/equilibrium/Equilibrium.hpp).  They
// select the equilibrium the device kernel evaluates for BGK and TRT, and
// evaluate it on the host for callers that build reference states.
#pragma once
#include "core/Types.hpp"
#include "lattice/Lattices.hpp"

namespace lbm {
// phi = (c.u)/cs2 + (c.u)^2/(2 cs4) - u.u/(2 cs2)
template <class L> struct SecondOrderPhi {
  static constexpr const char* name = "SecondOrder";
  static constexpr int device_code = 0;
  static Real phi(int i, Real ux, Real uy, Real uz) {
    const Real cu = cvel<L>(i, 0) * ux + cvel<L>(i, 1) * uy + cvel<L>(i, 2) * uz;
    const Real uu = ux * ux + uy * uy + uz * uz;
    return Real(3) * cu + Real(4.5) * cu * cu - Real(1.5) * uu;
  }
};
// phi = prod_a chi(c_a, u_a) - 1 with chi(0, u) = 1 - 3u^2/2 and
// chi(+-1, u) = 1 + 3u(c + u): the product of the 1-D equilibria over their weights
template <class L> struct ProductFormPhi {
  static constexpr const char* name = "ProductForm";
  static constexpr int device_code = 1;
  static Real chi(int c, Real u) {
    return c == 0 ? Real(1) - Real(1.5) * u * u : Real(1) + Real(3) * u * (Real(c) + u);
  }
  static Real phi(int i, Real ux, Real uy, Real uz) {
    Real p = chi(cvel<L>(i, 0), ux) * chi(cvel<L>(i, 1), uy);
    if (L::D == 3) p *= chi(cvel<L>(i, 2), uz);
    return p - Real(1);
  }
};
template <class L, class Phi> struct Equilibrium {
  using Lattice = L;
  static constexpr const char* name = Phi::name;
  static constexpr int device_code = Phi::device_code;
  static Real eq(int i, Real rho, Real ux, Real uy, Real uz) {
    return weight<L, Real>(i) * rho * (Real(1) + Phi::phi(i, ux, uy, uz));
  }
  // drho = rho - 1
  static Real eq_shifted(int i, Real drho, Real ux, Real uy, Real uz) {
    return weight<L, Real>(i) * (drho + (Real(1) + drho) * Phi::phi(i, ux, uy, uz));
  }
};
template <class L> using SecondOrderEquilibrium = Equilibrium<L, SecondOrderPhi<L>>;
template <class L> using ProductFormEquilibrium = Equilibrium<L, ProductFormPhi<L>>;
template <class L> struct BestEquilibriumOf { using type = SecondOrderEquilibrium<L>; };
template <> struct BestEquilibriumOf<D2Q9> { using type = ProductFormEquilibrium<D2Q9>; };
template <> struct BestEquilibriumOf<D3Q27> { using type = ProductFormEquilibrium<D3Q27>; };
template <class L> using HighOrderEquilibrium = typename BestEquilibriumOf<L>::type;
}  // namespace lbm
