// Equilibrium policies (names of src/equilibrium/Equilibrium.hpp).  They
// select the equilibrium the device kernel evaluates for BGK and TRT.
#pragma once
#include "lattice/Lattices.hpp"

namespace lbm {
template <class L> struct SecondOrderPhi {
  static constexpr const char* name = "SecondOrder";
  static constexpr int device_code = 0;
};
template <class L> struct ProductFormPhi {
  static constexpr const char* name = "ProductForm";
  static constexpr int device_code = 1;
};
template <class L, class Phi> struct Equilibrium {
  using Lattice = L;
  static constexpr const char* name = Phi::name;
  static constexpr int device_code = Phi::device_code;
};
template <class L> using SecondOrderEquilibrium = Equilibrium<L, SecondOrderPhi<L>>;
template <class L> using ProductFormEquilibrium = Equilibrium<L, ProductFormPhi<L>>;
template <class L> struct BestEquilibriumOf { using type = SecondOrderEquilibrium<L>; };
template <> struct BestEquilibriumOf<D2Q9> { using type = ProductFormEquilibrium<D2Q9>; };
template <> struct BestEquilibriumOf<D3Q27> { using type = ProductFormEquilibrium<D3Q27>; };
template <class L> using HighOrderEquilibrium = typename BestEquilibriumOf<L>::type;
}  // namespace lbm
