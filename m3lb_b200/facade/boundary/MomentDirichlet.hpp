// The on-node Dirichlet scalar wall (names of src/boundary/MomentDirichlet.hpp):
// the unknown-direction mask and the moment closure, on the host.  On the
// device they run inside ScalarSolver's step for ScalarMoment cells.
#pragma once
#include <cstdint>

#include "core/Types.hpp"
#include "grid/Domain.hpp"
#include "lattice/Lattices.hpp"

namespace lbm {

// Directions whose source node (x - c_i) lies outside the domain or is not
// part of the field (is_fluid false).
template <class L, class IsFluid>
std::uint32_t unknown_mask(const Domain& d, Index x, Index y, Index z, IsFluid is_fluid) {
  std::uint32_t m = 0;
  const Index p[3] = {x, y, z};
  const Index n[3] = {d.nx, d.ny, d.nz};
  for (int i = 0; i < L::Q; ++i) {
    Index s[3];
    bool outside = false;
    for (int a = 0; a < 3; ++a) {
      s[a] = p[a] - cvel<L>(i, a);
      if (d.periodic[a]) s[a] = (s[a] + n[a]) % n[a];
      else if (s[a] < 0 || s[a] >= n[a]) outside = true;
    }
    if (!outside && !is_fluid(s[0], s[1], s[2])) outside = true;
    if (outside) m |= 1u << i;
  }
  return m;
}

// The unknowns take the deficit target - sum(known) in proportion to their
// weights, so the zeroth moment equals target exactly.
template <class L>
inline void impose_moment(Real g[L::Q], Real target, std::uint32_t unknown) {
  Real known = Real(0), wsum = Real(0);
  for (int i = 0; i < L::Q; ++i) {
    if (unknown & (1u << i)) wsum += weight<L, Real>(i);
    else known += g[i];
  }
  if (!(wsum > Real(0))) return;
  const Real deficit = target - known;
  for (int i = 0; i < L::Q; ++i)
    if (unknown & (1u << i)) g[i] = deficit * weight<L, Real>(i) / wsum;
}

}  // namespace lbm
