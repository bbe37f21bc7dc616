// Body-force policies (names of src/forcing/Forcing.hpp).  The B200 path runs
// NoForcing and the uniform Guo force; the members are read at every step,
// so changing `forcing` between steps takes effect on the next one.
#pragma once
#include "core/Types.hpp"

namespace lbm {
struct NoForcing {
  static constexpr const char* name = "None";
  static constexpr bool active = false;
  void at(Index, Real F[3]) const { F[0] = F[1] = F[2] = Real(0); }
};
struct Guo {
  static constexpr const char* name = "Guo";
  static constexpr bool active = true;
  Real fx = Real(0), fy = Real(0), fz = Real(0);
  void at(Index, Real F[3]) const { F[0] = fx; F[1] = fy; F[2] = fz; }
};
}  // namespace lbm
