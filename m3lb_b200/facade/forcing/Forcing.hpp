// Body-force policies (names of src/forcing/Forcing.hpp).  The B200 path runs
// NoForcing, the uniform Guo force and Boussinesq buoyancy; the members are
// read at every step, so changing `forcing` between steps takes effect on the
// next one.
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
// Boussinesq buoyancy through the Guo machinery: F(n) = (fx, fy, fz) + g rho0
// beta (T(n) - T0).  T is read at every step; a view handed out by a scalar
// solver (ScalarSolver::temperature()) is read on the device directly, any
// other view is copied up before each step.
struct BoussinesqGuo {
  static constexpr const char* name = "Boussinesq";
  static constexpr bool active = true;
  View1D<Real> T;
  Real gx = Real(0), gy = Real(-1), gz = Real(0);
  Real rho0 = Real(1), beta = Real(1), T0 = Real(0);
  Real fx = Real(0), fy = Real(0), fz = Real(0);
  void at(Index n, Real F[3]) const {
    const Real b = rho0 * beta * (T(n) - T0);
    F[0] = fx + gx * b; F[1] = fy + gy * b; F[2] = fz + gz * b;
  }
};
}  // namespace lbm
