// Plane Poiseuille through the C++ drop-in headers (m3lb_b200/facade): the
// reference-style call sequence -- Domain, policy types, FluidSolver,
// set_geometry, initialize, step, compute_macroscopic, host mirrors -- run on
// the GPU.  Prints the relative L2 error against the analytic parabola, the
// mean fluid density and the mass drift.
//   usage: facade_poiseuille <op: bgk|trt|cm|mrt> <tau> <steps> [f16]
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "collision/BGK.hpp"
#include "collision/MomentCollision.hpp"
#include "collision/TRT.hpp"
#include "memory/EsotericPull.hpp"
#include "solver/FluidSolver.hpp"

using namespace lbm;
using L = D2Q9;

template <class Coll, class Store, class Setup>
int run(double tau, int steps, Setup setup) {
  const Index H = 32, nx = 8, ny = H + 2;
  const double nu = (tau - 0.5) / 3.0, umax = 0.01;
  const double G = 8.0 * nu * umax / double(H * H);
  Domain d(nx, ny, 1, true, false, true);
  Coll coll;
  setup(coll, Real(1.0 / tau));
  coll.forcing = Guo{Real(G), Real(0), Real(0)};
  FluidSolver<L, EsotericPull<L>, Coll, Store> s(d, coll);
  s.set_geometry([&](Index, Index y, Index) -> CellType {
    return (y == 0 || y == ny - 1) ? Solid : Fluid;
  });
  s.initialize(Real(1));
  const double m0 = double(s.total_mass());
  for (int t = 0; t < steps; ++t) s.step();
  Kokkos::fence();
  s.compute_macroscopic();
  auto hu = Kokkos::create_mirror_view_and_copy(HostSpace{}, s.ux());
  auto hr = Kokkos::create_mirror_view_and_copy(HostSpace{}, s.rho());
  double rs = 0;
  for (Index j = 1; j <= H; ++j) rs += double(hr(d.id(nx / 2, j)));
  const double rm = rs / H, A = G / (2 * rm * nu);
  double num = 0, den = 0;
  for (Index j = 1; j <= H; ++j) {
    const double ana = A * (j - 0.5) * (H + 0.5 - j);
    const double e = double(hu(d.id(nx / 2, j))) - ana;
    num += e * e;
    den += ana * ana;
  }
  std::printf("l2 %.6e rho_mean %.12f mass_drift %.3e steps %zu\n", std::sqrt(num / den), rm,
              double(s.total_mass()) / m0 - 1.0, s.timestep());
  return 0;
}

int main(int argc, char** argv) {
  Kokkos::initialize(argc, argv);
  const std::string op = argc > 1 ? argv[1] : "bgk";
  const double tau = argc > 2 ? std::atof(argv[2]) : 0.8;
  const int steps = argc > 3 ? std::atoi(argv[3]) : 60000;
  const bool f16 = argc > 4 && std::strcmp(argv[4], "f16") == 0;
  using SS = ShiftedPopulations;
  auto plain = [](auto& c, Real w) { c.omega = w; };
  auto trt = [](auto& c, Real w) {
    using T = std::decay_t<decltype(c)>;
    c.omega_p = w;
    c.omega_m = T::omega_minus_for(w, T::magic_3_16);
  };
  int rc = 2;
  if (op == "bgk")
    rc = f16 ? run<BGK<L, SecondOrderEquilibrium<L>, Guo, SS>, StoreF16>(tau, steps, plain)
             : run<BGK<L, SecondOrderEquilibrium<L>, Guo, SS>, StoreF64>(tau, steps, plain);
  else if (op == "trt")
    rc = run<TRT<L, SecondOrderEquilibrium<L>, Guo, SS>, StoreF64>(tau, steps, trt);
  else if (op == "cm")
    rc = run<CentralMoments<L, Guo, SS>, StoreF64>(tau, steps, plain);
  else if (op == "mrt")
    rc = run<MRT<L, Guo, SS>, StoreF64>(tau, steps, plain);
  Kokkos::finalize();
  return rc;
}
