#pragma once
// Shared part of the C-ABI driver over the REFERENCE's own FluidSolver (src/solver/FluidSolver.hpp),
// compiled unmodified against the host Kokkos-API stand-in in kokkos_shim/.
//
// Test infrastructure only: the parity tests and the CPU-baseline leg of
// bench.py load the resulting oracle/_ref/libm3lb_ref_{f32,f64}.so to run the
// reference's arithmetic on the same inputs as the CUDA path.  Nothing in the
// product links or loads it.
//
// Every entry point maps onto one public member of the reference solver:
//   ref_create            FluidSolver(Domain, Collision)      FluidSolver.hpp:42
//   ref_set_geometry      set_geometry(fn(x,y,z) -> CellType)  FluidSolver.hpp:74-82
//   ref_set_specular_walls set_specular_walls(fn -> NormalCode) FluidSolver.hpp:193-218
//   ref_set_specular_nodes set_specular_nodes(fn -> SpecFace)   FluidSolver.hpp:236-268
//   ref_set_regularized_walls set_regularized_walls(fn -> WallSpec) FluidSolver.hpp:372-552
//   ref_set_wall_* / ref_set_fd_corners / ref_set_force_correction / ref_set_outflow_*
//                         the wall setters of FluidSolver.hpp:272-370, 1311-1330
//   ref_initialize        initialize(rho0, ux, uy, uz)         FluidSolver.hpp:553-561
//   ref_initialize_field  initialize_field(fn(n) -> FlowState) FluidSolver.hpp:568-579
//   ref_step              step(store_macroscopic)              FluidSolver.hpp:582-591
//   ref_macro             compute_macroscopic + rho()/ux()..   FluidSolver.hpp:597-599
//   ref_total_mass        total_mass()                          FluidSolver.hpp:601-603
//   ref_total_momentum    total_momentum(a)                     FluidSolver.hpp:604-606
//   ref_gather            gather_populations()                  FluidSolver.hpp:620-624
//   ref_seed              seed_populations(fn(n, i) -> Real)    FluidSolver.hpp:634-637
//   ref_slot_sum          sum over populations().storage()      EsotericPull.hpp:119-123
#include "collision/BGK.hpp"
#include "collision/MomentCollision.hpp"
#include "collision/TRT.hpp"
#include "core/Types.hpp"
#include "grid/Domain.hpp"
#include "memory/EsotericPull.hpp"
#include "memory/TwoLattice.hpp"
#include "solver/FluidSolver.hpp"

#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

using namespace lbm;

namespace refdrv {

// Collision that leaves the populations untouched, so a run is pure streaming.
// Same contract as the NullCollision mock of tests/test_streaming.cpp:28-38.
template <class L>
struct NoCollision {
  using Lattice = L;
  using Equilibrium = SecondOrderEquilibrium<L>;
  using Storage = RawPopulations;
  KOKKOS_INLINE_FUNCTION Macro macroscopic(const Real[L::Q], Index = 0) const {
    return Macro{Real(1), Real(0), Real(0), Real(0)};
  }
  KOKKOS_INLINE_FUNCTION void collide(Real[L::Q], const Macro&, Index = 0) const {}
  KOKKOS_INLINE_FUNCTION static Real density(const Macro& m) { return m.dens; }
  KOKKOS_INLINE_FUNCTION static Real seed_value(int, Real r, Real, Real, Real) { return r; }
};

struct Params {
  double omega = 1, omega2 = -1, fx = 0, fy = 0, fz = 0;
  long long n_padded = 0;
};

// The forcing policy's parameters: the uniform Guo force, or the uniform part
// of BoussinesqGuo with a temperature view of the lattice's size (zero until
// ref_set_buoyancy fills it).
inline void set_force(NoForcing&, const Params&) {}
inline void set_force(Guo& g, const Params& p) { g = Guo{Real(p.fx), Real(p.fy), Real(p.fz)}; }
inline void set_force(BoussinesqGuo& b, const Params& p) {
  b.fx = Real(p.fx); b.fy = Real(p.fy); b.fz = Real(p.fz);
  b.T = View1D<Real>("T", p.n_padded);
}

struct Base {
  virtual ~Base() = default;
  // the driver's own record of the wall codes and the outflow order, for the
  // argument checks of ref_set_regularized_walls / ref_set_outflow_order
  std::vector<std::uint8_t> wall_codes;
  int out_order = 1;
  virtual void set_geometry(const std::uint8_t* flags) = 0;
  virtual void set_specular_walls(const std::uint8_t* codes) = 0;
  virtual void set_specular_nodes(const std::uint8_t* masks) = 0;
  virtual void set_regularized_walls(const std::uint8_t* codes, const double* spec) = 0;
  virtual void set_wall_velocity_scale(double sc) = 0;
  virtual void set_wall_density(double r) = 0;
  virtual void set_wall_velocity_field(const double* u3) = 0;
  virtual void set_wall_velocity_field_scale(double sc) = 0;
  virtual void set_fd_corners(bool on) = 0;
  virtual void set_force_correction(bool on) = 0;
  virtual void set_outflow_order(int k) = 0;
  virtual void set_outflow_density(double r) = 0;
  // BoussinesqGuo solvers only: T per interior node, buoyancy g rho0 beta (T - T0)
  virtual int set_buoyancy(const double*, double, double, double, double, double, double) {
    return -1;
  }
  virtual long long nx() const = 0;
  virtual long long ny() const = 0;
  virtual void initialize(double rho, double ux, double uy, double uz) = 0;
  virtual void initialize_field(const double* rho, const double* ux, const double* uy,
                                const double* uz) = 0;
  virtual void step(int n, int store) = 0;
  virtual void macro(double* rho, double* ux, double* uy, double* uz) = 0;
  virtual void stored_macro(double* rho, double* ux, double* uy, double* uz) = 0;
  virtual double mass() = 0;
  virtual double momentum(int a) = 0;
  virtual void gather(double* out) = 0;
  virtual void seed(const double* in) = 0;
  virtual double slot_sum() = 0;
  virtual long long n_padded() const = 0;
  virtual long long n_interior() const = 0;
  virtual long long timestep() const = 0;
};

template <class Coll> void apply_params(Coll& c, const Params& p);

template <class L, class E, class F, class S>
void apply_params(BGK<L, E, F, S>& c, const Params& p) {
  c.omega = Real(p.omega);
  set_force(c.forcing, p);
}
template <class L, class E, class F, class S>
void apply_params(TRT<L, E, F, S>& c, const Params& p) {
  c.omega_p = Real(p.omega);
  c.omega_m = Real(p.omega2);
  set_force(c.forcing, p);
}
template <class L, class F, class S, bool C>
void apply_params(MomentCollision<L, F, S, C>& c, const Params& p) {
  c.omega = Real(p.omega);
  c.omega_bulk = Real(p.omega2);
  set_force(c.forcing, p);
}
template <class L>
void apply_params(NoCollision<L>&, const Params&) {}

template <class L, class Strm, class Coll>
struct Impl final : Base {
  Domain d;
  FluidSolver<L, Strm, Coll> s;
  static Coll make(const Params& p) { Coll c{}; apply_params(c, p); return c; }
  Impl(const Domain& dom, const Params& p) : d(dom), s(dom, make(p)) {}

  void set_geometry(const std::uint8_t* flags) override {
    const Domain dd = d;
    s.set_geometry([&](Index x, Index y, Index z) -> CellType {
      return CellType(flags[(std::size_t(z) * dd.ny + y) * dd.nx + x]);
    });
  }
  void set_specular_walls(const std::uint8_t* codes) override {
    const Domain dd = d;
    s.set_specular_walls([&](Index x, Index y, Index z) -> std::uint8_t {
      return codes[(std::size_t(z) * dd.ny + y) * dd.nx + x];
    });
  }
  void set_specular_nodes(const std::uint8_t* masks) override {
    const Domain dd = d;
    s.set_specular_nodes([&](Index x, Index y, Index z) -> std::uint8_t {
      return masks[(std::size_t(z) * dd.ny + y) * dd.nx + x];
    });
  }
  void set_regularized_walls(const std::uint8_t* codes, const double* spec) override {
    const Domain dd = d;
    using WS = typename FluidSolver<L, Strm, Coll>::WallSpec;
    s.set_regularized_walls([&](Index x, Index y, Index z) -> WS {
      const std::size_t k = (std::size_t(z) * dd.ny + y) * dd.nx + x;
      WS w;
      w.normal = codes[k];
      if (spec) {
        w.ux = Real(spec[4 * k]); w.uy = Real(spec[4 * k + 1]);
        w.uz = Real(spec[4 * k + 2]); w.rho = Real(spec[4 * k + 3]);
      }
      return w;
    });
  }
  void set_wall_velocity_scale(double sc) override { s.set_wall_velocity_scale(Real(sc)); }
  void set_wall_density(double r) override { s.set_wall_density(Real(r)); }
  void set_wall_velocity_field(const double* u3) override {
    const Domain dd = d;
    s.set_wall_velocity_field([&](Index x, Index y, Index z) -> std::array<Real, 3> {
      const std::size_t k = (std::size_t(z) * dd.ny + y) * dd.nx + x;
      return {Real(u3[3 * k]), Real(u3[3 * k + 1]), Real(u3[3 * k + 2])};
    });
  }
  void set_wall_velocity_field_scale(double sc) override {
    s.set_wall_velocity_field_scale(Real(sc));
  }
  void set_fd_corners(bool on) override { s.set_fd_corners(on); }
  void set_force_correction(bool on) override { s.set_force_correction(on); }
  void set_outflow_order(int k) override { s.set_outflow_order(k); }
  void set_outflow_density(double r) override { s.set_outflow_density(Real(r)); }
  int set_buoyancy(const double* T, double gx, double gy, double gz, double rho0, double beta,
                   double T0) override {
    if constexpr (requires(Coll& c) { c.forcing.T; c.forcing.beta; }) {
      auto& f = s.collision().forcing;
      f.gx = Real(gx); f.gy = Real(gy); f.gz = Real(gz);
      f.rho0 = Real(rho0); f.beta = Real(beta); f.T0 = Real(T0);
      for (Index z = 0; z < d.nz; ++z)
        for (Index y = 0; y < d.ny; ++y)
          for (Index x = 0; x < d.nx; ++x)
            f.T(d.id(x, y, z)) = Real(T[(std::size_t(z) * d.ny + y) * d.nx + x]);
      return 0;
    } else {
      return -1;
    }
  }
  long long nx() const override { return d.nx; }
  long long ny() const override { return d.ny; }
  void initialize(double rho, double ux, double uy, double uz) override {
    s.initialize(Real(rho), Real(ux), Real(uy), Real(uz));
  }
  void initialize_field(const double* rho, const double* ux, const double* uy,
                        const double* uz) override {
    const Domain dd = d;
    s.initialize_field([=](Index n) {
      Index px, py, pz; dd.coords(n, px, py, pz);
      FlowState st;
      if (!dd.is_interior(px, py, pz)) return st;
      const std::size_t k =
          (std::size_t(pz - dd.hz) * dd.ny + (py - dd.hy)) * dd.nx + (px - dd.hx);
      st.rho = Real(rho[k]); st.ux = Real(ux[k]); st.uy = Real(uy[k]); st.uz = Real(uz[k]);
      return st;
    });
  }
  void step(int n, int store) override {
    for (int t = 0; t < n; ++t) s.step(store != 0);
  }
  void copy_interior(double* rho, double* ux, double* uy, double* uz) {
    auto r = s.rho(); auto a = s.ux(); auto b = s.uy(); auto c = s.uz();
    for (Index z = 0; z < d.nz; ++z)
      for (Index y = 0; y < d.ny; ++y)
        for (Index x = 0; x < d.nx; ++x) {
          const Index n = d.id(x, y, z);
          const std::size_t k = (std::size_t(z) * d.ny + y) * d.nx + x;
          rho[k] = double(r(n)); ux[k] = double(a(n)); uy[k] = double(b(n)); uz[k] = double(c(n));
        }
  }
  void macro(double* rho, double* ux, double* uy, double* uz) override {
    s.compute_macroscopic();
    copy_interior(rho, ux, uy, uz);
  }
  void stored_macro(double* rho, double* ux, double* uy, double* uz) override {
    copy_interior(rho, ux, uy, uz);
  }
  double mass() override { return double(s.total_mass()); }
  double momentum(int a) override { return double(s.total_momentum(a)); }
  void gather(double* out) override {
    auto g = s.gather_populations();
    const std::size_t n = std::size_t(d.n_padded) * L::Q;
    for (std::size_t i = 0; i < n; ++i) out[i] = double(g.data()[i]);
  }
  void seed(const double* in) override {
    constexpr int Q = L::Q;
    s.seed_populations([=](Index n, int i) { return Real(in[std::size_t(n) * Q + i]); });
  }
  double slot_sum() override {
    if constexpr (std::is_same_v<Strm, EsotericPull<L>>) {
      auto st = s.populations().storage();
      double acc = 0;
      for (std::size_t i = 0; i < st.size(); ++i) acc += double(st.data()[i]);
      return acc;
    } else {
      return 0.0 / 0.0;
    }
  }
  long long n_padded() const override { return d.n_padded; }
  long long n_interior() const override { return (long long)d.nx * d.ny * d.nz; }
  long long timestep() const override { return (long long)s.timestep(); }
};

}  // namespace refdrv
