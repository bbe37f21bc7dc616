// ScalarSolver<L, Streaming, Collision> (src/solver/ScalarSolver.hpp) on the
// B200: a D2Q5 / D3Q7 advection-diffusion lattice stepped on the device by
// libm3lb.so (m3lb_scalar_*).  Callbacks run on the host once and their
// results are uploaded; temperature() and flags() return host views.
//
// Coupling as the reference's drivers write it works unchanged:
//   * set_velocity(fl.ux(), fl.uy(), fl.uz()) with a FluidSolver's views makes
//     this solver read the fluid's stored velocity on the device, each step
//     ordered after the fluid's queued work;
//   * a BoussinesqGuo force whose T is this solver's temperature() reads the
//     field on the device, ordered after this solver's steps.
// Views that no solver handed out are copied up before each step.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "boundary/MomentDirichlet.hpp"
#include "boundary/Regularized.hpp"
#include "boundary/Specular.hpp"
#include "collision/ScalarBGK.hpp"
#include "core/Types.hpp"
#include "grid/Domain.hpp"
#include "lattice/Lattices.hpp"
#include "m3lb_facade_device.hpp"
#include "memory/EsotericPull.hpp"

namespace lbm {

template <class L, class Streaming, class Collision>
class ScalarSolver {
 public:
  using Lattice = L;
  static constexpr int Q = L::Q;
  static_assert(L::Q == 5 || L::Q == 7 || L::Q == 9 || L::Q == 27,
                "the B200 scalar path runs D2Q5, D3Q7, D2Q9 and D3Q27");
  static_assert(std::is_same_v<Streaming, EsotericPull<L>>, "the B200 scalar path streams with Esoteric Pull");

  ScalarSolver(const Domain& dom, const Collision& coll)
      : dom_(dom), coll_(coll), flags_("sflags", dom.n_padded), wall_("Twall", dom.n_padded),
        field_("T", dom.n_padded) {
    m3lb_facade::check(m3lb_scalar_create(L::Q, dom.nx, dom.ny, dom.nz, dom.periodic[0],
                                          dom.periodic[1], dom.periodic[2], Collision::device_op,
                                          sizeof(Real) == 8 ? M3LB_STORE_F64 : M3LB_STORE_F32, &h_),
                       "ScalarSolver");
    m3lb_facade::add(h_);
    for (Index n = 0; n < dom.n_padded; ++n) {
      Index px, py, pz;
      dom_.coords(n, px, py, pz);
      flags_(n) = dom_.is_interior(px, py, pz) ? ScalarBulk : ScalarExcluded;
    }
    bind_field();
  }
  ~ScalarSolver() {
    if (h_) {
      m3lb_facade::remove(h_);
      m3lb_scalar_destroy(h_);
    }
  }
  ScalarSolver(const ScalarSolver&) = delete;
  ScalarSolver& operator=(const ScalarSolver&) = delete;

  // fn(x, y, z) -> ScalarCell, over interior coordinates (:92-99).
  template <class Fn>
  void set_geometry(Fn fn) {
    std::vector<std::uint8_t> c(std::size_t(dom_.n_interior()));
    for_interior([&](Index x, Index y, Index z, std::size_t k) {
      c[k] = std::uint8_t(fn(x, y, z));
      flags_(dom_.id(x, y, z)) = c[k];
    });
    m3lb_facade::check(m3lb_scalar_set_cells(h_, c.data()), "set_geometry");
  }
  // fn(x, y, z) -> Real, the value Dirichlet and moment cells impose (:101-108).
  template <class Fn>
  void set_wall_values(Fn fn) {
    std::vector<double> v(std::size_t(dom_.n_interior()));
    for_interior([&](Index x, Index y, Index z, std::size_t k) {
      v[k] = double(fn(x, y, z));
      wall_(dom_.id(x, y, z)) = Real(v[k]);
    });
    m3lb_facade::check(m3lb_scalar_set_wall_values(h_, v.data()), "set_wall_values");
  }
  // fn(x, y, z) -> NormalCode of a ScalarSpecular cell (:113-132).
  template <class Fn>
  void set_specular_walls(Fn fn) {
    std::vector<std::uint8_t> c(std::size_t(dom_.n_interior()));
    for_interior([&](Index x, Index y, Index z, std::size_t k) { c[k] = std::uint8_t(fn(x, y, z)); });
    m3lb_facade::check(m3lb_scalar_set_specular_walls(h_, c.data()), "set_specular_walls");
  }
  // fn(x, y, z) -> SpecFace mask of a ScalarSpecular cell (:140-164).
  template <class Fn>
  void set_specular_nodes(Fn fn) {
    std::vector<std::uint8_t> c(std::size_t(dom_.n_interior()));
    for_interior([&](Index x, Index y, Index z, std::size_t k) { c[k] = std::uint8_t(fn(x, y, z)); });
    m3lb_facade::check(m3lb_scalar_set_specular_nodes(h_, c.data()), "set_specular_nodes");
  }
  // set_velocity (:166-168): views per padded node.
  void set_velocity(View1D<Real> ux, View1D<Real> uy, View1D<Real> uz) {
    ux_ = ux; uy_ = uy; uz_ = uz;
    u_up_.clear();
    if (ux.dev_ && uy.dev_ && uz.dev_) {
      // a solver's own fields: read on the device, each step ordered after
      // that solver's queued work (push)
      m3lb_facade::check(m3lb_scalar_set_velocity_device(h_, ux.dev_, uy.dev_, uz.dev_), "set_velocity");
    } else if (!ux.data()) {
      m3lb_facade::check(m3lb_scalar_set_velocity_device(h_, nullptr, nullptr, nullptr), "set_velocity");
    }
  }

  void initialize(Real T0) {
    initialize_field([=](Index) { return T0; });
  }
  // fn(n) -> Real over padded indices (:175-190).
  template <class Fn>
  void initialize_field(Fn fn) {
    std::vector<double> t(std::size_t(dom_.n_padded));
    for (Index n = 0; n < dom_.n_padded; ++n) t[std::size_t(n)] = double(fn(n));
    push();
    m3lb_facade::check(m3lb_scalar_init_field(h_, t.data()), "initialize_field");
    stale_ = true;
  }

  void step() {
    push();
    m3lb_facade::check(m3lb_scalar_step(h_, 1), "step");
    stale_ = true;
  }
  // fn(n) -> Real over padded indices, on bulk and specular cells (:205-208).
  template <class Fn>
  void add_source(Fn fn) {
    std::vector<double> d(std::size_t(dom_.n_interior()));
    for_interior([&](Index x, Index y, Index z, std::size_t k) { d[k] = double(fn(dom_.id(x, y, z))); });
    m3lb_facade::check(m3lb_scalar_add_source(h_, d.data()), "add_source");
  }
  void compute_field() {
    m3lb_facade::check(m3lb_scalar_compute_field(h_), "compute_field");
    stale_ = true;
  }
  View1D<Real> temperature() const {
    refresh();
    return field_;
  }
  View1D<std::uint8_t> flags() const { return flags_; }
  Real total_population() const {
    double t = 0;
    m3lb_facade::check(m3lb_scalar_total(h_, &t), "total_population");
    return Real(t);
  }
  void finalize_geometry() { m3lb_facade::check(m3lb_scalar_finalize_geometry(h_), "finalize_geometry"); }
  void build_donors() { finalize_geometry(); }
  const Domain& domain() const { return dom_; }
  std::size_t timestep() const {
    long long t = 0;
    m3lb_facade::check(m3lb_scalar_info(h_, nullptr, &t, nullptr), "timestep");
    return std::size_t(t);
  }
  m3lb_scalar* handle() const { return h_; }

 private:
  template <class F>
  void for_interior(F f) const {
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x) f(x, y, z, (std::size_t(z) * dom_.ny + y) * dom_.nx + x);
  }
  void bind_field() {
    void *t = nullptr, *st = nullptr;
    m3lb_facade::check(m3lb_scalar_field_device(h_, &t), "field");
    m3lb_facade::check(m3lb_scalar_get_stream(h_, &st), "stream");
    field_.dev_ = t;
    field_.dev_stream_ = st;
  }
  // parameters, per-node rates and host-side velocities, before a launch
  void push() {
    double lambda = 0.25;
    if constexpr (requires(const Collision& c) { c.Lambda; }) lambda = coll_.Lambda;
    m3lb_facade::check(m3lb_scalar_set_params(h_, coll_.omega, coll_.T_ref, lambda), "parameters");
    // host views are shared with the caller, who may change them between
    // steps: compare with what was uploaded last and upload on a change
    if (coll_.omega_of.data()) {
      std::vector<double> w(std::size_t(dom_.n_interior()));
      for_interior([&](Index x, Index y, Index z, std::size_t k) { w[k] = double(coll_.omega_of(dom_.id(x, y, z))); });
      if (w != omega_up_) {
        m3lb_facade::check(m3lb_scalar_set_omega_field(h_, w.data()), "omega field");
        omega_up_.swap(w);
      }
    }
    if (ux_.dev_) {
      void* st = nullptr;
      m3lb_facade::check(m3lb_scalar_get_stream(h_, &st), "stream");
      m3lb_facade::check(m3lb_stream_order(ux_.dev_stream_, st), "stream order");
    } else if (ux_.data()) {
      const std::size_t ni = std::size_t(dom_.n_interior());
      std::vector<double> u(3 * ni);
      for_interior([&](Index x, Index y, Index z, std::size_t k) {
        const Index n = dom_.id(x, y, z);
        u[k] = double(ux_(n)); u[ni + k] = double(uy_(n)); u[2 * ni + k] = double(uz_(n));
      });
      if (u != u_up_) {
        m3lb_facade::check(m3lb_scalar_set_velocity_host(h_, u.data(), u.data() + ni, u.data() + 2 * ni),
                           "velocity");
        u_up_.swap(u);
      }
    }
  }
  void refresh() const {
    if (!stale_) return;
    std::vector<double> t(std::size_t(dom_.n_interior()));
    m3lb_facade::check(m3lb_scalar_field(h_, t.data()), "temperature");
    for_interior([&](Index x, Index y, Index z, std::size_t k) { field_(dom_.id(x, y, z)) = Real(t[k]); });
    stale_ = false;
  }

  Domain dom_;
  Collision coll_;
  m3lb_scalar* h_ = nullptr;
  View1D<std::uint8_t> flags_;
  View1D<Real> wall_, field_;
  View1D<Real> ux_, uy_, uz_;
  std::vector<double> u_up_, omega_up_;  // host views as last uploaded
  mutable bool stale_ = false;
};

}  // namespace lbm
