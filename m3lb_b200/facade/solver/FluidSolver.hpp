// FluidSolver on the B200 (names and members of src/solver/FluidSolver.hpp).
//
// The population array, the flags and the time loop live on the GPU in
// libm3lb.so; every member below forwards to its C ABI (include/m3lb.h).
// What changes for a caller of the reference:
//   * callbacks given to set_geometry / initialize_field / seed_populations
//     run on the host, once, and their results are uploaded;
//   * rho()/ux()/uy()/uz()/flags() and gather_populations() return host arrays;
//   * an optional fourth template argument picks the precision the
//     populations are stored in on the device (StoreF32, StoreF16, StoreBF16,
//     StoreF64, StoreF16C); by default it follows Real, or
//     -DLBM_B200_STORAGE_F16 / _BF16 / _F16C selects 16-bit storage for
//     every solver;
//   * the policies must be ones the device runs: D2Q9 / D3Q27; BGK, TRT,
//     MomentCollision; NoForcing or Guo; Fluid, Solid and Excluded cells
//     and the wall cells RegWall, SpecWall and SpecNode.
//     Anything else fails to compile (static_assert) or is rejected at
//     set_geometry.
#pragma once
#include <array>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "boundary/Flags.hpp"
#include "boundary/Regularized.hpp"
#include "boundary/Specular.hpp"
#include "collision/BGK.hpp"
#include "collision/MomentCollision.hpp"
#include "collision/TRT.hpp"
#include "core/Types.hpp"
#include "grid/Domain.hpp"
#include "lattice/Lattices.hpp"
#include "memory/EsotericPull.hpp"
#include "memory/TwoLattice.hpp"

namespace lbm {

struct FlowState {
  Real rho = Real(1), ux = Real(0), uy = Real(0), uz = Real(0);
};

// Device storage precision of the populations.
struct StoreF32 { static constexpr int code = M3LB_STORE_F32; static constexpr const char* name = "FP32"; };
struct StoreF16 { static constexpr int code = M3LB_STORE_F16; static constexpr const char* name = "FP16"; };
struct StoreBF16 { static constexpr int code = M3LB_STORE_BF16; static constexpr const char* name = "BF16"; };
struct StoreF64 { static constexpr int code = M3LB_STORE_F64; static constexpr const char* name = "FP64"; };
// 1 sign, 4 exponent and 11 mantissa bits: FP16's bytes, half its rounding error
struct StoreF16C { static constexpr int code = M3LB_STORE_F16C; static constexpr const char* name = "FP16C"; };
#if defined(LBM_B200_STORAGE_F16)
using DefaultStore = StoreF16;
#elif defined(LBM_B200_STORAGE_BF16)
using DefaultStore = StoreBF16;
#elif defined(LBM_B200_STORAGE_F16C)
using DefaultStore = StoreF16C;
#else
using DefaultStore = std::conditional_t<sizeof(Real) == 4, StoreF32, StoreF64>;
#endif

namespace facade {
template <class S> struct IsDeviceStreaming : std::false_type {};
template <class L> struct IsDeviceStreaming<EsotericPull<L>> : std::true_type {};
template <class L> struct IsDeviceStreaming<TwoLattice<L>> : std::true_type {};
template <class F> struct IsDeviceForcing : std::false_type {};
template <> struct IsDeviceForcing<NoForcing> : std::true_type {};
template <> struct IsDeviceForcing<Guo> : std::true_type {};
template <> struct IsDeviceForcing<BoussinesqGuo> : std::true_type {};
template <class C, class = void> struct EqCode { static constexpr int value = 0; };
template <class C>
struct EqCode<C, std::void_t<decltype(C::Equilibrium::device_code)>> {
  static constexpr int value = C::Equilibrium::device_code;
};
}  // namespace facade

template <class L, class Streaming, class Collision, class Store = DefaultStore>
class FluidSolver {
 public:
  using Lattice = L;
  static constexpr int Q = L::Q;

  // One regularised wall node (:97-103): outward normal code, imposed
  // velocity, and the density the outlet codes impose.
  struct WallSpec {
    std::uint8_t normal = NrmNone;
    Real ux = 0, uy = 0, uz = 0;
    Real rho = Real(1);
  };

  static_assert(DeviceLattice<L>::code != 0, "the B200 path runs D2Q9 and D3Q27");
  static_assert(facade::IsDeviceStreaming<Streaming>::value,
                "the B200 path streams with Esoteric Pull (TwoLattice runs as Esoteric Pull)");
  static_assert(facade::IsDeviceForcing<typename Collision::ForcingPolicy>::value,
                "the B200 path runs NoForcing, the uniform Guo force and BoussinesqGuo");

  FluidSolver(const Domain& dom, const Collision& coll)
      : dom_(dom), coll_(coll), flags_("flags", dom.n_padded), rho_("rho", dom.n_padded),
        ux_("ux", dom.n_padded), uy_("uy", dom.n_padded), uz_("uz", dom.n_padded) {
    const int lat = DeviceLattice<L>::code;
    m3lb_facade::check(
        m3lb_create(lat, dom.nx, dom.ny, dom.nz, dom.periodic[0], dom.periodic[1],
                    dom.periodic[2], Collision::device_op, facade::EqCode<Collision>::value,
                    Store::code, Collision::Storage::shifted ? 1 : 0,
                    Collision::ForcingPolicy::active ? 1 : 0, &h_),
        "FluidSolver");
    m3lb_facade::add(h_);
    bind_fields();
    for (Index n = 0; n < dom.n_padded; ++n) {
      Index px, py, pz;
      dom_.coords(n, px, py, pz);
      flags_(n) = dom_.is_interior(px, py, pz) ? Fluid : Excluded;
    }
    push_params();
  }
  ~FluidSolver() {
    if (h_) {
      m3lb_facade::remove(h_);
      m3lb_destroy(h_);
    }
  }
  FluidSolver(const FluidSolver&) = delete;
  FluidSolver& operator=(const FluidSolver&) = delete;

  // set_geometry (:74-82): fn(x, y, z) -> CellType over interior coordinates.
  template <class Fn>
  void set_geometry(Fn fn) {
    std::vector<std::uint8_t> a(std::size_t(dom_.n_interior()));
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x) {
          const std::uint8_t v = std::uint8_t(fn(x, y, z));
          a[(std::size_t(z) * dom_.ny + y) * dom_.nx + x] = v;
          flags_(dom_.id(x, y, z)) = v;
        }
    m3lb_facade::check(m3lb_set_flags(h_, a.data()), "set_geometry");
  }

  // set_specular_walls (:193-218): fn(x, y, z) -> NormalCode; NrmNone leaves
  // the node, an axis code marks it a free-slip ghost (SpecWall).  A code
  // above NrmZm ends the program with the reference's message, as there.
  template <class Fn>
  void set_specular_walls(Fn fn) {
    std::vector<std::uint8_t> a(std::size_t(dom_.n_interior()));
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x)
          a[(std::size_t(z) * dom_.ny + y) * dom_.nx + x] = std::uint8_t(fn(x, y, z));
    m3lb_facade::check(m3lb_set_specular_walls(h_, a.data()), "set_specular_walls");
    mark(a, SpecWall);
  }

  // set_regularized_walls (:372-552): fn(x, y, z) -> WallSpec; NrmNone leaves
  // the node, any other code marks it a regularised on-node wall.
  template <class Fn>
  void set_regularized_walls(Fn fn) {
    const std::size_t ni = std::size_t(dom_.n_interior());
    std::vector<std::uint8_t> codes(ni, 0);
    std::vector<double> st(4 * ni, 0.0);
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x) {
          const std::size_t k = (std::size_t(z) * dom_.ny + y) * dom_.nx + x;
          const WallSpec w = fn(x, y, z);
          codes[k] = w.normal;
          st[4 * k] = w.ux; st[4 * k + 1] = w.uy; st[4 * k + 2] = w.uz; st[4 * k + 3] = w.rho;
        }
    m3lb_facade::check(m3lb_set_regularized_walls(h_, codes.data(), st.data()),
                       "set_regularized_walls");
    mark(codes, RegWall);
    // distinct wall states, as the reference's deduplicated table counts them
    std::vector<std::array<Real, 4>> table;
    for (std::size_t k = 0; k < ni; ++k) {
      if (!codes[k]) continue;
      const std::array<Real, 4> v{Real(st[4 * k]), Real(st[4 * k + 1]), Real(st[4 * k + 2]),
                                  Real(st[4 * k + 3])};
      bool seen = false;
      for (const auto& t : table) seen = seen || t == v;
      if (!seen) table.push_back(v);
    }
    n_wall_states_ = table.empty() ? 1 : table.size();
  }
  std::size_t n_wall_states() const { return n_wall_states_; }
  void set_wall_velocity_scale(Real sc) {
    m3lb_facade::check(m3lb_set_wall_velocity_scale(h_, sc), "set_wall_velocity_scale");
  }
  void set_wall_density(Real r) { m3lb_facade::check(m3lb_set_wall_density(h_, r), "set_wall_density"); }
  // fn(x, y, z) -> std::array<Real, 3>, lattice units, interior coordinates
  template <class Fn>
  void set_wall_velocity_field(Fn fn) {
    std::vector<double> u(3 * std::size_t(dom_.n_interior()));
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x) {
          const std::size_t k = (std::size_t(z) * dom_.ny + y) * dom_.nx + x;
          const auto v = fn(x, y, z);
          u[3 * k] = v[0]; u[3 * k + 1] = v[1]; u[3 * k + 2] = v[2];
        }
    m3lb_facade::check(m3lb_set_wall_velocity_field(h_, u.data()), "set_wall_velocity_field");
  }
  void set_wall_velocity_field_scale(Real s) {
    m3lb_facade::check(m3lb_set_wall_velocity_field_scale(h_, s), "set_wall_velocity_field_scale");
  }
  void set_fd_corners(bool on) { m3lb_facade::check(m3lb_set_fd_corners(h_, on), "set_fd_corners"); }
  void set_force_correction(bool on) {
    m3lb_facade::check(m3lb_set_force_correction(h_, on), "set_force_correction");
  }
  void set_outflow_order(int k) {
    m3lb_facade::check(m3lb_set_outflow_order(h_, k), "set_outflow_order");
  }
  void set_outflow_density(Real r) {
    out_rho_ = r;
    m3lb_facade::check(m3lb_set_outflow_density(h_, r), "set_outflow_density");
  }
  Real outflow_density() const { return out_rho_; }
  Index wall_count() const {
    Index n = 0;
    for (Index k = 0; k < dom_.n_padded; ++k) n += flags_(k) == RegWall;
    return n;
  }

  // set_specular_nodes (:236-268): fn(x, y, z) -> SpecFace mask; SpecNone
  // leaves the node, any valid mask marks it an on-node free-slip node.
  template <class Fn>
  void set_specular_nodes(Fn fn) {
    std::vector<std::uint8_t> a(std::size_t(dom_.n_interior()));
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x)
          a[(std::size_t(z) * dom_.ny + y) * dom_.nx + x] = std::uint8_t(fn(x, y, z));
    m3lb_facade::check(m3lb_set_specular_nodes(h_, a.data()), "set_specular_nodes");
    mark(a, SpecNode);
  }

  // initialize (:553-561)
  void initialize(Real rho0, Real ux0 = 0, Real uy0 = 0, Real uz0 = 0) {
    push_params();
    m3lb_facade::check(m3lb_init_eq(h_, rho0, ux0, uy0, uz0), "initialize");
  }

  // initialize_field (:568-579): fn(n) -> FlowState, n a padded index, called
  // on the host for the fluid nodes.
  template <class Fn>
  void initialize_field(Fn fn) {
    const std::size_t ni = std::size_t(dom_.n_interior());
    std::vector<double> r(ni, 1.0), u(ni, 0.0), v(ni, 0.0), w(ni, 0.0);
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x) {
          const Index n = dom_.id(x, y, z);
          if (flags_(n) != Fluid && flags_(n) != RegWall && flags_(n) != SpecNode) continue;
          const FlowState s = fn(n);
          const std::size_t k = (std::size_t(z) * dom_.ny + y) * dom_.nx + x;
          r[k] = s.rho; u[k] = s.ux; v[k] = s.uy; w[k] = s.uz;
        }
    push_params();
    m3lb_facade::check(m3lb_init_field_f64(h_, r.data(), u.data(), v.data(), w.data()),
                       "initialize_field");
  }

  // step (:582-591).  The collision's members are read at every step, as the
  // reference's kernel captures the policy by value at every launch.
  void step(bool store_macroscopic = false) {
    push_params();
    m3lb_facade::check(m3lb_step(h_, 1, store_macroscopic ? 1 : 0), "step");
    if (store_macroscopic) fields_stale_ = true;
  }

  // compute_macroscopic (:597-599)
  void compute_macroscopic() {
    std::vector<double> r, u, v, w;
    alloc4(r, u, v, w);
    m3lb_facade::check(m3lb_macro_f64(h_, r.data(), u.data(), v.data(), w.data()),
                       "compute_macroscopic");
    to_padded(r, u, v, w);
    fields_stale_ = false;
  }

  Real total_mass() const { return Real(reduce()[0]); }
  Real total_momentum(int a) const { return Real(reduce()[1 + a]); }

  const Domain& domain() const { return dom_; }
  Streaming& populations() { return pop_; }
  Collision& collision() { return coll_; }
  View1D<Real> rho() const { refresh(); return rho_; }
  View1D<Real> ux() const { refresh(); return ux_; }
  View1D<Real> uy() const { refresh(); return uy_; }
  View1D<Real> uz() const { refresh(); return uz_; }
  View1D<std::uint8_t> flags() const { return flags_; }
  std::size_t timestep() const {
    long long t = 0;
    m3lb_facade::check(m3lb_timestep(h_, &t), "timestep");
    return std::size_t(t);
  }
  Index active_count() const {
    Index c = 0;
    for (Index n = 0; n < dom_.n_padded; ++n) c += flags_(n) == Fluid;
    return c;
  }

  // gather_populations (:620-624)
  View2D<Real> gather_populations() const {
    std::vector<double> a(std::size_t(dom_.n_padded) * Q);
    m3lb_facade::check(m3lb_gather(h_, a.data()), "gather_populations");
    View2D<Real> out("gathered", dom_.n_padded, Q);
    for (std::size_t k = 0; k < a.size(); ++k) out.data()[k] = Real(a[k]);
    return out;
  }
  // seed_populations (:634-637): fn(n, i) -> Real, evaluated on the host.
  template <class Fn>
  void seed_populations(Fn fn) {
    std::vector<double> a(std::size_t(dom_.n_padded) * Q);
    for (Index n = 0; n < dom_.n_padded; ++n)
      for (int i = 0; i < Q; ++i) a[std::size_t(n) * Q + i] = double(fn(n, i));
    m3lb_facade::check(m3lb_scatter(h_, a.data()), "seed_populations");
  }

  // Additions of the B200 path.
  m3lb_solver* handle() const { return h_; }
  void set_stream(void* stream) { m3lb_facade::check(m3lb_set_stream(h_, stream), "set_stream"); }
  void steps(int n, bool store_macroscopic = false) {
    push_params();
    m3lb_facade::check(m3lb_step(h_, n, store_macroscopic ? 1 : 0), "steps");
    if (store_macroscopic) fields_stale_ = true;
  }

 private:
  // host copy of the flags after a specular setter marked the nonzero entries
  void mark(const std::vector<std::uint8_t>& a, CellType type) {
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x)
          if (a[(std::size_t(z) * dom_.ny + y) * dom_.nx + x]) flags_(dom_.id(x, y, z)) = type;
  }
  // The field views carry the device arrays they mirror, so that a scalar
  // solver given ux() / uy() / uz() reads the velocity on the device.
  void bind_fields() {
    void *r = nullptr, *u = nullptr, *v = nullptr, *w = nullptr, *st = nullptr;
    m3lb_facade::check(m3lb_macro_pointers(h_, &r, &u, &v, &w), "fields");
    m3lb_facade::check(m3lb_get_stream(h_, &st), "stream");
    View1D<Real>* views[4] = {&rho_, &ux_, &uy_, &uz_};
    void* ptrs[4] = {r, u, v, w};
    for (int i = 0; i < 4; ++i) { views[i]->dev_ = ptrs[i]; views[i]->dev_stream_ = st; }
  }
  // BoussinesqGuo: the temperature the force reads, bound before each step.
  void push_buoyancy() {
    if constexpr (std::is_same_v<typename Collision::ForcingPolicy, BoussinesqGuo>) {
      const BoussinesqGuo& F = coll_.forcing;
      if (F.T.dev_) {
        void* st = nullptr;
        m3lb_facade::check(m3lb_get_stream(h_, &st), "stream");
        m3lb_facade::check(m3lb_stream_order(F.T.dev_stream_, st), "stream order");
        m3lb_facade::check(m3lb_set_buoyancy(h_, F.T.dev_, F.gx, F.gy, F.gz, F.rho0, F.beta, F.T0),
                           "buoyancy");
      } else if (F.T.data()) {
        std::vector<double> t(std::size_t(dom_.n_interior()));
        for (Index z = 0; z < dom_.nz; ++z)
          for (Index y = 0; y < dom_.ny; ++y)
            for (Index x = 0; x < dom_.nx; ++x)
              t[(std::size_t(z) * dom_.ny + y) * dom_.nx + x] = double(F.T(dom_.id(x, y, z)));
        m3lb_facade::check(m3lb_set_buoyancy_host(h_, t.data(), F.gx, F.gy, F.gz, F.rho0, F.beta,
                                                  F.T0), "buoyancy");
      } else {
        m3lb_facade::check(m3lb_set_buoyancy(h_, nullptr, 0, 0, 0, 1, 1, 0), "buoyancy");
      }
    }
  }
  void push_params() {
    push_buoyancy();
    double w1 = 1, w2 = -1;
    coll_.device_rates(w1, w2);
    double f[3] = {0, 0, 0};
    if constexpr (Collision::ForcingPolicy::active) {
      f[0] = coll_.forcing.fx; f[1] = coll_.forcing.fy; f[2] = coll_.forcing.fz;
    }
    m3lb_facade::check(m3lb_set_params(h_, w1, w2, f[0], f[1], f[2]), "parameters");
  }
  std::array<double, 6> reduce() const {
    std::array<double, 6> out{};
    m3lb_facade::check(m3lb_reduce(h_, out.data()), "reduce");
    return out;
  }
  void alloc4(std::vector<double>& r, std::vector<double>& u, std::vector<double>& v,
              std::vector<double>& w) const {
    const std::size_t ni = std::size_t(dom_.n_interior());
    r.resize(ni); u.resize(ni); v.resize(ni); w.resize(ni);
  }
  void to_padded(const std::vector<double>& r, const std::vector<double>& u,
                 const std::vector<double>& v, const std::vector<double>& w) const {
    for (Index z = 0; z < dom_.nz; ++z)
      for (Index y = 0; y < dom_.ny; ++y)
        for (Index x = 0; x < dom_.nx; ++x) {
          const Index n = dom_.id(x, y, z);
          const std::size_t k = (std::size_t(z) * dom_.ny + y) * dom_.nx + x;
          rho_(n) = Real(r[k]); ux_(n) = Real(u[k]); uy_(n) = Real(v[k]); uz_(n) = Real(w[k]);
        }
  }
  // Fields written on the device by step(true) are brought to the host on
  // first access.
  void refresh() const {
    if (!fields_stale_) return;
    std::vector<double> r, u, v, w;
    alloc4(r, u, v, w);
    m3lb_facade::check(m3lb_stored_macro_f64(h_, r.data(), u.data(), v.data(), w.data()),
                       "fields");
    to_padded(r, u, v, w);
    fields_stale_ = false;
  }

  Domain dom_;
  Collision coll_;
  Streaming pop_{};
  m3lb_solver* h_ = nullptr;
  Real out_rho_ = Real(1);
  std::size_t n_wall_states_ = 0;
  View1D<std::uint8_t> flags_;
  View1D<Real> rho_, ux_, uy_, uz_;
  mutable bool fields_stale_ = false;
};

}  // namespace lbm
