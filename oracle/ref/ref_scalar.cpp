// C-ABI driver over the REFERENCE's own ScalarSolver (src/solver/ScalarSolver.hpp)
// with ScalarBGK / ScalarTRT / ScalarRegularised on D2Q5 and D3Q7, compiled
// unmodified against the host Kokkos-API stand-in.  Test infrastructure only.
//
//   ref_screate / ref_sdestroy       ScalarSolver(Domain, Collision)           :72-90
//   ref_sset_geometry                set_geometry(fn -> ScalarCell)            :92-99
//   ref_sset_wall_values             set_wall_values(fn -> Real)               :101-108
//   ref_sset_specular_walls / _nodes set_specular_walls / set_specular_nodes   :113-164
//   ref_sset_omega_field             Collision::omega_of (per-node rate)
//   ref_sset_velocity                set_velocity(ux, uy, uz)                  :166-168
//   ref_sfinalize_geometry           finalize_geometry()                       :223-238
//   ref_sinitialize / _field         initialize(T0) / initialize_field(fn(n))  :170-190
//   ref_sstep                        step()                                    :192-203
//   ref_sadd_source                  add_source(fn(n))                         :205-208
//   ref_scompute_field / ref_sfield  compute_field() / temperature()           :210-216
//   ref_stotal                       total_population()                        :219-228
#include "ref_impl.hpp"

#include "collision/ScalarBGK.hpp"
#include "collision/ScalarRegularised.hpp"
#include "collision/ScalarTRT.hpp"
#include "solver/ScalarSolver.hpp"

namespace refdrv {

struct SBase {
  virtual ~SBase() = default;
  virtual void set_geometry(const std::uint8_t* cells) = 0;
  virtual void set_wall_values(const double* tw) = 0;
  virtual void set_specular_walls(const std::uint8_t* codes) = 0;
  virtual void set_specular_nodes(const std::uint8_t* masks) = 0;
  virtual void set_omega_field(const double* om) = 0;
  virtual void set_velocity(const double* ux, const double* uy, const double* uz) = 0;
  virtual void finalize_geometry() = 0;
  virtual void initialize(double T0) = 0;
  virtual void initialize_field(const double* Tpad) = 0;
  virtual void step(int n) = 0;
  virtual void add_source(const double* dC) = 0;
  virtual void compute_field() = 0;
  virtual void field(double* T) = 0;
  virtual double total() = 0;
  virtual long long n_interior() const = 0;
  virtual long long n_padded() const = 0;
  virtual long long timestep() const = 0;
};

template <class L, class Coll>
struct SImpl final : SBase {
  Domain d;
  View1D<Real> omega_of;       // per-node rates, shared with the solver's copy
  View1D<Real> ux, uy, uz;     // advecting velocity, shared with the solver
  ScalarSolver<L, EsotericPull<L>, Coll> s;
  static Coll make(double omega, double T_ref, double Lambda, View1D<Real> om) {
    Coll c{};
    c.omega = Real(omega);
    c.T_ref = Real(T_ref);
    if constexpr (requires(Coll& k) { k.Lambda; }) c.Lambda = Real(Lambda);
    c.omega_of = om;
    return c;
  }
  static View1D<Real> rates(const Domain& dom, double omega) {
    View1D<Real> v("omega_of", dom.n_padded);
    for (Index n = 0; n < dom.n_padded; ++n) v(n) = Real(omega);
    return v;
  }
  SImpl(const Domain& dom, double omega, double T_ref, double Lambda)
      : d(dom), omega_of(rates(dom, omega)),
        s(dom, make(omega, T_ref, Lambda, omega_of)) {}

  std::size_t k_of(Index x, Index y, Index z) const {
    return (std::size_t(z) * d.ny + y) * d.nx + x;
  }
  void set_geometry(const std::uint8_t* c) override {
    s.set_geometry([&](Index x, Index y, Index z) { return ScalarCell(c[k_of(x, y, z)]); });
  }
  void set_wall_values(const double* tw) override {
    s.set_wall_values([&](Index x, Index y, Index z) { return Real(tw[k_of(x, y, z)]); });
  }
  void set_specular_walls(const std::uint8_t* c) override {
    s.set_specular_walls([&](Index x, Index y, Index z) -> std::uint8_t { return c[k_of(x, y, z)]; });
  }
  void set_specular_nodes(const std::uint8_t* m) override {
    s.set_specular_nodes([&](Index x, Index y, Index z) -> std::uint8_t { return m[k_of(x, y, z)]; });
  }
  void set_omega_field(const double* om) override {
    for (Index z = 0; z < d.nz; ++z)
      for (Index y = 0; y < d.ny; ++y)
        for (Index x = 0; x < d.nx; ++x) omega_of(d.id(x, y, z)) = Real(om[k_of(x, y, z)]);
  }
  void set_velocity(const double* a, const double* b, const double* c) override {
    if (!a) {
      s.set_velocity(View1D<Real>(), View1D<Real>(), View1D<Real>());
      return;
    }
    if (!ux.data()) {
      ux = View1D<Real>("ux", d.n_padded);
      uy = View1D<Real>("uy", d.n_padded);
      uz = View1D<Real>("uz", d.n_padded);
    }
    for (Index z = 0; z < d.nz; ++z)
      for (Index y = 0; y < d.ny; ++y)
        for (Index x = 0; x < d.nx; ++x) {
          const Index n = d.id(x, y, z);
          const std::size_t k = k_of(x, y, z);
          ux(n) = Real(a[k]); uy(n) = Real(b[k]); uz(n) = Real(c[k]);
        }
    s.set_velocity(ux, uy, uz);
  }
  void finalize_geometry() override { s.finalize_geometry(); }
  void initialize(double T0) override { s.initialize(Real(T0)); }
  void initialize_field(const double* Tp) override {
    s.initialize_field([=](Index n) { return Real(Tp[n]); });
  }
  void step(int n) override {
    for (int t = 0; t < n; ++t) s.step();
  }
  void add_source(const double* dC) override {
    const Domain dd = d;
    s.add_source([=](Index n) {
      Index px, py, pz; dd.coords(n, px, py, pz);
      if (!dd.is_interior(px, py, pz)) return Real(0);
      return Real(dC[(std::size_t(pz - dd.hz) * dd.ny + (py - dd.hy)) * dd.nx + (px - dd.hx)]);
    });
  }
  void compute_field() override { s.compute_field(); }
  void field(double* T) override {
    auto f = s.temperature();
    for (Index z = 0; z < d.nz; ++z)
      for (Index y = 0; y < d.ny; ++y)
        for (Index x = 0; x < d.nx; ++x) T[k_of(x, y, z)] = double(f(d.id(x, y, z)));
  }
  double total() override { return double(s.total_population()); }
  long long n_interior() const override { return (long long)d.nx * d.ny * d.nz; }
  long long n_padded() const override { return d.n_padded; }
  long long timestep() const override { return (long long)s.timestep(); }
};

template <class L>
SBase* make_scalar(int op, const Domain& d, double omega, double T_ref, double Lambda) {
  switch (op) {
    case 1: return new SImpl<L, ScalarBGK<L>>(d, omega, T_ref, Lambda);
    case 2: return new SImpl<L, ScalarTRT<L>>(d, omega, T_ref, Lambda);
    case 3: return new SImpl<L, ScalarRegularised<L>>(d, omega, T_ref, Lambda);
    default: return nullptr;
  }
}

// ScalarBGK on the fluid lattices (ScalarTRT / ScalarRegularised need the
// axis-pair lattices and do not compile for these).
template <class L>
SBase* make_scalar_bgk(int op, const Domain& d, double omega, double T_ref, double Lambda) {
  return op == 1 ? new SImpl<L, ScalarBGK<L>>(d, omega, T_ref, Lambda) : nullptr;
}

}  // namespace refdrv

extern "C" {
// lattice 5 (D2Q5) or 7 (D3Q7); op 1 ScalarBGK, 2 ScalarTRT, 3 ScalarRegularised;
// lattice 9 (D2Q9) / 27 (D3Q27) with ScalarBGK.
void* ref_screate(int lattice, int op, int nx, int ny, int nz, int px, int py, int pz,
                  double omega, double T_ref, double Lambda) {
  const Domain d(nx, ny, nz, px != 0, py != 0, pz != 0);
  if (lattice == 5 && nz == 1) return refdrv::make_scalar<D2Q5>(op, d, omega, T_ref, Lambda);
  if (lattice == 7) return refdrv::make_scalar<D3Q7>(op, d, omega, T_ref, Lambda);
  if (lattice == 9 && nz == 1) return refdrv::make_scalar_bgk<D2Q9>(op, d, omega, T_ref, Lambda);
  if (lattice == 27) return refdrv::make_scalar_bgk<D3Q27>(op, d, omega, T_ref, Lambda);
  return nullptr;
}
void ref_sdestroy(void* h) { delete static_cast<refdrv::SBase*>(h); }
void ref_sset_geometry(void* h, const std::uint8_t* c) { static_cast<refdrv::SBase*>(h)->set_geometry(c); }
void ref_sset_wall_values(void* h, const double* t) { static_cast<refdrv::SBase*>(h)->set_wall_values(t); }
// The reference aborts on a rejected code / mask; these check first.
int ref_sset_specular_walls(void* h, const std::uint8_t* c) {
  auto* b = static_cast<refdrv::SBase*>(h);
  for (long long k = 0; k < b->n_interior(); ++k)
    if (c[k] > NrmZm) return -1;
  b->set_specular_walls(c);
  return 0;
}
int ref_sset_specular_nodes(void* h, const std::uint8_t* m) {
  auto* b = static_cast<refdrv::SBase*>(h);
  for (long long k = 0; k < b->n_interior(); ++k) {
    const unsigned v = m[k];
    if (v > 0x3F) return -1;
    for (int a = 0; a < 3; ++a)
      if ((v & (1u << (2 * a))) && (v & (1u << (2 * a + 1)))) return -1;
  }
  b->set_specular_nodes(m);
  return 0;
}
void ref_sset_omega_field(void* h, const double* om) {
  if (om) static_cast<refdrv::SBase*>(h)->set_omega_field(om);
}
void ref_sset_velocity(void* h, const double* ux, const double* uy, const double* uz) {
  static_cast<refdrv::SBase*>(h)->set_velocity(ux, uy, uz);
}
void ref_sfinalize_geometry(void* h) { static_cast<refdrv::SBase*>(h)->finalize_geometry(); }
void ref_sinitialize(void* h, double T0) { static_cast<refdrv::SBase*>(h)->initialize(T0); }
void ref_sinitialize_field(void* h, const double* T) { static_cast<refdrv::SBase*>(h)->initialize_field(T); }
void ref_sstep(void* h, int n) { static_cast<refdrv::SBase*>(h)->step(n); }
void ref_sadd_source(void* h, const double* dC) { static_cast<refdrv::SBase*>(h)->add_source(dC); }
void ref_scompute_field(void* h) { static_cast<refdrv::SBase*>(h)->compute_field(); }
void ref_sfield(void* h, double* T) { static_cast<refdrv::SBase*>(h)->field(T); }
double ref_stotal(void* h) { return static_cast<refdrv::SBase*>(h)->total(); }
long long ref_sn_padded(void* h) { return static_cast<refdrv::SBase*>(h)->n_padded(); }
long long ref_stimestep(void* h) { return static_cast<refdrv::SBase*>(h)->timestep(); }
}  // extern "C"
