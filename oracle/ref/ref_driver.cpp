// C-ABI driver over the REFERENCE's own FluidSolver (src/solver/FluidSolver.hpp),
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
//   ref_initialize        initialize(rho0, ux, uy, uz)         FluidSolver.hpp:553-561
//   ref_initialize_field  initialize_field(fn(n) -> FlowState) FluidSolver.hpp:568-579
//   ref_step              step(store_macroscopic)              FluidSolver.hpp:582-591
//   ref_macro             compute_macroscopic + rho()/ux()..   FluidSolver.hpp:597-599
//   ref_total_mass        total_mass()                          FluidSolver.hpp:601-603
//   ref_total_momentum    total_momentum(a)                     FluidSolver.hpp:604-606
//   ref_gather            gather_populations()                  FluidSolver.hpp:620-624
//   ref_seed              seed_populations(fn(n, i) -> Real)    FluidSolver.hpp:634-637
//   ref_slot_sum          sum over populations().storage()      EsotericPull.hpp:119-123
#include "ref_impl.hpp"

#include <omp.h>

using namespace lbm;

namespace refdrv {
Base* make_D2Q9_EsotericPull_Guo_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_EsotericPull_Guo_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_EsotericPull_NoForcing_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_EsotericPull_NoForcing_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_TwoLattice_Guo_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_TwoLattice_Guo_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_TwoLattice_NoForcing_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_TwoLattice_NoForcing_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_EsotericPull_Guo_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_EsotericPull_Guo_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_EsotericPull_NoForcing_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_EsotericPull_NoForcing_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_TwoLattice_Guo_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_TwoLattice_Guo_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_TwoLattice_NoForcing_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_TwoLattice_NoForcing_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_EsotericPull_BoussinesqGuo_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D2Q9_EsotericPull_BoussinesqGuo_RawPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_EsotericPull_BoussinesqGuo_ShiftedPopulations(int, int, const Domain&, const Params&);
Base* make_D3Q27_EsotericPull_BoussinesqGuo_RawPopulations(int, int, const Domain&, const Params&);

static Base* make(int lattice, int streaming, int op, int eq, int shifted, int forcing,
                  const Domain& d, const Params& p) {
#define REF_PICK(LAT, STRM)                                                         \
  if (forcing) return shifted ? make_##LAT##_##STRM##_Guo_ShiftedPopulations(op, eq, d, p) \
                              : make_##LAT##_##STRM##_Guo_RawPopulations(op, eq, d, p);    \
  return shifted ? make_##LAT##_##STRM##_NoForcing_ShiftedPopulations(op, eq, d, p)        \
                 : make_##LAT##_##STRM##_NoForcing_RawPopulations(op, eq, d, p);
  if (forcing == 2 && !streaming) {  // Boussinesq buoyancy (BoussinesqGuo)
    if (lattice == 9)
      return shifted ? make_D2Q9_EsotericPull_BoussinesqGuo_ShiftedPopulations(op, eq, d, p)
                     : make_D2Q9_EsotericPull_BoussinesqGuo_RawPopulations(op, eq, d, p);
    if (lattice == 27)
      return shifted ? make_D3Q27_EsotericPull_BoussinesqGuo_ShiftedPopulations(op, eq, d, p)
                     : make_D3Q27_EsotericPull_BoussinesqGuo_RawPopulations(op, eq, d, p);
    return nullptr;
  }
  if (lattice == 9) {
    if (streaming) { REF_PICK(D2Q9, TwoLattice) }
    REF_PICK(D2Q9, EsotericPull)
  }
  if (lattice == 27) {
    if (streaming) { REF_PICK(D3Q27, TwoLattice) }
    REF_PICK(D3Q27, EsotericPull)
  }
#undef REF_PICK
  return nullptr;
}
}  // namespace refdrv

extern "C" {

int ref_real_bytes() { return int(sizeof(Real)); }

// OpenMP threads used by the reference's parallel_for / parallel_reduce.
void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }
int ref_get_threads() { return omp_get_max_threads(); }

// lattice: 9 (D2Q9) or 27 (D3Q27).  streaming: 0 EsotericPull, 1 TwoLattice.
// forcing: 0 none, 1 uniform Guo, 2 BoussinesqGuo (Esoteric Pull only).
void* ref_create(int lattice, int streaming, int op, int eq, int shifted, int forcing,
                 int nx, int ny, int nz, int px, int py, int pz, double omega,
                 double omega2, double fx, double fy, double fz) {
  const Domain d(nx, ny, nz, px != 0, py != 0, pz != 0);
  refdrv::Params p{omega, omega2, fx, fy, fz, d.n_padded};
  if (op < 0 || op > 4) return nullptr;
  return refdrv::make(lattice, streaming, op, eq, shifted, forcing, d, p);
}
void ref_destroy(void* h) { delete static_cast<refdrv::Base*>(h); }
void ref_set_geometry(void* h, const std::uint8_t* f) { static_cast<refdrv::Base*>(h)->set_geometry(f); }
// The reference aborts on a value it rejects; these check first and return -1
// instead, so a caller's mistake cannot end the process.
static long long ref_interior(void* h) { return static_cast<refdrv::Base*>(h)->n_interior(); }
int ref_set_specular_walls(void* h, const std::uint8_t* codes) {
  for (long long k = 0; k < ref_interior(h); ++k)
    if (codes[k] > NrmZm) return -1;
  static_cast<refdrv::Base*>(h)->set_specular_walls(codes);
  return 0;
}
// Normal codes per interior node and (ux, uy, uz, rho) per node or NULL.
// Rejected (-1, nothing changed), as the C ABI rejects them: a code above
// NrmOutEq, and a pressure / equilibrium outlet whose upstream stencil leaves
// the interior (x below the outflow order, resp. below 1).
int ref_set_regularized_walls(void* h, const std::uint8_t* codes, const double* spec) {
  auto* b = static_cast<refdrv::Base*>(h);
  const long long n = ref_interior(h), nx = b->nx();
  for (long long k = 0; k < n; ++k) {
    const unsigned c = codes[k];
    if (c > NrmOutEq) return -1;
    if ((c == NrmOutXp || c == NrmOutEq) && k % nx < (c == NrmOutXp ? b->out_order : 1)) return -1;
  }
  b->wall_codes.assign(codes, codes + n);
  b->set_regularized_walls(codes, spec);
  return 0;
}
void ref_set_wall_velocity_scale(void* h, double sc) { static_cast<refdrv::Base*>(h)->set_wall_velocity_scale(sc); }
void ref_set_wall_density(void* h, double r) { static_cast<refdrv::Base*>(h)->set_wall_density(r); }
void ref_set_wall_velocity_field(void* h, const double* u3) { static_cast<refdrv::Base*>(h)->set_wall_velocity_field(u3); }
void ref_set_wall_velocity_field_scale(void* h, double sc) {
  static_cast<refdrv::Base*>(h)->set_wall_velocity_field_scale(sc);
}
void ref_set_fd_corners(void* h, int on) { static_cast<refdrv::Base*>(h)->set_fd_corners(on != 0); }
void ref_set_force_correction(void* h, int on) { static_cast<refdrv::Base*>(h)->set_force_correction(on != 0); }
int ref_set_outflow_order(void* h, int k) {
  auto* b = static_cast<refdrv::Base*>(h);
  const long long nx = b->nx();
  for (std::size_t i = 0; i < b->wall_codes.size(); ++i)
    if (b->wall_codes[i] == NrmOutXp && (long long)(i % nx) < (k >= 2 ? 2 : 1)) return -1;
  b->out_order = k;
  b->set_outflow_order(k);
  return 0;
}
void ref_set_outflow_density(void* h, double r) { static_cast<refdrv::Base*>(h)->set_outflow_density(r); }
// A solver made with forcing 2 (BoussinesqGuo): the temperature per interior
// node and the buoyancy parameters; -1 for any other solver.
int ref_set_buoyancy(void* h, const double* T, double gx, double gy, double gz, double rho0,
                     double beta, double T0) {
  return static_cast<refdrv::Base*>(h)->set_buoyancy(T, gx, gy, gz, rho0, beta, T0);
}
int ref_set_specular_nodes(void* h, const std::uint8_t* masks) {
  for (long long k = 0; k < ref_interior(h); ++k) {
    const unsigned m = masks[k];
    if (m > 0x3F) return -1;
    for (int a = 0; a < 3; ++a)
      if ((m & (1u << (2 * a))) && (m & (1u << (2 * a + 1)))) return -1;
  }
  static_cast<refdrv::Base*>(h)->set_specular_nodes(masks);
  return 0;
}
void ref_initialize(void* h, double r, double a, double b, double c) {
  static_cast<refdrv::Base*>(h)->initialize(r, a, b, c);
}
void ref_initialize_field(void* h, const double* r, const double* a, const double* b,
                          const double* c) {
  static_cast<refdrv::Base*>(h)->initialize_field(r, a, b, c);
}
void ref_step(void* h, int n, int store) { static_cast<refdrv::Base*>(h)->step(n, store); }
void ref_macro(void* h, double* r, double* a, double* b, double* c) {
  static_cast<refdrv::Base*>(h)->macro(r, a, b, c);
}
void ref_stored_macro(void* h, double* r, double* a, double* b, double* c) {
  static_cast<refdrv::Base*>(h)->stored_macro(r, a, b, c);
}
double ref_total_mass(void* h) { return static_cast<refdrv::Base*>(h)->mass(); }
double ref_total_momentum(void* h, int a) { return static_cast<refdrv::Base*>(h)->momentum(a); }
void ref_gather(void* h, double* out) { static_cast<refdrv::Base*>(h)->gather(out); }
void ref_seed(void* h, const double* in) { static_cast<refdrv::Base*>(h)->seed(in); }
double ref_slot_sum(void* h) { return static_cast<refdrv::Base*>(h)->slot_sum(); }
long long ref_n_padded(void* h) { return static_cast<refdrv::Base*>(h)->n_padded(); }
long long ref_timestep(void* h) { return static_cast<refdrv::Base*>(h)->timestep(); }

}  // extern "C"
