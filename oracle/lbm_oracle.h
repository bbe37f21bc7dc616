/*
 * CPU oracle for the M3LB lattice-Boltzmann time step -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's hot path (src/ of M3LB): Esoteric
 * Pull in-place streaming on one population array, BGK / TRT / raw MRT /
 * central-moment collision, Guo forcing, halfway bounce-back by skipping
 * solid cells.  Only the tests, the smoke check and the CPU-baseline leg of
 * the benchmark use it, as the checker; the product never calls it.
 *
 * Two builds of one body (lbm_oracle_body.h): lbmo_f64_* computes in double,
 * lbmo_f32_* in float.  `quant` emulates narrow population storage with the
 * same arithmetic: every value written into the population array is rounded
 * to IEEE binary16 (1) or bfloat16 (2), round-to-nearest-even, or to the
 * library's FP16C format (3: 1 sign, 4 exponent, 11 mantissa bits, to
 * nearest with ties away from zero, saturating at 2 - 2^-11), exactly as a
 * GPU store of a 16-bit population does.  0 stores at full precision.
 *
 * The entry points and their argument meanings are those of
 * oracle/ref/ref_driver.cpp, so a test can run the reference build and this
 * restatement side by side on one input.
 *
 * Codes: lattice 9 (D2Q9) / 27 (D3Q27); op 0 none (pure streaming), 1 BGK,
 * 2 TRT, 3 MRT, 4 central moments; eq 0 second order, 1 product form (BGK and
 * TRT only); flags per interior node: 0 fluid, 1 solid, 2 excluded, 4 specular
 * ghost wall (SpecWall), 5 on-node specular wall (SpecNode).
 *
 * set_specular_walls takes one normal code per interior node (0 none, 1..6 =
 * +x,-x,+y,-y,+z,-z outward normal) and marks the coded nodes SpecWall;
 * set_specular_nodes takes one face mask per interior node (bit 2a: outward
 * +axis a, bit 2a+1: outward -axis a) and marks the masked nodes SpecNode.
 * Both return 0, or -1 without changing anything when a value is one the
 * reference rejects (FluidSolver.hpp:193-268: a code above 6, a mask above
 * 0x3F or with both faces of one axis).
 *
 * set_regularized_walls takes a normal code per interior node (0 none, 1..6
 * axis velocity walls, 7 corner, 8 pressure outlet +x, 9 arbitrary-face
 * outflow, 10 equilibrium outlet +x) and, per node, (ux, uy, uz, rho) or
 * NULL; it marks the coded nodes RegWall (3).  The other wall setters follow
 * FluidSolver.hpp:272-370, 1311-1330.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H
#include <stdint.h>

#define LBMO_DECLARE(P)                                                              \
  void* P##create(int lattice, int op, int eq, int shifted, int forcing, int quant,  \
                  int nx, int ny, int nz, int px, int py, int pz, double omega,      \
                  double omega2, double fx, double fy, double fz);                   \
  void P##destroy(void* h);                                                          \
  void P##set_geometry(void* h, const uint8_t* flags);                               \
  int P##set_specular_walls(void* h, const uint8_t* normal_codes);                   \
  int P##set_specular_nodes(void* h, const uint8_t* face_masks);                     \
  int P##set_regularized_walls(void* h, const uint8_t* codes, const double* spec);   \
  void P##set_wall_velocity_scale(void* h, double sc);                               \
  void P##set_wall_density(void* h, double r);                                       \
  void P##set_wall_velocity_field(void* h, const double* u3);                        \
  void P##set_wall_velocity_field_scale(void* h, double sc);                         \
  void P##set_fd_corners(void* h, int on);                                           \
  void P##set_force_correction(void* h, int on);                                     \
  int P##set_outflow_order(void* h, int k);                                          \
  void P##set_outflow_density(void* h, double r);                                    \
  void P##set_buoyancy(void* h, const double* T, double gx, double gy, double gz,    \
                       double rho0, double beta, double T0);                         \
  void P##initialize(void* h, double rho, double ux, double uy, double uz);          \
  void P##initialize_field(void* h, const double* rho, const double* ux,             \
                           const double* uy, const double* uz);                      \
  void P##step(void* h, int n, int store_macro);                                     \
  void P##macro(void* h, double* rho, double* ux, double* uy, double* uz);           \
  void P##stored_macro(void* h, double* rho, double* ux, double* uy, double* uz);    \
  double P##total_mass(void* h);                                                     \
  double P##total_momentum(void* h, int axis);                                       \
  void P##gather(void* h, double* out);                                              \
  void P##seed(void* h, const double* in);                                           \
  double P##slot_sum(void* h);                                                       \
  long long P##n_padded(void* h);                                                    \
  long long P##timestep(void* h);

/* The scalar (advection-diffusion) lattice: src/solver/ScalarSolver.hpp.
 * lattice 5 (D2Q5) / 7 (D3Q7); op 1 ScalarBGK, 2 ScalarTRT, 3 ScalarRegularised;
 * lattice 9 (D2Q9) / 27 (D3Q27) with ScalarBGK;
 * cells per interior node: 0 bulk, 1 adiabatic, 2 Dirichlet, 3 excluded,
 * 4 moment (on-node Dirichlet), 5 outflow, 6 specular.  initialize_field
 * takes one value per PADDED node, as the reference's fn(n) does. */
#define LBMO_DECLARE_SCALAR(P)                                                       \
  void* P##screate(int lattice, int op, int nx, int ny, int nz, int px, int py,      \
                   int pz, double omega, double T_ref, double Lambda);               \
  void P##sdestroy(void* h);                                                         \
  void P##sset_geometry(void* h, const uint8_t* cells);                              \
  void P##sset_wall_values(void* h, const double* tw);                               \
  int P##sset_specular_walls(void* h, const uint8_t* codes);                         \
  int P##sset_specular_nodes(void* h, const uint8_t* masks);                         \
  void P##sset_omega_field(void* h, const double* omega);                            \
  void P##sset_velocity(void* h, const double* ux, const double* uy,                 \
                        const double* uz);                                           \
  void P##sfinalize_geometry(void* h);                                               \
  void P##sinitialize(void* h, double T0);                                           \
  void P##sinitialize_field(void* h, const double* T_padded);                        \
  void P##sstep(void* h, int n);                                                     \
  void P##sadd_source(void* h, const double* dC);                                    \
  void P##scompute_field(void* h);                                                   \
  void P##sfield(void* h, double* T);                                                \
  double P##stotal(void* h);                                                         \
  void P##sgather(void* h, double* out);                                             \
  long long P##sn_padded(void* h);                                                   \
  long long P##stimestep(void* h);

LBMO_DECLARE(lbmo_f64_)
LBMO_DECLARE(lbmo_f32_)
LBMO_DECLARE_SCALAR(lbmo_f64_)
LBMO_DECLARE_SCALAR(lbmo_f32_)

#endif
