/*
 * m3lb.h -- C ABI of the B200 lattice-Boltzmann step (libm3lb.so).
 *
 * One handle = one lattice resident in HBM: the Esoteric-Pull population array
 * (one array, updated in place), the cell flags and the macroscopic fields.
 * Every call returns M3LB_OK (0) or a negative status; m3lb_last_error()
 * gives the message of the calling thread's last failure.  Nothing aborts.
 * A handle is used by one host thread at a time; work is queued on the
 * handle's CUDA stream (m3lb_set_stream), and calls that hand results to the
 * host synchronise that stream.
 *
 * Each entry point replaces one member of the reference's C++ solver API
 * (paths relative to the M3LB tree, src/solver/FluidSolver.hpp unless noted);
 * the C++ headers under m3lb_b200/facade/ put those members back on top of
 * this ABI.
 *
 * Codes
 *   lattice : 9 (D2Q9), 27 (D3Q27)                 src/lattice/Lattices.hpp:75-159
 *   op      : M3LB_OP_*                              src/collision/{BGK,TRT,MomentCollision}.hpp
 *   eq      : M3LB_EQ_* (BGK and TRT only)           src/equilibrium/Equilibrium.hpp:131-136
 *   storage : M3LB_STORE_* population element type; arithmetic is FP32 for
 *             F32/F16/BF16/F16C and FP64 for F64.  16-bit storage requires
 *             shifted (except for M3LB_OP_NONE, which never reads the
 *             convention).
 *   shifted : 1 stores g = f - w (ShiftedPopulations), 0 stores f (Raw)
 *                                                    src/memory/Storage.hpp:27-35
 *   flags   : per interior node, x fastest: 0 Fluid, 1 Solid, 2 Excluded
 *                                                    src/boundary/Flags.hpp:20-33
 */
#ifndef M3LB_H
#define M3LB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define M3LB_OK 0
#define M3LB_ERR_INVALID -1     /* bad argument */
#define M3LB_ERR_UNSUPPORTED -2 /* valid in the reference, not offered here */
#define M3LB_ERR_CUDA -3        /* CUDA runtime failure */
#define M3LB_ERR_MEMORY -4      /* device or host allocation failed */

#define M3LB_OP_NONE 0 /* pure streaming: the NullCollision mock, tests/test_streaming.cpp:28-38 */
#define M3LB_OP_BGK 1  /* src/collision/BGK.hpp:33-102 */
#define M3LB_OP_TRT 2  /* src/collision/TRT.hpp:35-136 */
#define M3LB_OP_MRT 3  /* MomentCollision<.., Central=false>, MomentCollision.hpp:380-381 */
#define M3LB_OP_CM 4   /* MomentCollision<.., Central=true>,  MomentCollision.hpp:378-379 */

#define M3LB_EQ_SECOND_ORDER 0 /* SecondOrderEquilibrium, Equilibrium.hpp:49-60 */
#define M3LB_EQ_PRODUCT_FORM 1 /* ProductFormEquilibrium, Equilibrium.hpp:71-124 */

#define M3LB_STORE_F32 0
#define M3LB_STORE_F16 1
#define M3LB_STORE_BF16 2
#define M3LB_STORE_F64 3
/* FP16C: a 16-bit float with IEEE binary16's top exponent bit given to the
 * mantissa (1 sign, 4 exponent bits with bias 15, 11 mantissa bits,
 * subnormals; magnitudes up to 2 - 2^-11, larger ones and NaN saturate;
 * round to nearest, ties away from zero).  The customised 16-bit format of
 * Lehmann et al. (2022) for shifted populations: the same bytes as FP16,
 * half the rounding error.  An addition of this library; the reference
 * stores FP32 or FP64 only. */
#define M3LB_STORE_F16C 4

#define M3LB_OPT_NODE_KERNEL 1 /* value 1: always use the one-node step kernel */
#define M3LB_OPT_KERNEL 2      /* value: one of M3LB_KERNEL_* below */
/* Test only: the row kernel's wait for a row's copies gives up after `value`
 * clock cycles instead of ~2 s (0 restores the default), so a test can make
 * the wait run out and see m3lb_sync report it.  The populations of a step
 * whose wait ran out are not valid. */
#define M3LB_OPT_WAIT_CYCLES 3

/* Step kernel choice (M3LB_OPT_KERNEL).  The chunk kernels (pairs, stream,
 * rows) need a periodic x axis and even nx, the row kernel also nx up to 512
 * with 16-bit storage and up to 256 with FP32 / FP64; a choice that does not
 * apply falls back to the paired kernel, and without a periodic x axis to the
 * one-node kernel.  All choices give identical stored bits. */
#define M3LB_KERNEL_AUTO 0   /* the fastest kernel for the lattice */
#define M3LB_KERNEL_NODES 1  /* one node per thread */
#define M3LB_KERNEL_PAIRS 2  /* one warp per 64-node chunk, two nodes per lane */
#define M3LB_KERNEL_STREAM 3 /* persistent chunk kernel, asynchronous copy pipeline */
#define M3LB_KERNEL_ROWS 4   /* whole rows through shared memory by TMA (nx <= 512) */

typedef struct m3lb_solver m3lb_solver;

/* Message of the calling thread's last failed call ("" if none). */
const char* m3lb_last_error(void);

/* Bytes of HBM a lattice of this shape needs (populations, flags, macroscopic
 * fields, reduction scratch): what an admission policy budgets. */
int m3lb_footprint(int lattice, int nx, int ny, int nz, int px, int py, int pz, int storage,
                   size_t* bytes);

/* FluidSolver(const Domain&, const Collision&) (:42) with
 * Domain(nx, ny, nz, px, py, pz) (src/grid/Domain.hpp:47-56) and
 * EsotericPull<L>(Domain) (src/memory/EsotericPull.hpp:58).  Every interior
 * node starts Fluid, halo nodes Excluded (:57-63); populations start at 0.
 * Allocates on the current CUDA device. */
int m3lb_create(int lattice, int nx, int ny, int nz, int px, int py, int pz, int op, int eq,
                int storage, int shifted, int forcing, m3lb_solver** out);
int m3lb_destroy(m3lb_solver* h);

/* Public members of the collision policy: BGK::omega (BGK.hpp:43),
 * TRT::omega_p / omega_m (TRT.hpp:46-47), MomentCollision::omega /
 * omega_bulk (MomentCollision.hpp:89-90, omega2 < 0 follows omega), and
 * Guo{fx, fy, fz} (src/forcing/Forcing.hpp:58-62, used when forcing != 0). */
int m3lb_set_params(m3lb_solver* h, double omega, double omega2, double fx, double fy,
                    double fz);

/* set_geometry(fn(x, y, z) -> CellType) (:74-82), the result of fn given as
 * an array over interior nodes: 0 Fluid, 1 Solid, 2 Excluded.  Resets every
 * interior flag, wall ones included; the wall types (3, 4, 5) are set by the
 * calls below (M3LB_ERR_UNSUPPORTED for any value above 2). */
int m3lb_set_flags(m3lb_solver* h, const uint8_t* flags);

/* Normal codes of set_specular_walls (src/boundary/Regularized.hpp:97-102):
 * the outward normal of the wall. */
#define M3LB_NRM_NONE 0
#define M3LB_NRM_XP 1
#define M3LB_NRM_XM 2
#define M3LB_NRM_YP 3
#define M3LB_NRM_YM 4
#define M3LB_NRM_ZP 5
#define M3LB_NRM_ZM 6
/* Face bits of set_specular_nodes (src/boundary/Specular.hpp:226-234). */
#define M3LB_SPEC_XP 0x01
#define M3LB_SPEC_XM 0x02
#define M3LB_SPEC_YP 0x04
#define M3LB_SPEC_YM 0x08
#define M3LB_SPEC_ZP 0x10
#define M3LB_SPEC_ZM 0x20

/* set_specular_walls(fn(x, y, z) -> NormalCode) (FluidSolver.hpp:193-218),
 * one code per interior node: 0 leaves the node as it is, 1..6 marks it a
 * SpecWall, a free-slip GHOST that reflects its incoming populations about
 * that axis (f_i <- f_m(i)) and does not collide (Specular.hpp:1-90); the
 * plane lies halfway between it and the last fluid node.  Codes above 6
 * (corner, outflow) are rejected with M3LB_ERR_INVALID and nothing changes
 * (the reference aborts).  Call after m3lb_set_flags, which resets flags. */
int m3lb_set_specular_walls(m3lb_solver* h, const uint8_t* normal_codes);

/* set_specular_nodes(fn(x, y, z) -> SpecFace mask) (FluidSolver.hpp:236-268),
 * one mask per interior node: 0 leaves the node, any other mask marks it a
 * SpecNode, a fluid node that replaces each direction pointing into the
 * domain across a masked face by its mirror image (composed over the masked
 * axes, so edges and corners work) and then collides (Specular.hpp:186-278).
 * Masks above 0x3F or with both faces of one axis are rejected with
 * M3LB_ERR_INVALID and nothing changes.  While any specular node exists the
 * step runs in the one-node kernel.  Call after m3lb_set_flags. */
int m3lb_set_specular_nodes(m3lb_solver* h, const uint8_t* face_masks);

/* Normal codes of set_regularized_walls beyond the six axis walls
 * (src/boundary/Regularized.hpp:97-105). */
#define M3LB_NRM_CORNER 7   /* two or more walls meet: extrapolated density */
#define M3LB_NRM_OUT_XP 8   /* pressure outlet on +x: imposed rho, closure u_n */
#define M3LB_NRM_OUT_FREE 9 /* arbitrary-face outflow: donor rescaled to a density */
#define M3LB_NRM_OUT_EQ 10  /* equilibrium outlet on +x */

/* set_regularized_walls(fn(x, y, z) -> WallSpec) (FluidSolver.hpp:372-552):
 * per interior node a normal code (0 leaves the node; 1..6 velocity walls
 * with that outward normal; 7..10 above) and, in `states`, four doubles per
 * node (ux, uy, uz, rho: the imposed velocity, and the density the outlet
 * codes impose), or NULL for (0, 0, 0, 1).  The coded nodes become RegWall:
 * on-node walls whose populations are rebuilt from (rho, u, Pi^(1)) each
 * step before they collide (Latt et al. 2008, Regularized.hpp:1-40).
 * Codes above 10, and an outlet (8, 10) without the upstream node(s) inside
 * the domain (x < 1, or x < 2 at outflow order 2), are rejected with
 * M3LB_ERR_INVALID and nothing changes.  Call after m3lb_set_flags. */
int m3lb_set_regularized_walls(m3lb_solver* h, const uint8_t* normal_codes, const double* states);
/* set_wall_velocity_scale (:294-303): every wall velocity as given times
 * `scale` (absolute, not cumulative); densities untouched. */
int m3lb_set_wall_velocity_scale(m3lb_solver* h, double scale);
/* set_wall_density (:328-333): the density every wall state imposes. */
int m3lb_set_wall_density(m3lb_solver* h, double rho);
/* set_wall_velocity_field (:353-368): a wall velocity per interior node
 * (three doubles, x fastest), replacing the states' velocities; then
 * set_wall_velocity_field_scale scales it (absolute). */
int m3lb_set_wall_velocity_field(m3lb_solver* h, const double* u3);
int m3lb_set_wall_velocity_field_scale(m3lb_solver* h, double scale);
/* set_fd_corners (:272): corner stress from finite-difference velocity
 * gradients (default on) or from the corner's own populations. */
int m3lb_set_fd_corners(m3lb_solver* h, int on);
/* set_force_correction (:1311): the Guo corrections of the reconstruction
 * (default on; they act under BGK, the one operator whose force the wall
 * sees in the reference). */
int m3lb_set_force_correction(m3lb_solver* h, int on);
/* set_outflow_order (:1324): tangential extrapolation order at pressure
 * outlets, 1 (default) or 2. */
int m3lb_set_outflow_order(m3lb_solver* h, int order);
/* set_outflow_density (:1330): target density of arbitrary-face outflows. */
int m3lb_set_outflow_density(m3lb_solver* h, double rho);

/* Boussinesq buoyancy (BoussinesqGuo, src/forcing/Forcing.hpp:93-127): the
 * body force at a node becomes (fx, fy, fz) + g rho0 beta (T - T0), with
 * (fx, fy, fz) from m3lb_set_params, g = (gx, gy, gz) the direction a warmer
 * parcel is pushed, and T a device array of one value per interior node (x
 * fastest) in the solver's arithmetic type (FP64 for FP64 storage, else
 * FP32), read at every step; NULL returns to the uniform force.  Needs a
 * solver created with forcing. */
int m3lb_set_buoyancy(m3lb_solver* h, const void* T, double gx, double gy, double gz, double rho0,
                      double beta, double T0);
/* The same with T given on the host (doubles per interior node), copied to a
 * device array the handle owns; call again when T changes. */
int m3lb_set_buoyancy_host(m3lb_solver* h, const double* T, double gx, double gy, double gz,
                           double rho0, double beta, double T0);
/* Make the work queued on stream `then` after this call wait for what is
 * queued on stream `first` now (an event; no host wait). */
int m3lb_stream_order(void* first, void* then);
/* Device arrays of the stored rho and u (written by m3lb_step with
 * store_macro and by m3lb_macro_device), without computing them. */
int m3lb_macro_pointers(const m3lb_solver* h, void** rho, void** ux, void** uy, void** uz);
/* The CUDA stream the handle queues its work on. */
int m3lb_get_stream(const m3lb_solver* h, void** stream);

/* initialize(rho0, ux, uy, uz) (:553-561): equilibrium on fluid nodes, rest
 * equilibrium at rho0 elsewhere; resets the time step to 0. */
int m3lb_init_eq(m3lb_solver* h, double rho0, double ux, double uy, double uz);

/* initialize_field(fn(n) -> FlowState) (:568-579), the field given as four
 * host arrays over interior nodes (x fastest); non-fluid nodes at rest, rho 1. */
int m3lb_init_field_f32(m3lb_solver* h, const float* rho, const float* ux, const float* uy,
                        const float* uz);
int m3lb_init_field_f64(m3lb_solver* h, const double* rho, const double* ux, const double* uy,
                        const double* uz);
/* Same, from device arrays of the arithmetic type (float, or double for F64). */
int m3lb_init_field_device(m3lb_solver* h, const void* rho, const void* ux, const void* uy,
                           const void* uz);

/* step(store_macroscopic) (:582-591), nsteps times: one fused stream-collide
 * kernel per step.  store_macro != 0 writes rho, u of fluid nodes (the last
 * step's values remain).  Asynchronous. */
int m3lb_step(m3lb_solver* h, int nsteps, int store_macro);

/* compute_macroscopic() + rho()/ux()/uy()/uz() (:597-599, :611-614): fields of
 * every interior node at the current time (non-fluid nodes 0), to host. */
int m3lb_macro_f32(m3lb_solver* h, float* rho, float* ux, float* uy, float* uz);
int m3lb_macro_f64(m3lb_solver* h, double* rho, double* ux, double* uy, double* uz);
/* The fields as last written (by step(store_macro) or a macro call), without
 * recomputing: the reference's rho()/ux()/uy()/uz() views (:611-614). */
int m3lb_stored_macro_f64(m3lb_solver* h, double* rho, double* ux, double* uy, double* uz);
/* compute_macroscopic() into device memory; *rho.. receive device pointers to
 * arrays of the arithmetic type owned by the handle.  Asynchronous. */
int m3lb_macro_device(m3lb_solver* h, void** rho, void** ux, void** uy, void** uz);

/* total_mass() / total_momentum(a) (:601-606) summed in FP64 on the device:
 * out[0] mass, out[1..3] momentum, out[4] kinetic energy sum(rho |u|^2 / 2)
 * over fluid nodes, out[5] sum of every stored population slot
 * (EsotericPull::storage(), src/memory/EsotericPull.hpp:119-123). */
int m3lb_reduce(m3lb_solver* h, double out[6]);
/* The validation campaign's flow diagnostics, diagnostics(s, d, nx, ny, nz)
 * of validation/Campaign.hpp:99-130, on the device: compute_macroscopic,
 * then over every interior node out[0] = sum 0.5 |u|^2 (kinetic energy) and
 * out[1] = sum 0.5 |w|^2 (enstrophy), the vorticity w from central
 * differences whose neighbours wrap around the interior on every axis (w_z
 * only when nz == 1), in FP64; out[2] = the number of nodes with a
 * non-finite velocity, which add nothing (the reference's `finite` is
 * out[2] == 0).  Waits for the result. */
int m3lb_diagnostics(m3lb_solver* h, double out[3]);

/* gather_populations() (:620-624): logical populations, n_padded x Q,
 * node-major, as double, or as raw storage elements. */
int m3lb_gather(m3lb_solver* h, double* out);
int m3lb_gather_raw(m3lb_solver* h, void* out);
/* seed_populations(fn(n, i)) (:634-637), exact inverse of gather. */
int m3lb_scatter(m3lb_solver* h, const double* in);
int m3lb_scatter_raw(m3lb_solver* h, const void* in);

/* timestep() (:617), domain() extents (:608): dims receives
 * {nx, ny, nz, hx, hy, hz, sx, sy, sz, pitch, Q, storage}. */
int m3lb_timestep(const m3lb_solver* h, long long* t);
int m3lb_dims(const m3lb_solver* h, int dims[12]);
/* populations() (:609): device pointer and byte size of the population array
 * (x-chunked layout: with nch = ceil(sx / 64), element (x,y,z,q) of the
 * padded block at (((z*sy+y)*nch + x/64)*Q + q)*64 + x%64). */
int m3lb_populations(const m3lb_solver* h, void** ptr, size_t* bytes);

/* Queue the handle's work on `stream` (a cudaStream_t; NULL = legacy default). */
int m3lb_set_stream(m3lb_solver* h, void* stream);
int m3lb_sync(m3lb_solver* h);
int m3lb_set_option(m3lb_solver* h, int option, int value);
/* Kernel launches queued by this handle since creation. */
int m3lb_launch_count(const m3lb_solver* h, long long* n);

/* No counterpart in the reference: an addition of this library.
 * The reduction of m3lb_reduce for callers that cannot allocate device memory
 * (who therefore cannot create a handle, which allocates): the caller passes
 * the population array and flags it holds (device pointers, the layout of
 * m3lb_populations; flags per padded node, or NULL for an all-fluid interior),
 * the lattice description, the time step (for the parity) and a device array
 * `out` of six doubles receiving the same sums as m3lb_reduce, bit for bit,
 * on a lattice without wall nodes.  Wall nodes are not supported: this call
 * has no wall table, so a node flagged RegWall (3), SpecWall (4) or SpecNode
 * (5) counts as solid and is left out of the mass, momentum and energy sums,
 * where m3lb_reduce on a handle with walls counts RegWall and SpecNode nodes.
 * Queued on `stream`; returns without waiting.  Allocates nothing: the
 * partial sums use a fixed 768 KiB array inside the library, so at most
 * 4,194,304 interior nodes are accepted (M3LB_ERR_INVALID beyond).  The
 * first call in a CUDA context looks that array's address up (again after
 * cudaDeviceReset or under another context); make it before any stream
 * capture.  Calls share the array: calls that overlap on the GPU race. */
int m3lb_reduce_static(int lattice, int nx, int ny, int nz, int px, int py, int pz, int op,
                       int storage, int shifted, int forcing, double fx, double fy, double fz,
                       const void* populations, const uint8_t* flags, long long timestep,
                       void* stream, double* out);

/* ------------------------------------------------------------ scalar lattice
 * ScalarSolver<L, EsotericPull<L>, Collision> (src/solver/ScalarSolver.hpp):
 * an advection-diffusion lattice, D2Q5 (lattice 5, nz = 1) or D3Q7 (7) with
 * the collision operators ScalarBGK, ScalarTRT and ScalarRegularised
 * (src/collision/Scalar*.hpp), or D2Q9 (9) / D3Q27 (27) with ScalarBGK,
 * stored in FP32 or FP64.  Cell types
 * per interior node (ScalarBGK.hpp ScalarCell): 0 bulk, 1 adiabatic (zero
 * flux), 2 Dirichlet (anti-bounce-back to the wall value), 3 excluded,
 * 4 moment (the wall value imposed ON the node, MomentDirichlet.hpp), 5
 * outflow (equilibrium at a bulk donor's value), 6 specular (on-node zero
 * flux, with faces from the two specular calls).  ny and nz are at most
 * 65535. */
typedef struct m3lb_scalar m3lb_scalar;

#define M3LB_SOP_BGK 1
#define M3LB_SOP_TRT 2
#define M3LB_SOP_REGULARISED 3

int m3lb_scalar_create(int lattice, int nx, int ny, int nz, int px, int py, int pz, int op,
                       int storage, m3lb_scalar** out);
int m3lb_scalar_destroy(m3lb_scalar* h);
/* ScalarBGK::omega, T_ref (the storage reference, 0 = raw), ScalarTRT::Lambda. */
int m3lb_scalar_set_params(m3lb_scalar* h, double omega, double T_ref, double Lambda);
/* Queue the handle's work on `stream` (NULL: the default stream), as
 * m3lb_set_stream does for a fluid handle. */
int m3lb_scalar_set_stream(m3lb_scalar* h, void* stream);
/* set_geometry(fn -> ScalarCell) (:92-99): cell types 0..6 per interior node. */
int m3lb_scalar_set_cells(m3lb_scalar* h, const uint8_t* cells);
/* set_wall_values (:101-108): the value Dirichlet and moment cells impose. */
int m3lb_scalar_set_wall_values(m3lb_scalar* h, const double* values);
/* set_specular_walls (:113-132, codes 1..6) / set_specular_nodes (:140-164,
 * face masks): the faces of specular cells. */
int m3lb_scalar_set_specular_walls(m3lb_scalar* h, const uint8_t* normal_codes);
int m3lb_scalar_set_specular_nodes(m3lb_scalar* h, const uint8_t* face_masks);
/* ScalarBGK::omega_of: a relaxation rate per interior node (NULL: uniform). */
int m3lb_scalar_set_omega_field(m3lb_scalar* h, const double* omega);
/* set_velocity (:166-168): device arrays of the advecting velocity per
 * interior node in the arithmetic type, read at every step (NULL: at rest). */
int m3lb_scalar_set_velocity_device(m3lb_scalar* h, const void* ux, const void* uy, const void* uz);
/* The advecting velocity given on the host (doubles per interior node),
 * copied to arrays the handle owns (NULL: at rest). */
int m3lb_scalar_set_velocity_host(m3lb_scalar* h, const double* ux, const double* uy,
                                  const double* uz);
int m3lb_scalar_get_stream(const m3lb_scalar* h, void** stream);
/* finalize_geometry (:223-296): moment-cell unknowns and outflow donors. */
int m3lb_scalar_finalize_geometry(m3lb_scalar* h);
/* initialize(T0) / initialize_field(fn(n)) (:170-190); the field is given
 * per PADDED node (n_padded values, x fastest). */
int m3lb_scalar_init(m3lb_scalar* h, double T0);
int m3lb_scalar_init_field(m3lb_scalar* h, const double* T_padded);
/* step() (:192-203): the lattice step, then the outflow pass. */
int m3lb_scalar_step(m3lb_scalar* h, int nsteps);
/* add_source(fn(n)) (:205-208, 421-437): dC per interior node. */
int m3lb_scalar_add_source(m3lb_scalar* h, const double* dC);
int m3lb_scalar_add_source_device(m3lb_scalar* h, const void* dC);
/* compute_field() (:210-212), then temperature(): the field per interior
 * node on the host, or its device array. */
int m3lb_scalar_compute_field(m3lb_scalar* h);
int m3lb_scalar_field(m3lb_scalar* h, double* T);
int m3lb_scalar_field_device(m3lb_scalar* h, void** T);
/* total_population() (:219-228), summed in FP64. */
int m3lb_scalar_total(m3lb_scalar* h, double* out);
/* Logical populations per padded node (n_padded x Q doubles). */
int m3lb_scalar_gather(m3lb_scalar* h, double* out);
int m3lb_scalar_info(const m3lb_scalar* h, long long* n_padded, long long* timestep,
                     long long* launches);
int m3lb_scalar_sync(m3lb_scalar* h);
/* Two-way thermal coupling of lattices of the same extent and arithmetic
 * type, as the reference's drivers wire it (force.T = th.temperature();
 * th.set_velocity(fl.ux(), fl.uy(), fl.uz()), validation/rayleigh_benard.cpp):
 * the fluid's Boussinesq force reads the scalar's field, the scalar is
 * advected by the fluid's stored velocity (store_macro), and the scalar's
 * work goes onto the fluid's stream so the two alternate in order.  The
 * scalar must not be stepped after the fluid is destroyed (destroying the
 * scalar afterwards is safe). */
int m3lb_couple_thermal(m3lb_solver* fluid, m3lb_scalar* scalar, double gx, double gy, double gz,
                        double rho0, double beta, double T0);

/* ------------------------------------------------------------ serving loop
 * Many independent lattices resident on one GPU and advanced together (no
 * counterpart in the reference, which runs one solver per process).  A
 * request is a periodic D3Q27 Taylor-Green box of extent N (even) with one of
 * the BGK, TRT, MRT or CM operators (shifted populations, no force), an
 * amplitude u0, relaxation rates and a step count.  Requests are admitted in
 * arrival order while their footprint (populations plus 16 B per node of
 * seed/readout fields) fits hbm_budget; every admitted lattice stays resident
 * until its last step.  Each time step of a round is one batched launch per
 * operator (and, through the row kernel, row width) over all resident
 * lattices, replayed from a CUDA graph (see M3LB_MAP_ROWS).  Results are FP64 mass, momentum and energy of
 * the final state (and rho, u with keep_fields); a request's result is
 * bit-identical alone, in any mix, and through m3lb_step with
 * M3LB_KERNEL_PAIRS. */
typedef struct m3lb_server m3lb_server;

typedef struct {
  size_t hbm_budget;  /* bytes the resident lattices may hold */
  int max_resident;   /* most lattices resident at once (0: budget only; at most 1024) */
  int round_steps;    /* most time steps per scheduling round (>= 1) */
  int storage;        /* M3LB_STORE_F16, _F16C, _BF16 or _F32, for every request */
  int keep_fields;    /* 1: keep rho, u of finished requests for m3lb_serve_fields */
  int mapping;        /* how the batched launches map lattices to warps: M3LB_MAP_AUTO (0),
                         _CHUNKS, _DENSE, _TUNE or _ROWS (same results, different speed) */
} m3lb_serve_config;

/* M3LB_MAP_CHUNKS: a warp updates one 64-slot chunk of a row (lanes past the
 * row's end idle when N is not a multiple of 64).  M3LB_MAP_DENSE: a warp
 * updates 64 consecutive nodes in x-fastest order, rows packed back to back,
 * so no lane idles.  M3LB_MAP_ROWS (16-bit storage): the row kernel, a CTA
 * moving whole x-rows of any lattice of its group through shared memory by
 * TMA, one persistent launch per step and (operator, row width) group;
 * rounds run their full length, a lattice that finishes inside a round sits
 * the rest of it out, and each (groups present, length) is captured into a
 * CUDA graph once and replayed whatever lattices come and go.
 * M3LB_MAP_AUTO: rows with 16-bit storage; otherwise dense for an operator's
 * launch when one of its lattices has N not a multiple of 64, chunks
 * otherwise.  M3LB_MAP_TUNE: an autotuner on the live stream: the first
 * rounds alternate the three (two without 16-bit storage), each timed on the
 * device (CUDA events around the round's launches) for 6 rounds, and the one
 * with the most lattice updates per second serves every later round
 * (reported in m3lb_serve_stats). */
#define M3LB_MAP_AUTO 0
#define M3LB_MAP_CHUNKS 1
#define M3LB_MAP_DENSE 2
#define M3LB_MAP_TUNE 3
#define M3LB_MAP_ROWS 4

typedef struct {
  long long id;         /* caller's tag */
  double arrival;       /* seconds after m3lb_serve_run starts */
  int n;                /* extent of the N^3 periodic box */
  int op;               /* M3LB_OP_BGK, _TRT, _MRT or _CM */
  int steps;            /* time steps */
  double u0;            /* Taylor-Green amplitude (the field of m3lb_tgv_field) */
  double omega, omega2; /* rates as in m3lb_set_params */
} m3lb_request;

typedef struct {
  long long id;
  double arrival, admitted, finished; /* seconds after the run started */
  int n, op, steps, status;
  long long node_steps;               /* n^3 * steps */
  double mass, momentum[3], energy;   /* FP64 reductions of the final state */
} m3lb_result;

typedef struct {
  long long rounds;         /* scheduling rounds */
  long long launches;       /* batched kernel launches (direct or in graphs) */
  long long graph_captures; /* rounds captured into a CUDA graph */
  long long graph_launches; /* rounds replayed from a graph */
  long long finished;       /* requests completed */
  long long node_steps;     /* sum of n^3 * steps over completed requests */
  double makespan;          /* seconds from the start of the last run to its end */
  long long dense_launches; /* batched launches with the dense mapping */
  int tuned_mapping;         /* M3LB_MAP_TUNE: the mapping chosen (_CHUNKS, _DENSE or _ROWS), 0 before */
  double tuned_chunks_mlups; /* the tuner's measured rates of its candidates (MLUPS) */
  double tuned_dense_mlups;
  long long rows_launches;   /* batched launches through the row kernel */
  double tuned_rows_mlups;
} m3lb_serve_stats;

int m3lb_serve_create(const m3lb_serve_config* cfg, m3lb_server** out);
/* Queue a request for the next m3lb_serve_run. */
int m3lb_serve_submit(m3lb_server* s, const m3lb_request* r);
/* Serve every submitted request, honouring arrival times (the loop waits for
 * them in real time); time_limit > 0 bounds the run in seconds. */
int m3lb_serve_run(m3lb_server* s, double time_limit);
/* Finished requests in completion order; *count = how many exist. */
int m3lb_serve_results(const m3lb_server* s, m3lb_result* out, int cap, int* count);
/* Host copies (n^3 floats each, x fastest) of a finished request's rho, u. */
int m3lb_serve_fields(const m3lb_server* s, long long id, float* rho, float* ux, float* uy,
                      float* uz);
int m3lb_serve_get_stats(const m3lb_server* s, m3lb_serve_stats* st);
int m3lb_serve_destroy(m3lb_server* s);
/* The serving loop's initial field into device arrays (n^3 floats each):
 * Taylor-Green u = u0 sin x cos y cos z, v = -u0 cos x sin y cos z, w = 0,
 * rho = 1 + 3 u0^2 / 16 (cos 2x + cos 2y)(cos 2z + 2), x = 2 pi i / n. */
int m3lb_tgv_field(int n, double u0, float* rho, float* ux, float* uy, float* uz, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* M3LB_H */
