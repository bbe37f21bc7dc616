// C ABI of the lattice-Boltzmann step (include/m3lb.h): handle lifetime,
// device memory, parity bookkeeping and dispatch into the launcher tables.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/m3lb.h"
#include "lbm_diag.cuh"
#include "lbm_host.h"
#include "lbm_walls.h"

using namespace m3lb;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CUDA_TRY(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      return fail(M3LB_ERR_CUDA, "%s: %s (%s)", #call, cudaGetErrorString(e_),      \
                  cudaGetErrorName(e_));                                            \
  } while (0)

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev) {
      prev = cur;
      cudaSetDevice(dev);
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

namespace m3lb {
// Lets other translation units of the library report through m3lb_last_error().
void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }

int elem_bytes(int storage) {
  switch (storage) {
    case M3LB_STORE_F32: return 4;
    case M3LB_STORE_F64: return 8;
    case M3LB_STORE_F16:
    case M3LB_STORE_BF16:
    case M3LB_STORE_F16C: return 2;
    default: return 0;
  }
}
int real_bytes(int storage) { return storage == M3LB_STORE_F64 ? 8 : 4; }

// Domain(nx, ny, nz, px, py, pz) geometry (src/grid/Domain.hpp:47-56, 104-108).
Geo make_geo(int nx, int ny, int nz, int px, int py, int pz) {
  auto halo = [](int n, int per) { return n <= 1 ? 0 : (per ? 0 : 1); };
  Geo g{};
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.px = px != 0; g.py = py != 0; g.pz = pz != 0;
  g.hx = halo(nx, g.px); g.hy = halo(ny, g.py); g.hz = halo(nz, g.pz);
  g.sx = nx + 2 * g.hx; g.sy = ny + 2 * g.hy; g.sz = nz + 2 * g.hz;
  g.nch = (g.sx + kChunk - 1) / kChunk;
  g.n_padded = (long long)g.sx * g.sy * g.sz;
  return g;
}

int reduce_blocks(const Geo& g) {
  const long long n = std::max<long long>((long long)g.nx * g.ny * g.nz, 1);
  return (int)std::min<long long>((n + kReduceThreads - 1) / kReduceThreads, 4 * 148);
}

size_t pop_elems(const Geo& g, int Q) {
  return (size_t)g.sz * g.sy * g.nch * Q * kChunk;
}

const Launchers* table_for(int lattice, int storage) {
  if (lattice == 9) {
    switch (storage) {
      case M3LB_STORE_F32: return launchers_D2Q9_F32();
      case M3LB_STORE_F16: return launchers_D2Q9_F16();
      case M3LB_STORE_BF16: return launchers_D2Q9_BF16();
      case M3LB_STORE_F64: return launchers_D2Q9_F64();
      case M3LB_STORE_F16C: return launchers_D2Q9_F16C();
    }
  } else if (lattice == 27) {
    switch (storage) {
      case M3LB_STORE_F32: return launchers_D3Q27_F32();
      case M3LB_STORE_F16: return launchers_D3Q27_F16();
      case M3LB_STORE_BF16: return launchers_D3Q27_BF16();
      case M3LB_STORE_F64: return launchers_D3Q27_F64();
      case M3LB_STORE_F16C: return launchers_D3Q27_F16C();
    }
  }
  return nullptr;
}
}  // namespace m3lb

// Shortest rows (in 64-node chunks) the automatic choice sends to the row
// kernel with 16-bit storage.
constexpr int kAutoRowsMinChunks = 2;

struct m3lb_solver {
  int lattice = 27, Q = 27, op = 0, eq = 0, storage = 0, shifted = 1, forcing = 0;
  Geo g{};
  int device = 0;
  cudaStream_t stream = nullptr;     // where the work is queued
  cudaStream_t own = nullptr;        // the stream the handle created
  void* f = nullptr;                 // populations
  size_t f_bytes = 0;
  uint8_t* flags = nullptr;          // per padded node
  uint8_t* row_flags = nullptr;      // per padded row: any interior node not fluid
  std::vector<uint8_t> flags_host;   // per padded node
  bool has_geometry = false;
  // wall nodes (regularised and free-slip) and their device list
  WallSet walls;
  // Boussinesq buoyancy: temperature per interior node (arithmetic type)
  const void* temp = nullptr;
  double bg[3] = {0, 0, 0}, brho0 = 1, bbeta = 1, bT0 = 0;
  void* temp_own = nullptr;          // m3lb_set_buoyancy_host's copy of T
  void* macro[4] = {nullptr, nullptr, nullptr, nullptr};  // interior, arithmetic type
  void* staging = nullptr;           // init_field uploads (4 interior arrays)
  double* partials = nullptr;        // reduction scratch
  double* red_out = nullptr;
  int* err = nullptr;                // device status word (after red_out)
  int nblocks = 0;
  long long t = 0;
  long long launches = 0;
  double omega = 1, omega2 = -1, fx = 0, fy = 0, fz = 0;
  bool node_kernel = false;
  int kernel = M3LB_KERNEL_AUTO;     // M3LB_OPT_KERNEL
  long long wait_cycles = 0;         // M3LB_OPT_WAIT_CYCLES (test only; 0 = default)
  const Launchers* L = nullptr;

  long long n_interior() const { return (long long)g.nx * g.ny * g.nz; }
  StepArgs args() const {
    StepArgs a{};
    a.g = g;
    a.f = f;
    a.flags = has_geometry ? flags : nullptr;
    a.row_flags = has_geometry ? row_flags : nullptr;
    a.spec = walls.count ? walls.spec : nullptr;
    a.parity = (int)(t & 1);
    a.omega = omega; a.omega2 = omega2;
    a.fx = forcing ? fx : 0; a.fy = forcing ? fy : 0; a.fz = forcing ? fz : 0;
    a.err = err;
    a.wait_cycles = wait_cycles;
    if (forcing && temp) {
      a.temp = temp;
      a.bgx = bg[0]; a.bgy = bg[1]; a.bgz = bg[2];
      a.brho0 = brho0; a.bbeta = bbeta; a.bT0 = bT0;
    }
    return a;
  }
  // The chunk kernels need a periodic x axis (no x halo) and even nx; the
  // one-node kernel runs everything.
  bool chunk_ok() const { return g.px && g.hx == 0 && (g.nx % 2) == 0; }
  int step_kernel() const {
    if (node_kernel || !chunk_ok() || kernel == M3LB_KERNEL_NODES) return kKernelNodes;
    // the streamed kernel addresses rows with 32-bit element counts
    const bool rows32 = (long long)g.nch * Q * 64 < (1LL << 31);
    // the row kernel: whole rows of at most 8 chunks with 16-bit storage, 4
    // with 32- or 64-bit storage (the last chunk may be partial), in stages
    // of 2, 3, 4 or 8 chunks that must fit a CTA's shared memory
    const int lw = g.nch <= 2 ? 2 : (g.nch == 3 ? 3 : (g.nch <= 4 ? 4 : 8));
    const bool rows_ok = g.nch <= (elem_bytes(storage) == 2 ? 8 : 4) &&
                         4LL * Q * lw * 64 * elem_bytes(storage) + 84 <= 227LL * 1024;
    if (kernel == M3LB_KERNEL_ROWS && rows_ok) return kKernelRows;
    if (kernel == M3LB_KERNEL_STREAM && rows32) return kKernelStream;
    // auto, from measurements on B200: with 16-bit storage the row kernel
    // for rows of at least kAutoRowsMinChunks chunks (256^3 CM: 0.34 ms
    // against 0.49 ms for the paired kernel), else the streamed kernel for
    // BGK/TRT and pure streaming; the paired kernel for everything else
    // (32/64-bit storage is already near the copy bandwidth with it)
    const bool narrow = elem_bytes(storage) == 2;
    if (kernel == M3LB_KERNEL_AUTO && narrow && rows_ok && g.nch >= kAutoRowsMinChunks)
      return kKernelRows;
    if (kernel == M3LB_KERNEL_AUTO && rows32 && narrow && op <= M3LB_OP_TRT) return kKernelStream;
    return kKernelPairs;
  }
};

extern "C" {

const char* m3lb_last_error(void) { return g_last_error.c_str(); }

int m3lb_footprint(int lattice, int nx, int ny, int nz, int px, int py, int pz, int storage,
                   size_t* bytes) {
  if (!bytes) return fail(M3LB_ERR_INVALID, "footprint: null output");
  if ((lattice != 9 && lattice != 27) || nx < 1 || ny < 1 || nz < 1 || !elem_bytes(storage))
    return fail(M3LB_ERR_INVALID, "footprint: bad lattice/extent/storage");
  const Geo g = make_geo(nx, ny, nz, px, py, pz);
  const size_t nint = (size_t)nx * ny * nz;
  *bytes = pop_elems(g, lattice) * elem_bytes(storage) + (size_t)g.n_padded +
           4 * nint * real_bytes(storage) + (size_t)reduce_blocks(g) * kReduceVals * 8 + 64;
  return M3LB_OK;
}

int m3lb_create(int lattice, int nx, int ny, int nz, int px, int py, int pz, int op, int eq,
                int storage, int shifted, int forcing, m3lb_solver** out) {
  if (!out) return fail(M3LB_ERR_INVALID, "create: null output handle");
  *out = nullptr;
  if (lattice != 9 && lattice != 27) return fail(M3LB_ERR_INVALID, "create: lattice must be 9 or 27");
  if (nx < 1 || ny < 1 || nz < 1) return fail(M3LB_ERR_INVALID, "create: extents must be >= 1");
  if (lattice == 9 && nz != 1) return fail(M3LB_ERR_INVALID, "create: D2Q9 needs nz == 1");
  if (op < M3LB_OP_NONE || op > M3LB_OP_CM) return fail(M3LB_ERR_INVALID, "create: bad operator %d", op);
  if (eq != 0 && eq != 1) return fail(M3LB_ERR_INVALID, "create: bad equilibrium %d", eq);
  if (!elem_bytes(storage)) return fail(M3LB_ERR_INVALID, "create: bad storage %d", storage);
  if (!shifted && op != M3LB_OP_NONE && elem_bytes(storage) == 2)
    return fail(M3LB_ERR_UNSUPPORTED, "create: 16-bit storage holds shifted populations only");
  const long long npad = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  if (npad > (1LL << 31)) return fail(M3LB_ERR_INVALID, "create: lattice exceeds 2^31 nodes");

  auto* h = new m3lb_solver();
  h->lattice = lattice; h->Q = lattice; h->op = op; h->eq = eq; h->storage = storage;
  h->shifted = shifted ? 1 : 0; h->forcing = forcing ? 1 : 0;
  h->g = make_geo(nx, ny, nz, px, py, pz);
  h->L = table_for(lattice, storage);
  cudaGetDevice(&h->device);
  auto cleanup = [&](int code) { m3lb_destroy(h); return code; };

  h->f_bytes = pop_elems(h->g, lattice) * elem_bytes(storage);
  if (cudaMalloc(&h->f, h->f_bytes) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_MEMORY, "create: cannot allocate %zu bytes of populations", h->f_bytes));
  if (cudaMalloc((void**)&h->flags, (size_t)h->g.n_padded) != cudaSuccess ||
      cudaMalloc((void**)&h->row_flags, (size_t)h->g.sy * h->g.sz) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_MEMORY, "create: cannot allocate flags"));
  const size_t mb = (size_t)h->n_interior() * real_bytes(storage);
  for (int i = 0; i < 4; ++i)
    if (cudaMalloc(&h->macro[i], mb) != cudaSuccess)
      return cleanup(fail(M3LB_ERR_MEMORY, "create: cannot allocate macroscopic fields"));
  h->nblocks = reduce_blocks(h->g);
  if (cudaMalloc((void**)&h->partials, (size_t)h->nblocks * kReduceVals * 8 + 64) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_MEMORY, "create: cannot allocate reduction scratch"));
  h->red_out = h->partials + (size_t)h->nblocks * kReduceVals;
  h->err = reinterpret_cast<int*>(h->red_out + kReduceVals);
  if (cudaMemset(h->err, 0, sizeof(int)) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_CUDA, "create: cannot clear the status word"));
  if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_CUDA, "create: cannot create stream"));
  h->stream = h->own;

  // Every interior node Fluid, halo Excluded (FluidSolver.hpp:57-63).
  h->flags_host.assign((size_t)h->g.n_padded, 0);
  const Geo& g = h->g;
  for (int z = 0; z < g.sz; ++z)
    for (int y = 0; y < g.sy; ++y)
      for (int x = 0; x < g.sx; ++x) {
        const bool in = x >= g.hx && x < g.hx + g.nx && y >= g.hy && y < g.hy + g.ny &&
                        z >= g.hz && z < g.hz + g.nz;
        h->flags_host[((size_t)z * g.sy + y) * g.sx + x] = in ? 0 : 2;
      }
  if (cudaMemcpy(h->flags, h->flags_host.data(), (size_t)g.n_padded, cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemsetAsync(h->f, 0, h->f_bytes, h->stream) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_CUDA, "create: initial copies failed"));
  for (int i = 0; i < 4; ++i)
    if (cudaMemsetAsync(h->macro[i], 0, mb, h->stream) != cudaSuccess)
      return cleanup(fail(M3LB_ERR_CUDA, "create: initial copies failed"));
  if (cudaStreamSynchronize(h->stream) != cudaSuccess)
    return cleanup(fail(M3LB_ERR_CUDA, "create: initial copies failed"));
  *out = h;
  return M3LB_OK;
}

int m3lb_destroy(m3lb_solver* h) {
  if (!h) return M3LB_OK;
  DeviceGuard dg(h->device);
  // the queue may be a caller's stream, possibly gone already: wait for the
  // whole device rather than for that stream
  cudaDeviceSynchronize();
  cudaFree(h->f);
  cudaFree(h->flags);
  cudaFree(h->row_flags);
  cudaFree(h->temp_own);
  h->walls.release();
  for (void* p : h->macro) cudaFree(p);
  cudaFree(h->staging);
  cudaFree(h->partials);
  if (h->own) cudaStreamDestroy(h->own);
  delete h;
  return M3LB_OK;
}

int m3lb_set_params(m3lb_solver* h, double omega, double omega2, double fx, double fy, double fz) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_params: null handle");
  h->omega = omega; h->omega2 = omega2; h->fx = fx; h->fy = fy; h->fz = fz;
  return M3LB_OK;
}

}  // extern "C"

// Upload the host flags, with the per-row summary the row kernel reads to
// skip the flag loads of rows that are all fluid, and rebuild the wall-node
// list.
static int upload_geometry(m3lb_solver* h) {
  const Geo& g = h->g;
  bool any = false;
  std::vector<uint8_t> rows((size_t)g.sy * g.sz, 0);
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y) {
      const size_t r = (size_t)(z + g.hz) * g.sy + (y + g.hy);
      bool row = false;
      for (int x = 0; x < g.nx; ++x) row |= h->flags_host[r * g.sx + (x + g.hx)] != 0;
      rows[r] = row ? 1 : 0;
      any |= row;
    }
  DeviceGuard dg(h->device);
  CUDA_TRY(cudaMemcpyAsync(h->flags, h->flags_host.data(), (size_t)g.n_padded,
                           cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(cudaMemcpyAsync(h->row_flags, rows.data(), rows.size(), cudaMemcpyHostToDevice,
                           h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->has_geometry = any;
  return h->walls.build(g, h->lattice, h->op, h->storage, h->flags_host, h->stream);
}
static int rebuild_walls(m3lb_solver* h) {
  DeviceGuard dg(h->device);
  return h->walls.build(h->g, h->lattice, h->op, h->storage, h->flags_host, h->stream);
}

extern "C" {
int m3lb_set_flags(m3lb_solver* h, const uint8_t* fl) {
  if (!h || !fl) return fail(M3LB_ERR_INVALID, "set_flags: null argument");
  const Geo& g = h->g;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const uint8_t v = fl[((size_t)z * g.ny + y) * g.nx + x];
        if (v > 2)
          return fail(M3LB_ERR_UNSUPPORTED,
                      "set_flags: cell type %u at (%d,%d,%d): Fluid, Solid and Excluded are set "
                      "here, specular walls by m3lb_set_specular_walls / _nodes", (unsigned)v, x,
                      y, z);
      }
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x)
        h->flags_host[((size_t)(z + g.hz) * g.sy + (y + g.hy)) * g.sx + (x + g.hx)] =
            fl[((size_t)z * g.ny + y) * g.nx + x];
  return upload_geometry(h);
}

int m3lb_set_specular_walls(m3lb_solver* h, const uint8_t* codes) {
  if (!h || !codes) return fail(M3LB_ERR_INVALID, "set_specular_walls: null argument");
  const Geo& g = h->g;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const unsigned c = codes[((size_t)z * g.ny + y) * g.nx + x];
        if (c > 6)
          return fail(M3LB_ERR_INVALID,
                      "set_specular_walls: normal code %u at (%d,%d,%d) is not an axis normal; "
                      "specular reflection is defined for codes 1..6 only", c, x, y, z);
      }
  h->walls.spec_nrm.assign((size_t)g.n_padded, 0);
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const uint8_t c = codes[((size_t)z * g.ny + y) * g.nx + x];
        if (!c) continue;
        const size_t n = ((size_t)(z + g.hz) * g.sy + (y + g.hy)) * g.sx + (x + g.hx);
        h->walls.spec_nrm[n] = c;
        h->flags_host[n] = kSpecWall;
      }
  return upload_geometry(h);
}

int m3lb_set_specular_nodes(m3lb_solver* h, const uint8_t* masks) {
  if (!h || !masks) return fail(M3LB_ERR_INVALID, "set_specular_nodes: null argument");
  const Geo& g = h->g;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const unsigned m = masks[((size_t)z * g.ny + y) * g.nx + x];
        if (m > 0x3F)
          return fail(M3LB_ERR_INVALID,
                      "set_specular_nodes: mask %u at (%d,%d,%d) has bits outside the six faces",
                      m, x, y, z);
        for (int a = 0; a < 3; ++a)
          if ((m & (1u << (2 * a))) && (m & (1u << (2 * a + 1))))
            return fail(M3LB_ERR_INVALID,
                        "set_specular_nodes: mask %u at (%d,%d,%d) carries both faces of axis %d; "
                        "an on-node mirror needs one plane per axis", m, x, y, z, a);
      }
  h->walls.spec_faces.assign((size_t)g.n_padded, 0);
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const uint8_t m = masks[((size_t)z * g.ny + y) * g.nx + x];
        if (!m) continue;
        const size_t n = ((size_t)(z + g.hz) * g.sy + (y + g.hy)) * g.sx + (x + g.hx);
        h->walls.spec_faces[n] = m;
        h->flags_host[n] = kSpecNode;
      }
  return upload_geometry(h);
}

int m3lb_set_regularized_walls(m3lb_solver* h, const uint8_t* codes, const double* states) {
  if (!h || !codes) return fail(M3LB_ERR_INVALID, "set_regularized_walls: null argument");
  const int rc = h->walls.set_regularized(h->g, h->lattice, h->flags_host, codes, states);
  if (rc) return rc;
  return upload_geometry(h);
}
int m3lb_set_wall_velocity_scale(m3lb_solver* h, double scale) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_wall_velocity_scale: null handle");
  h->walls.scale = scale;
  return M3LB_OK;
}
int m3lb_set_wall_density(m3lb_solver* h, double rho) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_wall_density: null handle");
  for (auto& kv : h->walls.reg) kv.second.u[3] = rho;
  return rebuild_walls(h);
}
int m3lb_set_wall_velocity_field(m3lb_solver* h, const double* u3) {
  if (!h || !u3) return fail(M3LB_ERR_INVALID, "set_wall_velocity_field: null argument");
  h->walls.field.assign(u3, u3 + 3 * (size_t)h->n_interior());
  h->walls.field_on = true;
  h->walls.field_scale = 1;
  return rebuild_walls(h);
}
int m3lb_set_wall_velocity_field_scale(m3lb_solver* h, double scale) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_wall_velocity_field_scale: null handle");
  h->walls.field_scale = scale;
  return M3LB_OK;
}
int m3lb_set_fd_corners(m3lb_solver* h, int on) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_fd_corners: null handle");
  h->walls.fd_corners = on != 0;
  return rebuild_walls(h);
}
int m3lb_set_force_correction(m3lb_solver* h, int on) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_force_correction: null handle");
  h->walls.force_bc = on != 0;
  return M3LB_OK;
}
int m3lb_set_outflow_order(m3lb_solver* h, int order) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_outflow_order: null handle");
  for (const auto& kv : h->walls.reg) {
    if (kv.second.code != kNrmOutXp || h->flags_host[kv.first] != kRegWall) continue;
    const int x = (int)(kv.first % h->g.sx) - h->g.hx;
    if (x < (order >= 2 ? 2 : 1))
      return fail(M3LB_ERR_INVALID, "set_outflow_order: the pressure outlet node at x = %d has no "
                  "second upstream node inside the domain", x);
  }
  h->walls.out_order = order;
  return rebuild_walls(h);
}
int m3lb_set_buoyancy(m3lb_solver* h, const void* T, double gx, double gy, double gz, double rho0,
                      double beta, double T0) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_buoyancy: null handle");
  if (T && !h->forcing)
    return fail(M3LB_ERR_INVALID, "set_buoyancy: the solver was created without forcing");
  h->temp = T;
  h->bg[0] = gx; h->bg[1] = gy; h->bg[2] = gz;
  h->brho0 = rho0; h->bbeta = beta; h->bT0 = T0;
  return M3LB_OK;
}
int m3lb_set_buoyancy_host(m3lb_solver* h, const double* T, double gx, double gy, double gz,
                           double rho0, double beta, double T0) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_buoyancy: null handle");
  if (!T) return m3lb_set_buoyancy(h, nullptr, gx, gy, gz, rho0, beta, T0);
  if (!h->forcing) return fail(M3LB_ERR_INVALID, "set_buoyancy: the solver was created without forcing");
  DeviceGuard dg(h->device);
  const size_t n = (size_t)h->n_interior(), rb = real_bytes(h->storage);
  if (!h->temp_own && cudaMalloc(&h->temp_own, n * rb) != cudaSuccess) {
    h->temp_own = nullptr;
    return fail(M3LB_ERR_MEMORY, "set_buoyancy: cannot allocate %zu bytes", n * rb);
  }
  std::vector<char> tmp(n * rb);
  for (size_t i = 0; i < n; ++i) {
    if (rb == 8) reinterpret_cast<double*>(tmp.data())[i] = T[i];
    else reinterpret_cast<float*>(tmp.data())[i] = (float)T[i];
  }
  CUDA_TRY(cudaMemcpyAsync(h->temp_own, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return m3lb_set_buoyancy(h, h->temp_own, gx, gy, gz, rho0, beta, T0);
}
int m3lb_stream_order(void* first, void* then) {
  if (first == then) return M3LB_OK;
  cudaEvent_t e;
  CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaError_t r = cudaEventRecord(e, (cudaStream_t)first);
  if (r == cudaSuccess) r = cudaStreamWaitEvent((cudaStream_t)then, e, 0);
  cudaEventDestroy(e);
  if (r != cudaSuccess) return fail(M3LB_ERR_CUDA, "stream_order: %s", cudaGetErrorString(r));
  return M3LB_OK;
}
int m3lb_macro_pointers(const m3lb_solver* h, void** rho, void** ux, void** uy, void** uz) {
  if (!h) return fail(M3LB_ERR_INVALID, "macro_pointers: null handle");
  if (rho) *rho = h->macro[0];
  if (ux) *ux = h->macro[1];
  if (uy) *uy = h->macro[2];
  if (uz) *uz = h->macro[3];
  return M3LB_OK;
}
int m3lb_get_stream(const m3lb_solver* h, void** stream) {
  if (!h || !stream) return fail(M3LB_ERR_INVALID, "get_stream: null argument");
  *stream = (void*)h->stream;
  return M3LB_OK;
}
int m3lb_set_outflow_density(m3lb_solver* h, double rho) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_outflow_density: null handle");
  h->walls.out_rho = rho;
  return M3LB_OK;
}

}  // extern "C"

// The boundary pass around one bulk step (lbm_bound.cuh): snapshots of the
// nodes read before their update and the corner densities ahead of the bulk
// kernel; the wall nodes, level by level, after it.
static int bound_before(m3lb_solver* h, const StepArgs& a, int* n) {
  const WallSet& w = h->walls;
  if (!w.count) return M3LB_OK;
  const BoundArgs b = w.args(0, w.count);
  const bool sh = h->shifted != 0, fo = h->forcing != 0;
  if (w.nsnap) {
    CUDA_TRY(h->L->bound(a, b, kBndSnapshot, h->op, h->eq, sh, fo, h->stream));
    *n += 1;
  }
  if (w.corners) {
    CUDA_TRY(h->L->bound(a, b, kBndCornerRho, h->op, h->eq, sh, fo, h->stream));
    *n += 2;
  }
  return M3LB_OK;
}
static int bound_after(m3lb_solver* h, const StepArgs& a, int* n) {
  const WallSet& w = h->walls;
  int begin = 0;
  for (int end : w.level_end) {
    CUDA_TRY(h->L->bound(a, w.args(begin, end), kBndUpdate, h->op, h->eq, h->shifted != 0,
                         h->forcing != 0, h->stream));
    *n += 1;
    begin = end;
  }
  return M3LB_OK;
}

extern "C" {
static int seed(m3lb_solver* h, SeedArgs& a) {
  a.g = h->g;
  a.f = h->f;
  a.flags = h->flags;
  a.parity = (int)(h->t & 1);
  CUDA_TRY(h->L->seed(a, h->op, h->eq, h->shifted != 0, h->stream));
  h->launches += 1;
  return M3LB_OK;
}

int m3lb_init_eq(m3lb_solver* h, double rho0, double ux, double uy, double uz) {
  if (!h) return fail(M3LB_ERR_INVALID, "init_eq: null handle");
  DeviceGuard dg(h->device);
  h->t = 0;
  SeedArgs a{};
  a.mode = 0;
  a.rho0 = rho0; a.ux0 = ux; a.uy0 = uy; a.uz0 = uz;
  return seed(h, a);
}

static int ensure_staging(m3lb_solver* h) {
  if (h->staging) return M3LB_OK;
  const size_t b = 4 * (size_t)h->n_interior() * real_bytes(h->storage);
  if (cudaMalloc(&h->staging, b) != cudaSuccess)
    return fail(M3LB_ERR_MEMORY, "init_field: cannot allocate %zu bytes of staging", b);
  return M3LB_OK;
}

int m3lb_init_field_device(m3lb_solver* h, const void* rho, const void* ux, const void* uy,
                           const void* uz) {
  if (!h || !rho || !ux || !uy || !uz) return fail(M3LB_ERR_INVALID, "init_field: null argument");
  DeviceGuard dg(h->device);
  h->t = 0;
  SeedArgs a{};
  a.mode = 1;
  a.rho0 = 1;
  a.rho = rho; a.ux = ux; a.uy = uy; a.uz = uz;
  return seed(h, a);
}

}  // extern "C"
template <class T>
static int init_field_host(m3lb_solver* h, const T* rho, const T* ux, const T* uy, const T* uz) {
  if (!h || !rho || !ux || !uy || !uz) return fail(M3LB_ERR_INVALID, "init_field: null argument");
  DeviceGuard dg(h->device);
  int rc = ensure_staging(h);
  if (rc) return rc;
  const size_t n = (size_t)h->n_interior();
  const size_t rb = real_bytes(h->storage);
  const T* src[4] = {rho, ux, uy, uz};
  char* dst = static_cast<char*>(h->staging);
  if (sizeof(T) == rb) {
    for (int i = 0; i < 4; ++i)
      CUDA_TRY(cudaMemcpyAsync(dst + i * n * rb, src[i], n * rb, cudaMemcpyHostToDevice, h->stream));
  } else {
    // convert on the host to the arithmetic type
    std::vector<char> tmp(n * rb);
    for (int i = 0; i < 4; ++i) {
      if (rb == 4) for (size_t k = 0; k < n; ++k) reinterpret_cast<float*>(tmp.data())[k] = (float)src[i][k];
      else for (size_t k = 0; k < n; ++k) reinterpret_cast<double*>(tmp.data())[k] = (double)src[i][k];
      CUDA_TRY(cudaMemcpyAsync(dst + i * n * rb, tmp.data(), n * rb, cudaMemcpyHostToDevice, h->stream));
      CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
  }
  return m3lb_init_field_device(h, dst, dst + n * rb, dst + 2 * n * rb, dst + 3 * n * rb);
}

extern "C" {
int m3lb_init_field_f32(m3lb_solver* h, const float* rho, const float* ux, const float* uy,
                        const float* uz) {
  return init_field_host(h, rho, ux, uy, uz);
}
int m3lb_init_field_f64(m3lb_solver* h, const double* rho, const double* ux, const double* uy,
                        const double* uz) {
  return init_field_host(h, rho, ux, uy, uz);
}

int m3lb_step(m3lb_solver* h, int nsteps, int store_macro) {
  if (!h) return fail(M3LB_ERR_INVALID, "step: null handle");
  if (nsteps < 0) return fail(M3LB_ERR_INVALID, "step: negative step count");
  DeviceGuard dg(h->device);
  const int kernel = h->step_kernel();
  for (int s = 0; s < nsteps; ++s) {
    StepArgs a = h->args();
    if (store_macro && s == nsteps - 1) {
      a.rho = h->macro[0]; a.ux = h->macro[1]; a.uy = h->macro[2]; a.uz = h->macro[3];
    }
    int n = 0;
    int rc = bound_before(h, a, &n);
    if (rc) return rc;
    CUDA_TRY(h->L->step(a, h->op, h->eq, h->shifted != 0, h->forcing != 0, kernel, h->stream, &n));
    rc = bound_after(h, a, &n);
    if (rc) return rc;
    h->launches += n;
    ++h->t;
  }
  return M3LB_OK;
}

int m3lb_macro_device(m3lb_solver* h, void** rho, void** ux, void** uy, void** uz) {
  if (!h) return fail(M3LB_ERR_INVALID, "macro: null handle");
  DeviceGuard dg(h->device);
  StepArgs a = h->args();
  a.flags = h->flags;  // non-fluid nodes report zeros
  a.rho = h->macro[0]; a.ux = h->macro[1]; a.uy = h->macro[2]; a.uz = h->macro[3];
  CUDA_TRY(h->L->macro(a, h->op, h->shifted != 0, h->forcing != 0, h->stream));
  h->launches += 1;
  if (h->walls.count) {  // the state RegWall nodes report
    CUDA_TRY(h->L->bound(a, h->walls.args(0, h->walls.count), kBndMacro, h->op, h->eq,
                         h->shifted != 0, h->forcing != 0, h->stream));
    h->launches += 1;
  }
  if (rho) *rho = h->macro[0];
  if (ux) *ux = h->macro[1];
  if (uy) *uy = h->macro[2];
  if (uz) *uz = h->macro[3];
  return M3LB_OK;
}

}  // extern "C"
template <class T>
static int copy_macro(m3lb_solver* h, T* out[4]) {
  const size_t n = (size_t)h->n_interior();
  const size_t rb = real_bytes(h->storage);
  if (sizeof(T) == rb) {
    for (int i = 0; i < 4; ++i)
      if (out[i]) CUDA_TRY(cudaMemcpyAsync(out[i], h->macro[i], n * rb, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return M3LB_OK;
  }
  std::vector<char> tmp(n * rb);
  for (int i = 0; i < 4; ++i) {
    if (!out[i]) continue;
    CUDA_TRY(cudaMemcpyAsync(tmp.data(), h->macro[i], n * rb, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (size_t k = 0; k < n; ++k)
      out[i][k] = rb == 4 ? (T) reinterpret_cast<float*>(tmp.data())[k]
                          : (T) reinterpret_cast<double*>(tmp.data())[k];
  }
  return M3LB_OK;
}

extern "C" {
int m3lb_macro_f32(m3lb_solver* h, float* rho, float* ux, float* uy, float* uz) {
  int rc = m3lb_macro_device(h, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  float* o[4] = {rho, ux, uy, uz};
  DeviceGuard dg(h->device);
  return copy_macro(h, o);
}
int m3lb_macro_f64(m3lb_solver* h, double* rho, double* ux, double* uy, double* uz) {
  int rc = m3lb_macro_device(h, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  double* o[4] = {rho, ux, uy, uz};
  DeviceGuard dg(h->device);
  return copy_macro(h, o);
}
int m3lb_stored_macro_f64(m3lb_solver* h, double* rho, double* ux, double* uy, double* uz) {
  if (!h) return fail(M3LB_ERR_INVALID, "stored_macro: null handle");
  double* o[4] = {rho, ux, uy, uz};
  DeviceGuard dg(h->device);
  return copy_macro(h, o);
}

int m3lb_reduce(m3lb_solver* h, double out[6]) {
  if (!h || !out) return fail(M3LB_ERR_INVALID, "reduce: null argument");
  DeviceGuard dg(h->device);
  StepArgs a = h->args();
  CUDA_TRY(h->L->reduce(a, h->op, h->shifted != 0, h->forcing != 0, h->partials, h->nblocks,
                        h->red_out, h->stream));
  h->launches += 2;
  CUDA_TRY(cudaMemcpyAsync(out, h->red_out, kReduceVals * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}

int m3lb_diagnostics(m3lb_solver* h, double out[3]) {
  if (!h || !out) return fail(M3LB_ERR_INVALID, "diagnostics: null argument");
  int rc = m3lb_macro_device(h, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  DeviceGuard dg(h->device);
  const Geo& g = h->g;
  // one partial of three values per block fits the reduction scratch
  // (nblocks partials of kReduceVals = 6)
  const int nb = h->nblocks;
  if (h->storage == M3LB_STORE_F64)
    diag_kernel<double><<<nb, kDiagThreads, 0, h->stream>>>(
        static_cast<const double*>(h->macro[1]), static_cast<const double*>(h->macro[2]),
        static_cast<const double*>(h->macro[3]), g.nx, g.ny, g.nz, h->partials);
  else
    diag_kernel<float><<<nb, kDiagThreads, 0, h->stream>>>(
        static_cast<const float*>(h->macro[1]), static_cast<const float*>(h->macro[2]),
        static_cast<const float*>(h->macro[3]), g.nx, g.ny, g.nz, h->partials);
  CUDA_TRY(cudaGetLastError());
  diag_finish<<<1, 32, 0, h->stream>>>(h->partials, nb, h->red_out);
  CUDA_TRY(cudaGetLastError());
  h->launches += 2;
  CUDA_TRY(cudaMemcpyAsync(out, h->red_out, kDiagVals * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}

static int gather_impl(m3lb_solver* h, double* out, void* raw) {
  DeviceGuard dg(h->device);
  const size_t n = (size_t)h->g.n_padded * h->Q;
  const size_t b = n * (out ? sizeof(double) : (size_t)elem_bytes(h->storage));
  void* d = nullptr;
  if (cudaMalloc(&d, b) != cudaSuccess) return fail(M3LB_ERR_MEMORY, "gather: cannot allocate %zu bytes", b);
  cudaError_t e = h->L->gather(h->g, h->f, (int)(h->t & 1), out ? (double*)d : nullptr,
                               out ? nullptr : d, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out ? (void*)out : raw, d, b, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(M3LB_ERR_CUDA, "gather: %s", cudaGetErrorString(e));
  h->launches += 1;
  return M3LB_OK;
}
int m3lb_gather(m3lb_solver* h, double* out) {
  if (!h || !out) return fail(M3LB_ERR_INVALID, "gather: null argument");
  return gather_impl(h, out, nullptr);
}
int m3lb_gather_raw(m3lb_solver* h, void* out) {
  if (!h || !out) return fail(M3LB_ERR_INVALID, "gather: null argument");
  return gather_impl(h, nullptr, out);
}

static int scatter_impl(m3lb_solver* h, const double* in, const void* raw) {
  DeviceGuard dg(h->device);
  const size_t n = (size_t)h->g.n_padded * h->Q;
  const size_t b = n * (in ? sizeof(double) : (size_t)elem_bytes(h->storage));
  void* d = nullptr;
  if (cudaMalloc(&d, b) != cudaSuccess) return fail(M3LB_ERR_MEMORY, "scatter: cannot allocate %zu bytes", b);
  cudaError_t e = cudaMemcpyAsync(d, in ? (const void*)in : raw, b, cudaMemcpyHostToDevice, h->stream);
  int rc = M3LB_OK;
  if (e == cudaSuccess) {
    SeedArgs a{};
    a.mode = 2;
    a.pops = in ? (const double*)d : nullptr;
    a.raw = in ? nullptr : d;
    rc = seed(h, a);
  }
  if (e == cudaSuccess && rc == M3LB_OK) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(M3LB_ERR_CUDA, "scatter: %s", cudaGetErrorString(e));
  return rc;
}
int m3lb_scatter(m3lb_solver* h, const double* in) {
  if (!h || !in) return fail(M3LB_ERR_INVALID, "scatter: null argument");
  return scatter_impl(h, in, nullptr);
}
int m3lb_scatter_raw(m3lb_solver* h, const void* in) {
  if (!h || !in) return fail(M3LB_ERR_INVALID, "scatter: null argument");
  return scatter_impl(h, nullptr, in);
}

int m3lb_timestep(const m3lb_solver* h, long long* t) {
  if (!h || !t) return fail(M3LB_ERR_INVALID, "timestep: null argument");
  *t = h->t;
  return M3LB_OK;
}
int m3lb_dims(const m3lb_solver* h, int d[12]) {
  if (!h || !d) return fail(M3LB_ERR_INVALID, "dims: null argument");
  const Geo& g = h->g;
  const int v[12] = {g.nx, g.ny, g.nz, g.hx, g.hy, g.hz, g.sx, g.sy, g.sz, g.nch, h->Q, h->storage};
  std::memcpy(d, v, sizeof v);
  return M3LB_OK;
}
int m3lb_populations(const m3lb_solver* h, void** ptr, size_t* bytes) {
  if (!h) return fail(M3LB_ERR_INVALID, "populations: null handle");
  if (ptr) *ptr = h->f;
  if (bytes) *bytes = h->f_bytes;
  return M3LB_OK;
}
int m3lb_set_stream(m3lb_solver* h, void* stream) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_stream: null handle");
  DeviceGuard dg(h->device);
  // the handle's own stream stays alive until the handle is destroyed: other
  // work may have been ordered after it (m3lb_stream_order)
  if (h->stream) cudaStreamSynchronize(h->stream);
  h->stream = static_cast<cudaStream_t>(stream);
  return M3LB_OK;
}
int m3lb_sync(m3lb_solver* h) {
  if (!h) return fail(M3LB_ERR_INVALID, "sync: null handle");
  DeviceGuard dg(h->device);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  // a kernel whose bounded wait expired leaves a status in the word and
  // returns; report it once
  int st = 0;
  CUDA_TRY(cudaMemcpy(&st, h->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (st != 0) {
    CUDA_TRY(cudaMemset(h->err, 0, sizeof(int)));
    return fail(M3LB_ERR_CUDA, "sync: a step kernel gave up waiting for its copies (status %d); "
                "the populations of that step are not valid", st);
  }
  return M3LB_OK;
}
int m3lb_set_option(m3lb_solver* h, int option, int value) {
  if (!h) return fail(M3LB_ERR_INVALID, "set_option: null handle");
  if (option == M3LB_OPT_NODE_KERNEL) {
    h->node_kernel = value != 0;
    return M3LB_OK;
  }
  if (option == M3LB_OPT_KERNEL) {
    if (value < M3LB_KERNEL_AUTO || value > M3LB_KERNEL_ROWS)
      return fail(M3LB_ERR_INVALID, "set_option: bad kernel %d", value);
    h->kernel = value;
    return M3LB_OK;
  }
  if (option == M3LB_OPT_WAIT_CYCLES) {
    if (value < 0) return fail(M3LB_ERR_INVALID, "set_option: negative wait %d", value);
    h->wait_cycles = value;
    return M3LB_OK;
  }
  return fail(M3LB_ERR_INVALID, "set_option: unknown option %d", option);
}
int m3lb_launch_count(const m3lb_solver* h, long long* n) {
  if (!h || !n) return fail(M3LB_ERR_INVALID, "launch_count: null argument");
  *n = h->launches;
  return M3LB_OK;
}

}  // extern "C"
