// The scalar (advection-diffusion) lattice: D2Q5 / D3Q7 (and, with ScalarBGK,
// D2Q9 / D3Q27) on Esoteric Pull,
// the reference's ScalarSolver (src/solver/ScalarSolver.hpp) with ScalarBGK,
// ScalarTRT and ScalarRegularised (src/collision/Scalar*.hpp), its cell types
// (adiabatic, Dirichlet, on-node moment, outflow, specular) and the thermal
// coupling to a fluid handle: the fluid's stored velocity advects the scalar,
// the scalar's field drives the fluid's Boussinesq force.
//
// Same storage layout as the fluid (x-chunked, lbm_common.cuh) with Q = 5, 7,
// 9 or 27; one thread per node, x fastest, so each direction's loads and stores of
// a warp are contiguous.  FP32 or FP64 storage; arithmetic in the same type.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/m3lb.h"
#include "lbm_host.h"
#include "lbm_kernels.cuh"

namespace m3lb {
namespace {

constexpr int kScalarThreads = 128;
enum : uint8_t { kSBulk = 0, kSAdiabatic = 1, kSDirichlet = 2, kSExcluded = 3, kSMoment = 4,
                 kSOutflow = 5, kSSpecular = 6 };

struct ScalarArgs {
  Geo g;
  void* f;                  // populations
  const uint8_t* cells;     // ScalarCell per padded node
  const uint8_t* spec;      // specular face mask per padded node, or nullptr
  const uint32_t* unk;      // moment-wall unknown directions per padded node, or nullptr
  const void* wall;         // wall values per interior node (arithmetic type)
  void* field;              // the scalar per interior node
  const void* omega_of;     // per-node rate per interior node, or nullptr
  const void* ux;           // advecting velocity per interior node, or nullptr
  const void* uy;
  const void* uz;
  int parity;
  double omega, T_ref, Lambda;
};

__device__ __forceinline__ void coords_of(const Geo& g, long long k, int& x, int& y, int& z) {
  x = (int)(k % g.nx) + g.hx;
  y = (int)((k / g.nx) % g.ny) + g.hy;
  z = (int)(k / ((long long)g.nx * g.ny)) + g.hz;
}
// The per-node kernels run a 3-D grid: blockIdx.x the x segment of a row,
// blockIdx.y and blockIdx.z the row's y and z, so a node's coordinates need
// no division (ny and nz are at most 65535, checked at creation).
__device__ __forceinline__ bool row_node(const Geo& g, long long& k, int& x, int& y, int& z) {
  const int xi = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (xi >= g.nx) return false;
  const int yi = (int)blockIdx.y, zi = (int)blockIdx.z;
  k = ((long long)zi * g.ny + yi) * g.nx + xi;
  x = xi + g.hx; y = yi + g.hy; z = zi + g.hz;
  return true;
}
inline dim3 row_grid(const Geo& g, int threads) {
  return dim3((unsigned)((g.nx + threads - 1) / threads), (unsigned)g.ny, (unsigned)g.nz);
}

// ScalarBGK::eq (ScalarBGK.hpp:43-49): w_i (dT + (T_ref + dT) c_i.u / cs2).
template <class L, int I, class R>
__device__ __forceinline__ R s_eq(R T_ref, R dT, R ux, R uy, R uz) {
  constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
  const R cu = R(cx) * ux + R(cy) * uy + R(cz) * uz;
  return R(weight<L, I>()) * (dT + (T_ref + dT) * R(L::CS2D) * cu);
}

template <class L, class R>
__device__ __forceinline__ R deviation(const R* h) {
  R t = 0;
#pragma unroll
  for (int i = 0; i < L::Q; ++i) t += h[i];
  return t;
}

// The three operators: BGK (ScalarBGK.hpp:51-58), TRT with the magic
// parameter Lambda (ScalarTRT.hpp:30-52), regularised (ScalarRegularised.hpp:33-46).
template <class L, int OP, class R>
__device__ __forceinline__ void s_collide(R* h, R dT, R ux, R uy, R uz, R w, R T_ref, R Lambda) {
  if constexpr (OP == 1) {
    static_for<0, L::Q>([&](auto I) {
      constexpr int i = decltype(I)::value;
      h[i] += w * (s_eq<L, i>(T_ref, dT, ux, uy, uz) - h[i]);
    });
  } else {
    const R cs2v = R(1) / R(L::CS2D);
    const R T = T_ref + dT;
    const R u[3] = {ux, uy, uz};
    const R d = cs2v * dT;
    if constexpr (OP == 2) {
      const R tm = R(1) / w - R(0.5);
      const R wp = tm > R(0) ? R(1) / (Lambda / tm + R(0.5)) : R(0);
      R msum = 0;
#pragma unroll
      for (int a = 0; a < L::D; ++a) {
        const R j = h[2 * a + 1] - h[2 * a + 2];
        const R m = h[2 * a + 1] + h[2 * a + 2];
        const R p = j + w * (T * u[a] - j);
        const R gg = m + wp * (d - m);
        h[2 * a + 1] = R(0.5) * (gg + p);
        h[2 * a + 2] = R(0.5) * (gg - p);
        msum += gg;
      }
      h[0] = dT - msum;
    } else {
#pragma unroll
      for (int a = 0; a < L::D; ++a) {
        const R j = h[2 * a + 1] - h[2 * a + 2];
        const R p = j + w * (T * u[a] - j);
        h[2 * a + 1] = R(0.5) * (d + p);
        h[2 * a + 2] = R(0.5) * (d - p);
      }
      h[0] = dT - R(L::D) * d;
    }
  }
}

// impose_moment (src/boundary/MomentDirichlet.hpp): the unknown directions
// share the deficit target - sum(known) in proportion to their weights.
template <class L, class R>
__device__ __forceinline__ void impose_moment(R* g, R target, uint32_t unknown) {
  R known = 0, wsum = 0;
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if (unknown & (1u << i)) wsum += R(weight<L, i>());
    else known += g[i];
  });
  if (!(wsum > R(0))) return;
  const R deficit = target - known;
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if (unknown & (1u << i)) g[i] = deficit * R(weight<L, i>()) / wsum;
  });
}

template <class R>
__device__ __forceinline__ void velocity_at(const ScalarArgs& a, long long k, R& vx, R& vy, R& vz) {
  vx = a.ux ? reinterpret_cast<const R*>(a.ux)[k] : R(0);
  vy = a.uy ? reinterpret_cast<const R*>(a.uy)[k] : R(0);
  vz = a.uz ? reinterpret_cast<const R*>(a.uz)[k] : R(0);
}

// run_step<P> (ScalarSolver.hpp:302-372): one thread per interior node.
// Every load a bulk node needs is issued before the cell type is examined
// (each address is inside the lattice whatever the type), so a thread waits
// for memory once.
template <class L, int ST, int OP>
__global__ void __launch_bounds__(kScalarThreads) scalar_step(ScalarArgs a) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const Geo& g = a.g;
  long long k;
  int x, y, z;
  if (!row_node(g, k, x, y, z)) return;
  const long long pn = ((long long)z * g.sy + y) * g.sx + x;
  const uint8_t cell = a.cells[pn];
  const AxisSteps<Q> st = axis_steps<Q>(g, x, y, z);
  E* own = reinterpret_cast<E*>(a.f) + slot<Q>(g, x, y, z, 0);
  const int P = a.parity;
  // direction i (odd) sits at slot i + P of the node, i + 1 at slot i + 1 - P
  // of the neighbour along c_i
  E* up = own + P * kChunk;
  E* dn = own + (1 - P) * kChunk;
  R h[Q];
  h[0] = to_real(own[0]);
  static_for<1, Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    h[i] = to_real(up[i * kChunk]);
    h[i + 1] = to_real(dn[nb_offset<L, i>(st) + i * kChunk]);
  });
  R vx, vy, vz;
  velocity_at(a, k, vx, vy, vz);
  const R w = a.omega_of ? reinterpret_cast<const R*>(a.omega_of)[k] : R(a.omega);
  // excluded: not simulated; outflow: second pass; adiabatic: bounce-back,
  // the identity on this storage
  if (cell == kSExcluded || cell == kSOutflow || cell == kSAdiabatic) return;
  const R T_ref = R(a.T_ref);
  R* field = reinterpret_cast<R*>(a.field);
  if (cell == kSDirichlet) {  // anti-bounce-back toward the wall value
    const R Tw = reinterpret_cast<const R*>(a.wall)[k] - T_ref;
    R o[Q];
    static_for<0, Q>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int opp = i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1);
      o[i] = -h[opp] + R(2) * R(weight<L, i>()) * Tw;
    });
#pragma unroll
    for (int i = 0; i < Q; ++i) h[i] = o[i];
  } else {
    if (cell == kSMoment)
      impose_moment<L>(h, reinterpret_cast<const R*>(a.wall)[k] - T_ref, a.unk ? a.unk[pn] : 0u);
    else if (cell == kSSpecular && a.spec)
      spec_node_mirror<L>(h, a.spec[pn]);
    const R dT = deviation<L>(h);
    s_collide<L, OP>(h, dT, vx, vy, vz, w, T_ref, R(a.Lambda));
    field[k] = T_ref + dT;
  }
  own[0] = from_real<E>(h[0]);
  static_for<1, Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    dn[nb_offset<L, i>(st) + i * kChunk] = from_real<E>(h[i]);
    up[i * kChunk] = from_real<E>(h[i + 1]);
  });
}

// outflow_kernel<P> (:393-419): equilibrium at the donor's value and the
// node's own velocity, after the main pass has written the donor's field.
template <class L, int ST>
__global__ void __launch_bounds__(kScalarThreads)
scalar_outflow(ScalarArgs a, const long long* node_k, const long long* donor_k, int count) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const int j = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (j >= count) return;
  const Geo& g = a.g;
  const long long k = node_k[j];
  int x, y, z;
  coords_of(g, k, x, y, z);
  NodeNb<L> nb;
  node_neighbours<L>(g, x, y, z, nb);
  R* field = reinterpret_cast<R*>(a.field);
  const R T_ref = R(a.T_ref);
  const R dT = field[donor_k[j]] - T_ref;
  R vx, vy, vz;
  velocity_at(a, k, vx, vy, vz);
  R o[Q];
  static_for<0, Q>([&](auto I) { o[decltype(I)::value] = s_eq<L, decltype(I)::value>(T_ref, dT, vx, vy, vz); });
  E* A = reinterpret_cast<E*>(a.f);
  const int P = a.parity;
  A[slot<Q>(g, x, y, z, 0)] = from_real<E>(o[0]);
#pragma unroll
  for (int i = 1; i < Q; i += 2) {
    const int* m = nb.nb[i];
    A[slot<Q>(g, m[0], m[1], m[2], i + 1 - P)] = from_real<E>(o[i]);
    A[slot<Q>(g, x, y, z, i + P)] = from_real<E>(o[i + 1]);
  }
  field[k] = T_ref + dT;
}

// field_kernel<P> (:375-391): compute_field.
template <class L, int ST>
__global__ void __launch_bounds__(kScalarThreads) scalar_field(ScalarArgs a) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const Geo& g = a.g;
  long long k;
  int x, y, z;
  if (!row_node(g, k, x, y, z)) return;
  const long long pn = ((long long)z * g.sy + y) * g.sx + x;
  const uint8_t cell = a.cells[pn];
  R* field = reinterpret_cast<R*>(a.field);
  if (cell == kSExcluded || cell == kSAdiabatic) { field[k] = R(0); return; }
  if (cell == kSDirichlet || cell == kSMoment) { field[k] = reinterpret_cast<const R*>(a.wall)[k]; return; }
  if (cell == kSOutflow) return;
  NodeNb<L> nb;
  node_neighbours<L>(g, x, y, z, nb);
  const E* A = reinterpret_cast<const E*>(a.f);
  R h[Q];
#pragma unroll
  for (int i = 0; i < Q; ++i) h[i] = to_real(A[load_slot<L>(g, nb, a.parity, i)]);
  if (cell == kSSpecular && a.spec) spec_node_mirror<L>(h, a.spec[pn]);
  field[k] = R(a.T_ref) + deviation<L>(h);
}

// source_kernel<P> (:421-437): dC w_i added to every population of bulk and
// specular nodes.
template <class L, int ST>
__global__ void __launch_bounds__(kScalarThreads) scalar_source(ScalarArgs a, const void* dC) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  const Geo& g = a.g;
  long long k;
  int x, y, z;
  if (!row_node(g, k, x, y, z)) return;
  const uint8_t cell = a.cells[((long long)z * g.sy + y) * g.sx + x];
  if (cell != kSBulk && cell != kSSpecular) return;
  const R d = reinterpret_cast<const R*>(dC)[k];
  if (d == R(0)) return;
  NodeNb<L> nb;
  node_neighbours<L>(g, x, y, z, nb);
  E* A = reinterpret_cast<E*>(a.f);
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    const size_t s = load_slot<L>(g, nb, a.parity, i);
    A[s] = from_real<E>(to_real(A[s]) + R(weight<L, i>()) * d);
  });
}

// initialize_field (:175-190): equilibrium at rest at T per padded node (a
// Dirichlet node at its wall value), scattered at parity 0 with the
// reference's sequential last-writer rule on clamped edges.
template <class L, int ST>
__global__ void __launch_bounds__(kScalarThreads) scalar_init(ScalarArgs a, const void* Tpad) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  const Geo& g = a.g;
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.n_padded) return;
  const int x = (int)(n % g.sx), y = (int)((n / g.sx) % g.sy), z = (int)(n / ((long long)g.sx * g.sy));
  const bool inside = x >= g.hx && x < g.hx + g.nx && y >= g.hy && y < g.hy + g.ny &&
                      z >= g.hz && z < g.hz + g.nz;
  const long long k = inside ? ((long long)(z - g.hz) * g.ny + (y - g.hy)) * g.nx + (x - g.hx) : -1;
  const R T = (inside && a.cells[n] == kSDirichlet) ? reinterpret_cast<const R*>(a.wall)[k]
                                                     : reinterpret_cast<const R*>(Tpad)[n];
  if (inside) reinterpret_cast<R*>(a.field)[k] = T;
  const R dT = T - R(a.T_ref);
  NodeNb<L> nb;
  node_neighbours<L>(g, x, y, z, nb);
  E* A = reinterpret_cast<E*>(a.f);
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if constexpr (i > 0 && (i & 1) == 0) {
      constexpr int cx = L::cx[i - 1], cy = L::cy[i - 1], cz = L::cz[i - 1];
      const int* m = nb.nb[i - 1];
      if (!axis_winner(x, cx, m[0], g.px, g.sx) || !axis_winner(y, cy, m[1], g.py, g.sy) ||
          !axis_winner(z, cz, m[2], g.pz, g.sz))
        return;
    }
    A[load_slot<L>(g, nb, 0, i)] = from_real<E>(s_eq<L, i>(R(a.T_ref), dT, R(0), R(0), R(0)));
  });
}

// Sum of every stored population (total_population, :209-218) in FP64:
// per-block partials, then one block adds them in a fixed order.
template <class L, int ST>
__global__ void __launch_bounds__(kReduceThreads) scalar_total(ScalarArgs a, double* partials) {
  using E = typename StoreT<ST>::elem;
  __shared__ double sh[kReduceThreads / 32];
  const Geo& g = a.g;
  const E* A = reinterpret_cast<const E*>(a.f);
  const double acc = slot_sum_part<L::Q>(A, g, (long long)blockIdx.x * blockDim.x + threadIdx.x,
                                         (long long)gridDim.x * blockDim.x);
  const double s = block_sum(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}
__global__ void scalar_total_finish(const double* partials, int nb, double* out) {
  if (threadIdx.x < 32) warp_fixed_sums(partials, nb, 1, out);
}

// Logical populations per padded node as double (tests).
template <class L, int ST>
__global__ void __launch_bounds__(kScalarThreads) scalar_gather(ScalarArgs a, double* out) {
  using E = typename StoreT<ST>::elem;
  const Geo& g = a.g;
  const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.n_padded) return;
  const int x = (int)(n % g.sx), y = (int)((n / g.sx) % g.sy), z = (int)(n / ((long long)g.sx * g.sy));
  NodeNb<L> nb;
  node_neighbours<L>(g, x, y, z, nb);
  const E* A = reinterpret_cast<const E*>(a.f);
  for (int i = 0; i < L::Q; ++i) out[n * L::Q + i] = (double)to_real(A[load_slot<L>(g, nb, a.parity, i)]);
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Launchers per (lattice, storage); the operator is a runtime choice.
template <class L, int ST>
struct ScalarOps {
  static cudaError_t step(const ScalarArgs& a, int op, cudaStream_t s) {
    const dim3 b = row_grid(a.g, kScalarThreads);
    if (op == 1) {
      scalar_step<L, ST, 1><<<b, kScalarThreads, 0, s>>>(a);
    } else if constexpr (L::Q == 2 * L::D + 1) {  // TRT / regularised: axis-pair lattices
      if (op == 2) scalar_step<L, ST, 2><<<b, kScalarThreads, 0, s>>>(a);
      else scalar_step<L, ST, 3><<<b, kScalarThreads, 0, s>>>(a);
    } else {
      return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
  }
  static cudaError_t outflow(const ScalarArgs& a, const long long* nk, const long long* dk, int c,
                             cudaStream_t s) {
    scalar_outflow<L, ST><<<blocks(c, kScalarThreads), kScalarThreads, 0, s>>>(a, nk, dk, c);
    return cudaGetLastError();
  }
  static cudaError_t field(const ScalarArgs& a, cudaStream_t s) {
    scalar_field<L, ST><<<row_grid(a.g, kScalarThreads), kScalarThreads, 0, s>>>(a);
    return cudaGetLastError();
  }
  static cudaError_t source(const ScalarArgs& a, const void* dC, cudaStream_t s) {
    scalar_source<L, ST><<<row_grid(a.g, kScalarThreads), kScalarThreads, 0, s>>>(a, dC);
    return cudaGetLastError();
  }
  static cudaError_t init(const ScalarArgs& a, const void* Tpad, cudaStream_t s) {
    scalar_init<L, ST><<<blocks(a.g.n_padded, kScalarThreads), kScalarThreads, 0, s>>>(a, Tpad);
    return cudaGetLastError();
  }
  static cudaError_t total(const ScalarArgs& a, double* partials, int nb, double* out, cudaStream_t s) {
    scalar_total<L, ST><<<nb, kReduceThreads, 0, s>>>(a, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    scalar_total_finish<<<1, 32, 0, s>>>(partials, nb, out);
    return cudaGetLastError();
  }
  static cudaError_t gather(const ScalarArgs& a, double* out, cudaStream_t s) {
    scalar_gather<L, ST><<<blocks(a.g.n_padded, kScalarThreads), kScalarThreads, 0, s>>>(a, out);
    return cudaGetLastError();
  }
};

struct ScalarTable {
  cudaError_t (*step)(const ScalarArgs&, int, cudaStream_t);
  cudaError_t (*outflow)(const ScalarArgs&, const long long*, const long long*, int, cudaStream_t);
  cudaError_t (*field)(const ScalarArgs&, cudaStream_t);
  cudaError_t (*source)(const ScalarArgs&, const void*, cudaStream_t);
  cudaError_t (*init)(const ScalarArgs&, const void*, cudaStream_t);
  cudaError_t (*total)(const ScalarArgs&, double*, int, double*, cudaStream_t);
  cudaError_t (*gather)(const ScalarArgs&, double*, cudaStream_t);
};
template <class L, int ST>
const ScalarTable* table() {
  using O = ScalarOps<L, ST>;
  static const ScalarTable t = {O::step, O::outflow, O::field, O::source, O::init, O::total, O::gather};
  return &t;
}
const ScalarTable* scalar_table(int lattice, int storage) {
  const bool f64 = storage == M3LB_STORE_F64;
  switch (lattice) {
    case 5: return f64 ? table<D2Q5, kF64>() : table<D2Q5, kF32>();
    case 7: return f64 ? table<D3Q7, kF64>() : table<D3Q7, kF32>();
    case 9: return f64 ? table<D2Q9, kF64>() : table<D2Q9, kF32>();
    case 27: return f64 ? table<D3Q27, kF64>() : table<D3Q27, kF32>();
    default: return nullptr;
  }
}

int sfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}
#define S_TRY(call)                                                                  \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return sfail(M3LB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

}  // namespace
}  // namespace m3lb

using namespace m3lb;

struct m3lb_scalar {
  int lattice = 7, Q = 7, op = 1, storage = M3LB_STORE_F32;
  Geo g{};
  int device = 0;
  cudaStream_t stream = nullptr;  // where the work is queued
  cudaStream_t own = nullptr;     // the stream the handle created
  double omega = 1, T_ref = 0, Lambda = 0.25;
  long long t = 0, launches = 0;
  void* f = nullptr;
  uint8_t* cells = nullptr;
  uint8_t* spec = nullptr;
  uint32_t* unk = nullptr;
  void* wall = nullptr;
  void* field = nullptr;
  void* omega_of = nullptr;
  const void* ux = nullptr;
  const void* uy = nullptr;
  const void* uz = nullptr;
  void* u_own = nullptr;          // m3lb_scalar_set_velocity_host's copy (3 arrays)
  void* src = nullptr;            // m3lb_scalar_add_source's array on the device
  std::vector<double> src_host;   // ... and what it holds
  void* scratch = nullptr;        // host-array uploads and the source array
  size_t scratch_bytes = 0;
  double* partials = nullptr;     // total: per-block sums, then the result
  int nblocks = 0;
  long long* out_nodes = nullptr; // outflow list: node and donor interior indices
  long long* out_donor = nullptr;
  int n_out = 0;
  std::vector<uint8_t> cells_host;   // per padded node
  std::vector<uint8_t> spec_host;    // per padded node
  const ScalarTable* T = nullptr;

  size_t rb() const { return storage == M3LB_STORE_F64 ? 8 : 4; }
  long long nint() const { return (long long)g.nx * g.ny * g.nz; }
  ScalarArgs args() const {
    ScalarArgs a{};
    a.g = g; a.f = f; a.cells = cells; a.spec = spec; a.unk = unk; a.wall = wall; a.field = field;
    a.omega_of = omega_of; a.ux = ux; a.uy = uy; a.uz = uz;
    a.parity = (int)(t & 1);
    a.omega = omega; a.T_ref = T_ref; a.Lambda = Lambda;
    return a;
  }
  long long pidx(int x, int y, int z) const {
    return ((long long)(z + g.hz) * g.sy + (y + g.hy)) * g.sx + (x + g.hx);
  }
};

namespace {
struct SGuard {
  int prev = -1;
  explicit SGuard(int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev) { prev = cur; cudaSetDevice(dev); }
  }
  ~SGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// Copy n values of the caller's doubles into the scratch array as the
// arithmetic type; returns the device pointer.
int upload_real(m3lb_scalar* h, const double* src, size_t n, void** dst) {
  const size_t b = n * h->rb();
  if (b > h->scratch_bytes) {
    cudaFree(h->scratch);
    h->scratch = nullptr;
    h->scratch_bytes = 0;
    if (cudaMalloc(&h->scratch, b) != cudaSuccess)
      return sfail(M3LB_ERR_MEMORY, "scalar: cannot allocate %zu bytes of staging", b);
    h->scratch_bytes = b;
  }
  std::vector<char> tmp(b);
  if (h->rb() == 8) std::memcpy(tmp.data(), src, b);
  else for (size_t i = 0; i < n; ++i) reinterpret_cast<float*>(tmp.data())[i] = (float)src[i];
  S_TRY(cudaMemcpyAsync(h->scratch, tmp.data(), b, cudaMemcpyHostToDevice, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  *dst = h->scratch;
  return M3LB_OK;
}
int ensure(void** p, size_t bytes) {
  if (*p) return M3LB_OK;
  if (cudaMalloc(p, bytes) != cudaSuccess) return sfail(M3LB_ERR_MEMORY, "scalar: cannot allocate %zu bytes", bytes);
  if (cudaMemset(*p, 0, bytes) != cudaSuccess) return sfail(M3LB_ERR_CUDA, "scalar: memset failed");
  return M3LB_OK;
}
int upload_cells(m3lb_scalar* h) {
  S_TRY(cudaMemcpyAsync(h->cells, h->cells_host.data(), h->cells_host.size(), cudaMemcpyHostToDevice,
                        h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}
}  // namespace

extern "C" {

int m3lb_scalar_create(int lattice, int nx, int ny, int nz, int px, int py, int pz, int op,
                       int storage, m3lb_scalar** out) {
  if (!out) return sfail(M3LB_ERR_INVALID, "scalar_create: null output handle");
  *out = nullptr;
  if (lattice != 5 && lattice != 7 && lattice != 9 && lattice != 27)
    return sfail(M3LB_ERR_INVALID, "scalar_create: lattice must be 5, 7, 9 or 27");
  if ((lattice == 5 || lattice == 9) && nz != 1)
    return sfail(M3LB_ERR_INVALID, "scalar_create: a 2-D lattice needs nz == 1");
  if ((lattice == 9 || lattice == 27) && op != M3LB_SOP_BGK)
    return sfail(M3LB_ERR_INVALID, "scalar_create: ScalarTRT and ScalarRegularised need D2Q5 or D3Q7");
  if (nx < 1 || ny < 1 || nz < 1) return sfail(M3LB_ERR_INVALID, "scalar_create: extents must be >= 1");
  if (ny > 65535 || nz > 65535)
    return sfail(M3LB_ERR_INVALID, "scalar_create: ny and nz must be at most 65535");
  if (op < M3LB_SOP_BGK || op > M3LB_SOP_REGULARISED)
    return sfail(M3LB_ERR_INVALID, "scalar_create: bad operator %d", op);
  if (storage != M3LB_STORE_F32 && storage != M3LB_STORE_F64)
    return sfail(M3LB_ERR_UNSUPPORTED, "scalar_create: the scalar is stored in FP32 or FP64");
  if ((long long)(nx + 2) * (ny + 2) * (nz + 2) > (1LL << 31))
    return sfail(M3LB_ERR_INVALID, "scalar_create: lattice exceeds 2^31 nodes");
  auto* h = new m3lb_scalar();
  h->lattice = lattice; h->Q = lattice; h->op = op; h->storage = storage;
  h->g = make_geo(nx, ny, nz, px, py, pz);
  h->T = scalar_table(lattice, storage);
  cudaGetDevice(&h->device);
  auto cleanup = [&](int code) { m3lb_scalar_destroy(h); return code; };
  const Geo& g = h->g;
  const size_t fb = pop_elems(g, h->Q) * h->rb();
  if (cudaMalloc(&h->f, fb) != cudaSuccess || cudaMalloc((void**)&h->cells, (size_t)g.n_padded) != cudaSuccess ||
      cudaMalloc(&h->field, (size_t)h->nint() * h->rb()) != cudaSuccess ||
      cudaMalloc(&h->wall, (size_t)h->nint() * h->rb()) != cudaSuccess)
    return cleanup(sfail(M3LB_ERR_MEMORY, "scalar_create: cannot allocate the lattice"));
  h->nblocks = reduce_blocks(g);
  if (cudaMalloc((void**)&h->partials, ((size_t)h->nblocks + 1) * 8) != cudaSuccess)
    return cleanup(sfail(M3LB_ERR_MEMORY, "scalar_create: cannot allocate reduction scratch"));
  if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(sfail(M3LB_ERR_CUDA, "scalar_create: cannot create stream"));
  h->stream = h->own;
  // interior nodes bulk, halo excluded (ScalarSolver.hpp:81-86)
  h->cells_host.assign((size_t)g.n_padded, kSExcluded);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) h->cells_host[h->pidx(x, y, z)] = kSBulk;
  if (cudaMemsetAsync(h->f, 0, fb, h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->field, 0, (size_t)h->nint() * h->rb(), h->stream) != cudaSuccess ||
      cudaMemsetAsync(h->wall, 0, (size_t)h->nint() * h->rb(), h->stream) != cudaSuccess)
    return cleanup(sfail(M3LB_ERR_CUDA, "scalar_create: initial copies failed"));
  int rc = upload_cells(h);
  if (rc) return cleanup(rc);
  *out = h;
  return M3LB_OK;
}

int m3lb_scalar_destroy(m3lb_scalar* h) {
  if (!h) return M3LB_OK;
  SGuard dg(h->device);
  // the queue may be another handle's stream, possibly gone already: wait
  // for the whole device rather than for that stream
  cudaDeviceSynchronize();
  for (void* p : {h->f, (void*)h->cells, (void*)h->spec, (void*)h->unk, h->wall, h->field, h->omega_of,
                  h->u_own, h->src, h->scratch, (void*)h->partials, (void*)h->out_nodes, (void*)h->out_donor})
    cudaFree(p);
  if (h->own) cudaStreamDestroy(h->own);
  delete h;
  return M3LB_OK;
}

int m3lb_scalar_set_params(m3lb_scalar* h, double omega, double T_ref, double Lambda) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_set_params: null handle");
  h->omega = omega; h->T_ref = T_ref; h->Lambda = Lambda;
  return M3LB_OK;
}

int m3lb_scalar_set_stream(m3lb_scalar* h, void* stream) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_set_stream: null handle");
  SGuard dg(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  // as m3lb_set_stream: NULL is the default stream; the handle's own stream
  // lives until the handle does, as callers may still order work after it
  h->stream = (cudaStream_t)stream;
  return M3LB_OK;
}

int m3lb_scalar_set_cells(m3lb_scalar* h, const uint8_t* cells) {
  if (!h || !cells) return sfail(M3LB_ERR_INVALID, "scalar_set_cells: null argument");
  const Geo& g = h->g;
  for (long long k = 0; k < h->nint(); ++k)
    if (cells[k] > kSSpecular) return sfail(M3LB_ERR_INVALID, "scalar_set_cells: cell type %u is not 0..6", cells[k]);
  SGuard dg(h->device);
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) h->cells_host[h->pidx(x, y, z)] = cells[((size_t)z * g.ny + y) * g.nx + x];
  return upload_cells(h);
}

int m3lb_scalar_set_wall_values(m3lb_scalar* h, const double* tw) {
  if (!h || !tw) return sfail(M3LB_ERR_INVALID, "scalar_set_wall_values: null argument");
  SGuard dg(h->device);
  void* d = nullptr;
  int rc = upload_real(h, tw, (size_t)h->nint(), &d);
  if (rc) return rc;
  S_TRY(cudaMemcpyAsync(h->wall, d, (size_t)h->nint() * h->rb(), cudaMemcpyDeviceToDevice, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}

static int set_spec(m3lb_scalar* h, const uint8_t* m, bool codes) {
  const Geo& g = h->g;
  for (long long k = 0; k < h->nint(); ++k) {
    const unsigned v = m[k];
    if (codes && v > 6)
      return sfail(M3LB_ERR_INVALID, "scalar_set_specular_walls: code %u is not an axis normal", v);
    if (!codes && v > 0x3F)
      return sfail(M3LB_ERR_INVALID, "scalar_set_specular_nodes: mask %u has bits outside the six faces", v);
    if (!codes)
      for (int a = 0; a < 3; ++a)
        if ((v & (1u << (2 * a))) && (v & (1u << (2 * a + 1))))
          return sfail(M3LB_ERR_INVALID, "scalar_set_specular_nodes: mask %u carries both faces of axis %d", v, a);
  }
  if (h->spec_host.empty()) h->spec_host.assign((size_t)g.n_padded, 0);
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const uint8_t v = m[((size_t)z * g.ny + y) * g.nx + x];
        if (v) h->spec_host[h->pidx(x, y, z)] = codes ? (uint8_t)(1u << (v - 1)) : v;  // faces_of_normal
      }
  SGuard dg(h->device);
  int rc = ensure((void**)&h->spec, (size_t)g.n_padded);
  if (rc) return rc;
  S_TRY(cudaMemcpyAsync(h->spec, h->spec_host.data(), h->spec_host.size(), cudaMemcpyHostToDevice, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}
int m3lb_scalar_set_specular_walls(m3lb_scalar* h, const uint8_t* codes) {
  if (!h || !codes) return sfail(M3LB_ERR_INVALID, "scalar_set_specular_walls: null argument");
  return set_spec(h, codes, true);
}
int m3lb_scalar_set_specular_nodes(m3lb_scalar* h, const uint8_t* masks) {
  if (!h || !masks) return sfail(M3LB_ERR_INVALID, "scalar_set_specular_nodes: null argument");
  return set_spec(h, masks, false);
}

int m3lb_scalar_set_omega_field(m3lb_scalar* h, const double* omega) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_set_omega_field: null handle");
  SGuard dg(h->device);
  if (!omega) {
    cudaFree(h->omega_of);
    h->omega_of = nullptr;
    return M3LB_OK;
  }
  int rc = ensure(&h->omega_of, (size_t)h->nint() * h->rb());
  if (rc) return rc;
  void* d = nullptr;
  rc = upload_real(h, omega, (size_t)h->nint(), &d);
  if (rc) return rc;
  S_TRY(cudaMemcpyAsync(h->omega_of, d, (size_t)h->nint() * h->rb(), cudaMemcpyDeviceToDevice, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}

int m3lb_scalar_set_velocity_device(m3lb_scalar* h, const void* ux, const void* uy, const void* uz) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_set_velocity: null handle");
  if ((ux == nullptr) != (uy == nullptr) || (ux == nullptr) != (uz == nullptr))
    return sfail(M3LB_ERR_INVALID, "scalar_set_velocity: give all three components or none");
  h->ux = ux; h->uy = uy; h->uz = uz;
  return M3LB_OK;
}

int m3lb_scalar_set_velocity_host(m3lb_scalar* h, const double* ux, const double* uy,
                                  const double* uz) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_set_velocity: null handle");
  if (!ux || !uy || !uz) return m3lb_scalar_set_velocity_device(h, nullptr, nullptr, nullptr);
  SGuard dg(h->device);
  const size_t n = (size_t)h->nint(), rb = h->rb();
  int rc = ensure(&h->u_own, 3 * n * rb);
  if (rc) return rc;
  std::vector<char> tmp(3 * n * rb);
  const double* src[3] = {ux, uy, uz};
  for (int c = 0; c < 3; ++c)
    for (size_t i = 0; i < n; ++i) {
      if (rb == 8) reinterpret_cast<double*>(tmp.data())[c * n + i] = src[c][i];
      else reinterpret_cast<float*>(tmp.data())[c * n + i] = (float)src[c][i];
    }
  S_TRY(cudaMemcpyAsync(h->u_own, tmp.data(), tmp.size(), cudaMemcpyHostToDevice, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  char* b = static_cast<char*>(h->u_own);
  return m3lb_scalar_set_velocity_device(h, b, b + n * rb, b + 2 * n * rb);
}

int m3lb_scalar_get_stream(const m3lb_scalar* h, void** stream) {
  if (!h || !stream) return sfail(M3LB_ERR_INVALID, "scalar_get_stream: null argument");
  *stream = (void*)h->stream;
  return M3LB_OK;
}

int m3lb_scalar_finalize_geometry(m3lb_scalar* h) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_finalize_geometry: null handle");
  const Geo& g = h->g;
  const int nn[3] = {g.nx, g.ny, g.nz};
  const int per[3] = {g.px, g.py, g.pz};
  const int* cv[3];
  int Q = h->Q;
  switch (Q) {
    case 5: cv[0] = D2Q5::cx; cv[1] = D2Q5::cy; cv[2] = D2Q5::cz; break;
    case 7: cv[0] = D3Q7::cx; cv[1] = D3Q7::cy; cv[2] = D3Q7::cz; break;
    case 9: cv[0] = D2Q9::cx; cv[1] = D2Q9::cy; cv[2] = D2Q9::cz; break;
    default: cv[0] = D3Q27::cx; cv[1] = D3Q27::cy; cv[2] = D3Q27::cz; break;
  }
  // unknown directions of moment nodes (MomentDirichlet.hpp unknown_mask)
  std::vector<uint32_t> unk;
  bool any_moment = false;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        const long long n = h->pidx(x, y, z);
        if (h->cells_host[n] != kSMoment) continue;
        if (!any_moment) { unk.assign((size_t)g.n_padded, 0); any_moment = true; }
        uint32_t m = 0;
        for (int i = 0; i < Q; ++i) {
          int src[3] = {x - cv[0][i], y - cv[1][i], z - cv[2][i]};
          bool outside = false;
          for (int a = 0; a < 3; ++a) {
            if (per[a]) src[a] = (src[a] + nn[a]) % nn[a];
            else if (src[a] < 0 || src[a] >= nn[a]) outside = true;
          }
          if (!outside && h->cells_host[h->pidx(src[0], src[1], src[2])] == kSExcluded) outside = true;
          if (outside) m |= 1u << i;
        }
        unk[n] = m;
      }
  // outflow donors (build_donors, :240-296)
  auto flag_at = [&](int x, int y, int z) -> uint8_t {
    int q[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
      if (per[a]) { if (q[a] < 0) q[a] += nn[a]; else if (q[a] >= nn[a]) q[a] -= nn[a]; }
      if (q[a] < 0 || q[a] >= nn[a]) return kSExcluded;
    }
    return h->cells_host[h->pidx(q[0], q[1], q[2])];
  };
  // the reference takes the donor's index without wrapping; keep it only when
  // it names a node of the lattice's interior
  auto kidx = [&](int x, int y, int z) -> long long {
    if (x < 0 || y < 0 || z < 0 || x >= g.nx || y >= g.ny || z >= g.nz) return -1;
    return ((long long)z * g.ny + y) * g.nx + x;
  };
  static const int d6[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  std::vector<long long> onode, odonor;
  int degenerate = 0, nout = 0;
  for (int z = 0; z < g.nz; ++z)
    for (int y = 0; y < g.ny; ++y)
      for (int x = 0; x < g.nx; ++x) {
        if (h->cells_host[h->pidx(x, y, z)] != kSOutflow) continue;
        ++nout;
        int ix = 0, iy = 0, iz = 0;
        for (int k = 0; k < 6; ++k)
          if (flag_at(x + d6[k][0], y + d6[k][1], z + d6[k][2]) == kSExcluded) {
            ix -= d6[k][0]; iy -= d6[k][1]; iz -= d6[k][2];
          }
        long long best = -1;
        if ((ix || iy || iz) && flag_at(x + ix, y + iy, z + iz) == kSBulk) best = kidx(x + ix, y + iy, z + iz);
        if (best < 0)
          for (int k = 0; k < 6; ++k)
            if (flag_at(x + d6[k][0], y + d6[k][1], z + d6[k][2]) == kSBulk) {
              best = kidx(x + d6[k][0], y + d6[k][1], z + d6[k][2]);
              if (best >= 0) break;
            }
        if (best < 0) { ++degenerate; continue; }
        onode.push_back(kidx(x, y, z));
        odonor.push_back(best);
      }
  if (degenerate)
    std::printf("  [scalar] %d of %d outflow node(s) have no bulk neighbour and are inert\n", degenerate, nout);
  SGuard dg(h->device);
  if (any_moment) {
    int rc = ensure((void**)&h->unk, (size_t)g.n_padded * 4);
    if (rc) return rc;
    S_TRY(cudaMemcpyAsync(h->unk, unk.data(), unk.size() * 4, cudaMemcpyHostToDevice, h->stream));
  }
  cudaFree(h->out_nodes); cudaFree(h->out_donor);
  h->out_nodes = h->out_donor = nullptr;
  h->n_out = (int)onode.size();
  if (h->n_out) {
    if (cudaMalloc((void**)&h->out_nodes, onode.size() * 8) != cudaSuccess ||
        cudaMalloc((void**)&h->out_donor, odonor.size() * 8) != cudaSuccess)
      return sfail(M3LB_ERR_MEMORY, "scalar_finalize_geometry: cannot allocate the outflow list");
    S_TRY(cudaMemcpyAsync(h->out_nodes, onode.data(), onode.size() * 8, cudaMemcpyHostToDevice, h->stream));
    S_TRY(cudaMemcpyAsync(h->out_donor, odonor.data(), odonor.size() * 8, cudaMemcpyHostToDevice, h->stream));
  }
  S_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}

int m3lb_scalar_init_field(m3lb_scalar* h, const double* T_padded) {
  if (!h || !T_padded) return sfail(M3LB_ERR_INVALID, "scalar_init_field: null argument");
  SGuard dg(h->device);
  void* d = nullptr;
  int rc = upload_real(h, T_padded, (size_t)h->g.n_padded, &d);
  if (rc) return rc;
  h->t = 0;
  S_TRY(h->T->init(h->args(), d, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  h->launches += 1;
  return M3LB_OK;
}
int m3lb_scalar_init(m3lb_scalar* h, double T0) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_init: null handle");
  std::vector<double> T((size_t)h->g.n_padded, T0);
  return m3lb_scalar_init_field(h, T.data());
}

int m3lb_scalar_step(m3lb_scalar* h, int nsteps) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_step: null handle");
  if (nsteps < 0) return sfail(M3LB_ERR_INVALID, "scalar_step: negative step count");
  SGuard dg(h->device);
  for (int s = 0; s < nsteps; ++s) {
    const ScalarArgs a = h->args();
    S_TRY(h->T->step(a, h->op, h->stream));
    h->launches += 1;
    if (h->n_out) {
      S_TRY(h->T->outflow(a, h->out_nodes, h->out_donor, h->n_out, h->stream));
      h->launches += 1;
    }
    ++h->t;
  }
  return M3LB_OK;
}

int m3lb_scalar_add_source(m3lb_scalar* h, const double* dC) {
  if (!h || !dC) return sfail(M3LB_ERR_INVALID, "scalar_add_source: null argument");
  SGuard dg(h->device);
  const size_t n = (size_t)h->nint();
  // a source repeated step after step is copied to the device once
  if (!h->src || h->src_host.size() != n || std::memcmp(h->src_host.data(), dC, n * 8) != 0) {
    int rc = ensure(&h->src, n * h->rb());
    if (rc) return rc;
    void* d = nullptr;
    rc = upload_real(h, dC, n, &d);
    if (rc) return rc;
    S_TRY(cudaMemcpyAsync(h->src, d, n * h->rb(), cudaMemcpyDeviceToDevice, h->stream));
    h->src_host.assign(dC, dC + n);
  }
  S_TRY(h->T->source(h->args(), h->src, h->stream));
  h->launches += 1;
  return M3LB_OK;
}
int m3lb_scalar_add_source_device(m3lb_scalar* h, const void* dC) {
  if (!h || !dC) return sfail(M3LB_ERR_INVALID, "scalar_add_source: null argument");
  SGuard dg(h->device);
  S_TRY(h->T->source(h->args(), dC, h->stream));
  h->launches += 1;
  return M3LB_OK;
}

int m3lb_scalar_compute_field(m3lb_scalar* h) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_compute_field: null handle");
  SGuard dg(h->device);
  S_TRY(h->T->field(h->args(), h->stream));
  h->launches += 1;
  return M3LB_OK;
}

int m3lb_scalar_field(m3lb_scalar* h, double* T) {
  if (!h || !T) return sfail(M3LB_ERR_INVALID, "scalar_field: null argument");
  SGuard dg(h->device);
  const size_t n = (size_t)h->nint();
  std::vector<char> tmp(n * h->rb());
  S_TRY(cudaMemcpyAsync(tmp.data(), h->field, tmp.size(), cudaMemcpyDeviceToHost, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  for (size_t i = 0; i < n; ++i)
    T[i] = h->rb() == 8 ? reinterpret_cast<double*>(tmp.data())[i] : (double)reinterpret_cast<float*>(tmp.data())[i];
  return M3LB_OK;
}
int m3lb_scalar_field_device(m3lb_scalar* h, void** T) {
  if (!h || !T) return sfail(M3LB_ERR_INVALID, "scalar_field_device: null argument");
  *T = h->field;
  return M3LB_OK;
}

int m3lb_scalar_total(m3lb_scalar* h, double* out) {
  if (!h || !out) return sfail(M3LB_ERR_INVALID, "scalar_total: null argument");
  SGuard dg(h->device);
  S_TRY(h->T->total(h->args(), h->partials, h->nblocks, h->partials + h->nblocks, h->stream));
  S_TRY(cudaMemcpyAsync(out, h->partials + h->nblocks, 8, cudaMemcpyDeviceToHost, h->stream));
  S_TRY(cudaStreamSynchronize(h->stream));
  h->launches += 2;
  return M3LB_OK;
}

int m3lb_scalar_gather(m3lb_scalar* h, double* out) {
  if (!h || !out) return sfail(M3LB_ERR_INVALID, "scalar_gather: null argument");
  SGuard dg(h->device);
  const size_t b = (size_t)h->g.n_padded * h->Q * 8;
  double* d = nullptr;
  if (cudaMalloc((void**)&d, b) != cudaSuccess) return sfail(M3LB_ERR_MEMORY, "scalar_gather: cannot allocate");
  cudaError_t e = h->T->gather(h->args(), d, h->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, b, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return sfail(M3LB_ERR_CUDA, "scalar_gather: %s", cudaGetErrorString(e));
  return M3LB_OK;
}

int m3lb_scalar_info(const m3lb_scalar* h, long long* n_padded, long long* timestep, long long* launches) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_info: null handle");
  if (n_padded) *n_padded = h->g.n_padded;
  if (timestep) *timestep = h->t;
  if (launches) *launches = h->launches;
  return M3LB_OK;
}

int m3lb_couple_thermal(m3lb_solver* fluid, m3lb_scalar* th, double gx, double gy, double gz,
                        double rho0, double beta, double T0) {
  if (!fluid || !th) return sfail(M3LB_ERR_INVALID, "couple_thermal: null handle");
  int d[12];
  int rc = m3lb_dims(fluid, d);
  if (rc) return rc;
  if (d[0] != th->g.nx || d[1] != th->g.ny || d[2] != th->g.nz)
    return sfail(M3LB_ERR_INVALID, "couple_thermal: the lattices differ in extent");
  if ((size_t)real_bytes(d[11]) != th->rb())
    return sfail(M3LB_ERR_INVALID, "couple_thermal: the fluid computes in %s, the scalar in %s",
                 real_bytes(d[11]) == 8 ? "FP64" : "FP32", th->rb() == 8 ? "FP64" : "FP32");
  void *ux = nullptr, *uy = nullptr, *uz = nullptr, *stream = nullptr;
  if ((rc = m3lb_macro_pointers(fluid, nullptr, &ux, &uy, &uz)) != M3LB_OK) return rc;
  if ((rc = m3lb_get_stream(fluid, &stream)) != M3LB_OK) return rc;
  if ((rc = m3lb_set_buoyancy(fluid, th->field, gx, gy, gz, rho0, beta, T0)) != M3LB_OK) return rc;
  if ((rc = m3lb_scalar_set_stream(th, stream)) != M3LB_OK) return rc;
  return m3lb_scalar_set_velocity_device(th, ux, uy, uz);
}

int m3lb_scalar_sync(m3lb_scalar* h) {
  if (!h) return sfail(M3LB_ERR_INVALID, "scalar_sync: null handle");
  SGuard dg(h->device);
  S_TRY(cudaStreamSynchronize(h->stream));
  return M3LB_OK;
}

}  // extern "C"
