// Kernel instantiations and launchers for one (lattice, storage format),
// selected at compile time:
//   -DM3LB_LAT=D2Q9|D3Q27 -DM3LB_ST=kF32|kF16|kBF16|kF64|kF16C -DM3LB_NAME=launchers_<...>
#include "lbm_kernels.cuh"
#include <cudaTypedefs.h>

#include "lbm_stream.cuh"
#include "lbm_rows.cuh"
#include "lbm_bound.cuh"
#include "lbm_launch.h"

#ifndef M3LB_LAT
#error "M3LB_LAT not defined"
#endif

namespace m3lb {
namespace {

using L = M3LB_LAT;
constexpr int ST = M3LB_ST;
// 16-bit storage exists only as shifted populations.
constexpr bool kRawOK = (ST == kF32 || ST == kF64);

inline unsigned blocks_for(long long n, int threads) {
  return (unsigned)((n + threads - 1) / threads);
}

// Persistent grid of the streamed kernel: the resident blocks of every SM
// (occupancy queried once per device), never more warps than chunks.
template <int OP, int EQ, bool SH, bool FORCE, bool FULL>
cudaError_t launch_stream_t(const StepArgs& a, cudaStream_t s) {
  using Cfg = StreamCfg<L, ST>;
  auto kern = step_stream<L, ST, OP, EQ, SH, FORCE, FULL>;
  constexpr int kMaxDev = 64;
  static int cached[kMaxDev];  // resident blocks per SM x SMs, 0 = not yet known
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
  if (cached[dev] == 0) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
    if (e != cudaSuccess) return e;
    int per_sm = 0, nsm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPairThreads, Cfg::SMEM);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    cached[dev] = per_sm * nsm;
  }
  const Geo& g = a.g;
  const long long units = (long long)g.ny * g.nz * g.nch;
  const long long need = (units + Cfg::WARPS - 1) / Cfg::WARPS;
  const unsigned grid = (unsigned)(need < cached[dev] ? need : cached[dev]);
  kern<<<grid, kPairThreads, Cfg::SMEM, s>>>(a);
  return cudaGetLastError();
}
// Every chunk full (nx a multiple of 64) and at least two chunks per row:
// the lane layout of the chunk edges is fixed at compile time.
template <int OP, int EQ, bool SH, bool FORCE>
cudaError_t launch_stream(const StepArgs& a, cudaStream_t s) {
  if ((a.g.nx % kChunk) == 0 && a.g.nch >= 2) return launch_stream_t<OP, EQ, SH, FORCE, true>(a, s);
  return launch_stream_t<OP, EQ, SH, FORCE, false>(a, s);
}

// The 3-D tensor maps of the population array for the row kernel: x (64
// elements of a chunk), direction (Q), chunk (sz * sy * nch); one map per
// copy shape of the row plan, box (64, span, nch) with traversal stride s
// along the direction axis (span = (count - 1) * s + 1).
cudaError_t rows_maps(const StepArgs& a, RowMaps<L>* maps) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  using E = typename WordOps<ST>::E;
  using Pl = RowPlan<L>;
  constexpr int EB = (int)sizeof(E);
  const Geo& g = a.g;
  const CUtensorMapDataType dt = EB == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16
                                 : EB == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                           : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const cuuint64_t dims[3] = {(cuuint64_t)kChunk, (cuuint64_t)L::Q,
                              (cuuint64_t)g.sz * g.sy * g.nch};
  const cuuint64_t strides[2] = {(cuuint64_t)kChunk * EB, (cuuint64_t)L::Q * kChunk * EB};
  for (int m = 0; m < Pl::NMAPS; ++m) {
    const int span = (Pl::map_count[m] - 1) * Pl::map_stride[m] + 1;
    const cuuint32_t box[3] = {(cuuint32_t)kChunk, (cuuint32_t)span, (cuuint32_t)g.nch};
    const cuuint32_t estr[3] = {1u, (cuuint32_t)Pl::map_stride[m], 1u};
    const CUresult r = encode(&maps->m[m], dt, 3, a.f, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  }
  return cudaSuccess;
}

// Persistent row kernel: one CTA of nch update warps per row (and, for rows
// of 3 chunks or more, one copy warp), stages of LW chunks (the smallest of
// 2, 3, 4, 8 that holds the row), as many CTAs as are resident (occupancy
// queried once per device and shape).
template <int OP, int EQ, bool SH, bool FORCE, int LW>
cudaError_t launch_rows_lw(const StepArgs& a, cudaStream_t s) {
  constexpr bool CW = LW != 2;
  using Cfg = RowsCfg<L, ST, LW, rows_stages<CW>()>;
  if constexpr (Cfg::SMEM > kRowsSmemMax) {
    return cudaErrorInvalidValue;
  } else {
    const Geo& g = a.g;
    auto kern = step_rows<L, ST, OP, EQ, SH, FORCE, LW, CW>;
    const int threads = (g.nch + (CW ? 1 : 0)) * 32;
    constexpr int kMaxDev = 64;
    static int cached[kMaxDev][LW + 1];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    if (cached[dev][g.nch] == 0) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
      if (e != cudaSuccess) return e;
      int per_sm = 0, nsm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, Cfg::SMEM);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      if (per_sm < 1) return cudaErrorInvalidConfiguration;
      cached[dev][g.nch] = per_sm * nsm;
    }
    RowMaps<L> maps;
    e = rows_maps(a, &maps);
    if (e != cudaSuccess) return e;
    const long long rows = (long long)g.ny * g.nz;
    const unsigned grid = (unsigned)(rows < cached[dev][g.nch] ? rows : cached[dev][g.nch]);
    kern<<<grid, threads, Cfg::SMEM, s>>>(a, maps);
    return cudaGetLastError();
  }
}
template <int OP, int EQ, bool SH, bool FORCE>
cudaError_t launch_rows(const StepArgs& a, cudaStream_t s) {
  const Geo& g = a.g;
  if (g.nch < 1 || g.nch > kRowsMaxChunks || (g.nx % 2) != 0) return cudaErrorInvalidValue;
  switch (rows_lw(g.nch)) {
    case 2: return launch_rows_lw<OP, EQ, SH, FORCE, 2>(a, s);
    case 3: return launch_rows_lw<OP, EQ, SH, FORCE, 3>(a, s);
    case 4: return launch_rows_lw<OP, EQ, SH, FORCE, 4>(a, s);
    default:
      // 8-chunk stages hold 16-bit rows only (FP32 fits one CTA per SM,
      // FP64 none)
      if constexpr (sizeof(typename WordOps<ST>::E) == 2) return launch_rows_lw<OP, EQ, SH, FORCE, 8>(a, s);
      else return cudaErrorInvalidValue;
  }
}

template <int OP, int EQ, bool SH, bool FORCE>
cudaError_t step_t(const StepArgs& a, int kernel, cudaStream_t s) {
  const Geo& g = a.g;
  if (kernel == kKernelRows) return launch_rows<OP, EQ, SH, FORCE>(a, s);
  if (kernel == kKernelStream) return launch_stream<OP, EQ, SH, FORCE>(a, s);
  if (kernel == kKernelPairs) {
    // one warp per 64-node chunk of every interior row
    const long long nthreads = (long long)g.ny * g.nz * g.nch * 32;
    step_pairs<L, ST, OP, EQ, SH, FORCE><<<blocks_for(nthreads, kPairThreads), kPairThreads, 0, s>>>(a);
  } else {
    step_nodes<L, ST, OP, EQ, SH, FORCE>
        <<<node_grid(g.nx, (long long)g.ny * g.nz, kNodeThreads), kNodeThreads, 0, s>>>(a);
  }
  return cudaGetLastError();
}

template <int OP, int EQ, bool SH>
cudaError_t step_f(const StepArgs& a, bool force, int kernel, cudaStream_t s) {
  return force ? step_t<OP, EQ, SH, true>(a, kernel, s) : step_t<OP, EQ, SH, false>(a, kernel, s);
}
template <int OP, int EQ>
cudaError_t step_s(const StepArgs& a, bool sh, bool force, int kernel, cudaStream_t s) {
  if (sh) return step_f<OP, EQ, true>(a, force, kernel, s);
  if constexpr (kRawOK) return step_f<OP, EQ, false>(a, force, kernel, s);
  return cudaErrorInvalidValue;
}

cudaError_t step(const StepArgs& a, int op, int eq, bool sh, bool force, int kernel,
                 cudaStream_t s, int* launches) {
  if (launches) *launches += 1;
  switch (op) {
    case 0: return step_t<0, 0, true, false>(a, kernel, s);
    case 1: return eq ? step_s<1, 1>(a, sh, force, kernel, s) : step_s<1, 0>(a, sh, force, kernel, s);
    case 2: return eq ? step_s<2, 1>(a, sh, force, kernel, s) : step_s<2, 0>(a, sh, force, kernel, s);
    case 3: return step_s<3, 0>(a, sh, force, kernel, s);
    case 4: return step_s<4, 0>(a, sh, force, kernel, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int OP, int EQ, bool SH>
cudaError_t seed_t(const SeedArgs& a, cudaStream_t s) {
  seed_kernel<L, ST, OP, EQ, SH><<<node_grid(a.g.sx, (long long)a.g.sy * a.g.sz, 128), 128, 0, s>>>(a);
  return cudaGetLastError();
}
template <int OP, int EQ>
cudaError_t seed_s(const SeedArgs& a, bool sh, cudaStream_t s) {
  if (sh) return seed_t<OP, EQ, true>(a, s);
  if constexpr (kRawOK) return seed_t<OP, EQ, false>(a, s);
  return cudaErrorInvalidValue;
}
cudaError_t seed(const SeedArgs& a, int op, int eq, bool sh, cudaStream_t s) {
  switch (op) {
    case 0: return seed_t<0, 0, true>(a, s);
    case 1:
    case 2: return eq ? seed_s<1, 1>(a, sh, s) : seed_s<1, 0>(a, sh, s);
    case 3:
    case 4: return seed_s<3, 0>(a, sh, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t gather(const Geo& g, const void* f, int parity, double* out, void* raw,
                   cudaStream_t s) {
  gather_kernel<L, ST><<<node_grid(g.sx, (long long)g.sy * g.sz, 128), 128, 0, s>>>(g, f, parity, out, raw);
  return cudaGetLastError();
}

// Macroscopic readout depends on the operator only through "none" vs the
// rest: every collision shares BGK's moment sums (BGK.hpp:63-78).
template <bool SH, bool FORCE>
cudaError_t macro_t(const StepArgs& a, int op, cudaStream_t s) {
  const dim3 grid = node_grid(a.g.nx, (long long)a.g.ny * a.g.nz, 128);
  if (op == 0)
    macro_kernel<L, ST, 0, true, false><<<grid, 128, 0, s>>>(a);
  else
    macro_kernel<L, ST, 1, SH, FORCE><<<grid, 128, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t macro(const StepArgs& a, int op, bool sh, bool force, cudaStream_t s) {
  if (sh) return force ? macro_t<true, true>(a, op, s) : macro_t<true, false>(a, op, s);
  if constexpr (kRawOK) return force ? macro_t<false, true>(a, op, s) : macro_t<false, false>(a, op, s);
  return cudaErrorInvalidValue;
}

template <bool SH, bool FORCE>
cudaError_t reduce_t(const StepArgs& a, int op, double* partials, int nb, double* out,
                     cudaStream_t s) {
  if (op == 0)
    reduce_kernel<L, ST, 0, true, false><<<nb, kReduceThreads, 0, s>>>(a, partials);
  else
    reduce_kernel<L, ST, 1, SH, FORCE><<<nb, kReduceThreads, 0, s>>>(a, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  reduce_finish<<<1, 32, 0, s>>>(partials, nb, out);
  return cudaGetLastError();
}
cudaError_t reduce(const StepArgs& a, int op, bool sh, bool force, double* partials, int nb,
                   double* out, cudaStream_t s) {
  if (sh) return force ? reduce_t<true, true>(a, op, partials, nb, out, s)
                       : reduce_t<true, false>(a, op, partials, nb, out, s);
  if constexpr (kRawOK)
    return force ? reduce_t<false, true>(a, op, partials, nb, out, s)
                 : reduce_t<false, false>(a, op, partials, nb, out, s);
  return cudaErrorInvalidValue;
}

template <int OP, int EQ, bool SH, bool FORCE>
cudaError_t bound_t(const StepArgs& a, const BoundArgs& b, int phase, cudaStream_t s) {
  using R = typename StoreT<ST>::real;
  constexpr bool USH = SH && OP != 0;
  const long long n = b.end - b.begin;
  if (n <= 0) return cudaSuccess;
  const unsigned grid = blocks_for(n, kBndThreads);
  switch (phase) {
    case kBndSnapshot: bnd_snapshot<L, ST><<<grid, kBndThreads, 0, s>>>(a, b); break;
    case kBndCornerRho: {
      bnd_wall_rho<L, ST, USH><<<grid, kBndThreads, 0, s>>>(a, b);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      bnd_corner_rho<R><<<grid, kBndThreads, 0, s>>>(b);
      break;
    }
    case kBndUpdate: bnd_step<L, ST, OP, EQ, SH, FORCE><<<grid, kBndThreads, 0, s>>>(a, b); break;
    case kBndMacro: bnd_macro<L, ST, USH><<<grid, kBndThreads, 0, s>>>(a, b); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}
template <int OP, int EQ, bool SH>
cudaError_t bound_f(const StepArgs& a, const BoundArgs& b, int phase, bool force, cudaStream_t s) {
  return force ? bound_t<OP, EQ, SH, true>(a, b, phase, s) : bound_t<OP, EQ, SH, false>(a, b, phase, s);
}
template <int OP, int EQ>
cudaError_t bound_s(const StepArgs& a, const BoundArgs& b, int phase, bool sh, bool force,
                    cudaStream_t s) {
  if (sh) return bound_f<OP, EQ, true>(a, b, phase, force, s);
  if constexpr (kRawOK) return bound_f<OP, EQ, false>(a, b, phase, force, s);
  return cudaErrorInvalidValue;
}
cudaError_t bound(const StepArgs& a, const BoundArgs& b, int phase, int op, int eq, bool sh,
                  bool force, cudaStream_t s) {
  switch (op) {
    case 0: return bound_t<0, 0, true, false>(a, b, phase, s);
    case 1: return eq ? bound_s<1, 1>(a, b, phase, sh, force, s) : bound_s<1, 0>(a, b, phase, sh, force, s);
    case 2: return eq ? bound_s<2, 1>(a, b, phase, sh, force, s) : bound_s<2, 0>(a, b, phase, sh, force, s);
    case 3: return bound_s<3, 0>(a, b, phase, sh, force, s);
    case 4: return bound_s<4, 0>(a, b, phase, sh, force, s);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t row_maps(const StepArgs& a, void* maps, size_t bytes) {
  if (bytes != sizeof(RowMaps<L>)) return cudaErrorInvalidValue;
  return rows_maps(a, static_cast<RowMaps<L>*>(maps));
}

// Batched row launches (the serving loop): 16-bit storage, shifted
// populations, no force.  A persistent grid of the resident CTAs of the
// shape, which does not depend on the batch's size, so the launch can be
// captured once and serve any resident set of its (operator, row width).
template <int OP, int LW>
cudaError_t launch_batch_rows(const void* items, const void* desc, int nch, int step,
                              cudaStream_t s) {
  constexpr bool CW = LW != 2;
  using Cfg = RowsCfg<L, ST, LW, rows_stages<CW>()>;
  if constexpr (Cfg::SMEM > kRowsSmemMax || sizeof(typename WordOps<ST>::E) != 2) {
    return cudaErrorNotSupported;
  } else {
    auto kern = batch_rows<L, ST, OP, 0, LW>;
    const int threads = (nch + (CW ? 1 : 0)) * 32;
    constexpr int kMaxDev = 64;
    static int cached[kMaxDev][LW + 1];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDev) return cudaErrorInvalidDevice;
    if (cached[dev][nch] == 0) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
      if (e != cudaSuccess) return e;
      int per_sm = 0, nsm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, Cfg::SMEM);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      if (per_sm < 1) return cudaErrorInvalidConfiguration;
      cached[dev][nch] = per_sm * nsm;
    }
    kern<<<cached[dev][nch], threads, Cfg::SMEM, s>>>(static_cast<const RowItem<L>*>(items),
                                                      static_cast<const RowBatch*>(desc), step);
    return cudaGetLastError();
  }
}
template <int OP>
cudaError_t batch_rows_op(const void* items, const void* desc, int nch, int step, cudaStream_t s) {
  if (nch < 1 || nch > kRowsMaxChunks) return cudaErrorInvalidValue;
  switch (rows_lw(nch)) {
    case 2: return launch_batch_rows<OP, 2>(items, desc, nch, step, s);
    case 3: return launch_batch_rows<OP, 3>(items, desc, nch, step, s);
    case 4: return launch_batch_rows<OP, 4>(items, desc, nch, step, s);
    default: return launch_batch_rows<OP, 8>(items, desc, nch, step, s);
  }
}
cudaError_t batch_rows_launch(const void* items, const void* desc, int op, int nch, int step,
                              cudaStream_t s) {
  if constexpr (sizeof(typename WordOps<ST>::E) != 2 || L::Q != 27) {
    return cudaErrorNotSupported;
  } else {
    switch (op) {
      case 1: return batch_rows_op<1>(items, desc, nch, step, s);
      case 2: return batch_rows_op<2>(items, desc, nch, step, s);
      case 3: return batch_rows_op<3>(items, desc, nch, step, s);
      case 4: return batch_rows_op<4>(items, desc, nch, step, s);
      default: return cudaErrorInvalidValue;
    }
  }
}

const Launchers kTable = {step, seed, gather, macro, reduce, bound, row_maps, batch_rows_launch};

}  // namespace

const Launchers* M3LB_NAME() { return &kTable; }

}  // namespace m3lb
