// Launcher tables: one per (lattice, storage format), each built by one
// compilation of lbm_inst.cu, so the kernel instantiations compile in
// parallel.  Host-only interface between the C ABI and the kernels.
#pragma once
#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace m3lb {

// Step kernels: one node per thread (any geometry), and, for a periodic x
// axis with even nx, the paired kernel (one warp per 64-node chunk) or its
// persistent, copy-pipelined form.
// The row kernel moves whole rows with the tensor-memory accelerator
// (16-bit storage; the row widths it takes are in lbm_capi.cu).
enum StepKernel { kKernelNodes = 1, kKernelPairs = 2, kKernelStream = 3, kKernelRows = 4 };

struct Launchers {
  // one step with the given StepKernel
  cudaError_t (*step)(const StepArgs& a, int op, int eq, bool sh, bool force, int kernel,
                      cudaStream_t s, int* launches);
  cudaError_t (*seed)(const SeedArgs& a, int op, int eq, bool sh, cudaStream_t s);
  cudaError_t (*gather)(const Geo& g, const void* f, int parity, double* out, void* raw,
                        cudaStream_t s);
  cudaError_t (*macro)(const StepArgs& a, int op, bool sh, bool force, cudaStream_t s);
  cudaError_t (*reduce)(const StepArgs& a, int op, bool sh, bool force, double* partials,
                        int nblocks, double* out, cudaStream_t s);
  // boundary pass over the wall-node list b.begin..b.end (lbm_bound.cuh)
  cudaError_t (*bound)(const StepArgs& a, const BoundArgs& b, int phase, int op, int eq, bool sh,
                       bool force, cudaStream_t s);
  // the row kernel's tensor maps of a lattice (RowMaps of lbm_rows.cuh,
  // `bytes` long), for the items of batched row launches
  cudaError_t (*row_maps)(const StepArgs& a, void* maps, size_t bytes);
  // one time step of a batch of lattices through the row kernel: `items` a
  // device table of RowItem, `desc` the device RowBatch of this launch (all
  // its lattices with operator op, shifted, no force, rows of nch chunks)
  cudaError_t (*batch_rows)(const void* items, const void* desc, int op, int nch, int step,
                            cudaStream_t s);
};
// phases of the boundary pass
enum BoundPhase { kBndSnapshot = 0, kBndCornerRho = 1, kBndUpdate = 2, kBndMacro = 3 };

#define M3LB_DECLARE_LAUNCHERS(NAME) const Launchers* NAME();
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F32)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F16)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_BF16)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F64)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F16C)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F32)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F16)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_BF16)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F64)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F16C)
#undef M3LB_DECLARE_LAUNCHERS

}  // namespace m3lb
