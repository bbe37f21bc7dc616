// Launcher tables: one per (lattice, storage format), each built by one
// compilation of lbm_inst.cu, so the kernel instantiations compile in
// parallel.  Host-only interface between the C ABI and the kernels.
#pragma once
#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace m3lb {

struct Launchers {
  // one step; pairs selects the paired kernel (periodic x, even nx)
  cudaError_t (*step)(const StepArgs& a, int op, int eq, bool sh, bool force, bool pairs,
                      cudaStream_t s, int* launches);
  cudaError_t (*seed)(const SeedArgs& a, int op, int eq, bool sh, cudaStream_t s);
  cudaError_t (*gather)(const Geo& g, const void* f, int parity, double* out, void* raw,
                        cudaStream_t s);
  cudaError_t (*macro)(const StepArgs& a, int op, bool sh, bool force, cudaStream_t s);
  cudaError_t (*reduce)(const StepArgs& a, int op, bool sh, bool force, double* partials,
                        int nblocks, double* out, cudaStream_t s);
};

#define M3LB_DECLARE_LAUNCHERS(NAME) const Launchers* NAME();
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F32)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F16)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_BF16)
M3LB_DECLARE_LAUNCHERS(launchers_D2Q9_F64)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F32)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F16)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_BF16)
M3LB_DECLARE_LAUNCHERS(launchers_D3Q27_F64)
#undef M3LB_DECLARE_LAUNCHERS

}  // namespace m3lb
