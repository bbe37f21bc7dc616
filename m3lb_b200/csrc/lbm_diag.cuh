// Flow diagnostics of the validation campaign on the device: the
// volume-integrated kinetic energy and enstrophy of validation/Campaign.hpp
// (diagnostics(), :99-130), from the macroscopic velocity of every interior
// node.  energy = sum 0.5 |u|^2, enstrophy = sum 0.5 |w|^2 with the vorticity w
// from central differences whose neighbours wrap around the interior on every
// axis ((x + n) % n, as the reference writes it); 2-D lattices (nz = 1) keep
// only w_z.  A node with a non-finite velocity component adds nothing and is
// counted.  Sums in FP64, one partial per block, added in a fixed order by
// one warp (deterministic, no atomics).
#pragma once
#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace m3lb {

constexpr int kDiagThreads = 256;
constexpr int kDiagVals = 3;  // energy, enstrophy, non-finite nodes

__device__ __forceinline__ double diag_block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
  return r;
}

template <class R>
__global__ void __launch_bounds__(kDiagThreads)
diag_kernel(const R* __restrict__ ux, const R* __restrict__ uy, const R* __restrict__ uz, int nx,
            int ny, int nz, double* partials) {
  __shared__ double sh[kDiagThreads / 32];
  const long long n = (long long)nx * ny * nz;
  const long long nxy = (long long)nx * ny;
  double e = 0, w = 0, bad = 0;
  auto at = [&](int x, int y, int z) {
    x = x < 0 ? x + nx : (x >= nx ? x - nx : x);
    y = y < 0 ? y + ny : (y >= ny ? y - ny : y);
    z = z < 0 ? z + nz : (z >= nz ? z - nz : z);
    return ((long long)z * ny + y) * nx + x;
  };
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(k % nx), y = (int)((k / nx) % ny), z = (int)(k / nxy);
    const double a = (double)ux[k], b = (double)uy[k], c = (double)uz[k];
    if (!isfinite(a) || !isfinite(b) || !isfinite(c)) {
      bad += 1;
      continue;
    }
    e = __dadd_rn(e, __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)),
                                               __dmul_rn(c, c))));
    auto dif = [&](const R* u, long long p, long long m) {
      return __dmul_rn(0.5, __dadd_rn((double)u[p], -(double)u[m]));
    };
    const double wz = __dadd_rn(dif(uy, at(x + 1, y, z), at(x - 1, y, z)),
                                -dif(ux, at(x, y + 1, z), at(x, y - 1, z)));
    double wx = 0, wy = 0;
    if (nz > 1) {
      wx = __dadd_rn(dif(uz, at(x, y + 1, z), at(x, y - 1, z)), -dif(uy, at(x, y, z + 1), at(x, y, z - 1)));
      wy = __dadd_rn(dif(ux, at(x, y, z + 1), at(x, y, z - 1)), -dif(uz, at(x + 1, y, z), at(x - 1, y, z)));
    }
    w = __dadd_rn(w, __dmul_rn(0.5, __dadd_rn(__dadd_rn(__dmul_rn(wx, wx), __dmul_rn(wy, wy)),
                                               __dmul_rn(wz, wz))));
  }
  const double vals[kDiagVals] = {e, w, bad};
#pragma unroll
  for (int v = 0; v < kDiagVals; ++v) {
    const double s = diag_block_sum(vals[v], sh);
    if (threadIdx.x == 0) partials[(size_t)blockIdx.x * kDiagVals + v] = s;
  }
}

// One warp adds the partials in a fixed order: lane l takes blocks l,
// l + 32, ..., then a fixed shuffle tree.
__global__ void diag_finish(const double* partials, int nblocks, double* out) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x >= 32) return;
  for (int v = 0; v < kDiagVals; ++v) {
    double s = 0;
    for (int b = lane; b < nblocks; b += 32) s += partials[(size_t)b * kDiagVals + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[v] = s;
  }
}

}  // namespace m3lb
