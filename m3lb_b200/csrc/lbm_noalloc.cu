// m3lb_reduce_static: the FP64 mass / momentum / energy / slot-sum reduction
// for callers that cannot allocate device memory.
//
// Why it exists.  Every other entry point works on a handle, and creating a
// handle allocates (cudaMalloc) the populations, flags, fields and the
// reduction's scratch.  Some callers cannot allocate at all: a host that
// manages every byte of device memory itself (the populations sit in its own
// pool), or a loop that must not touch the allocator while it runs.  They
// hold the population array and the flags themselves and only need the
// reduction.  This entry point runs the same two reduction kernels as
// m3lb_reduce, but takes the partial sums' scratch from a fixed array
// compiled into the library, so it allocates nothing.
//
// The scratch is `g_reduce_scratch` below: kStaticBlocks block partials of
// six doubles (768 KiB).  Every GPU that loads the library holds it until the
// process exits.  Stage one uses one thread per interior node, so the largest
// lattice accepted is kStaticBlocks * 256 = 4,194,304 interior nodes (for
// example 160^3); larger ones are rejected with M3LB_ERR_INVALID.
//
// Host code may not pass the array's name to a kernel: in host code the name
// is a host-side stand-in, not a device address.  The device address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current, on the first call made on that device; make that first call before
// any stream capture.
//
// All calls share the one array and each call overwrites the partials the
// previous call left there.  Nothing in it needs clearing: the second kernel
// reads only partials the first kernel of the same call has written.  Calls
// that overlap on the GPU (different streams, or different host threads,
// without ordering between them) race on the array and give wrong sums.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/m3lb.h"
#include "lbm_launch.h"

namespace m3lb {
void set_last_error(const char* msg);  // lbm_capi.cu
}

using namespace m3lb;

namespace {

constexpr int kStaticBlocks = 16384;
constexpr long long kStaticMaxNodes = (long long)kStaticBlocks * kReduceThreads;

static __device__ __align__(256) double g_reduce_scratch[kStaticBlocks * kReduceVals];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

int fail(int code, const std::string& msg) {
  set_last_error(msg.c_str());  // read back through m3lb_last_error()
  return code;
}

// Device address of the scratch array on the current device, looked up once
// per device.
int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(M3LB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(M3LB_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_reduce_scratch);
    if (e != cudaSuccess || !p)
      return fail(M3LB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_reduce_scratch): ") +
                                     cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return M3LB_OK;
}

const Launchers* table(int lattice, int storage) {
  if (lattice == 9) {
    switch (storage) {
      case M3LB_STORE_F32: return launchers_D2Q9_F32();
      case M3LB_STORE_F16: return launchers_D2Q9_F16();
      case M3LB_STORE_BF16: return launchers_D2Q9_BF16();
      case M3LB_STORE_F64: return launchers_D2Q9_F64();
    }
  } else if (lattice == 27) {
    switch (storage) {
      case M3LB_STORE_F32: return launchers_D3Q27_F32();
      case M3LB_STORE_F16: return launchers_D3Q27_F16();
      case M3LB_STORE_BF16: return launchers_D3Q27_BF16();
      case M3LB_STORE_F64: return launchers_D3Q27_F64();
    }
  }
  return nullptr;
}

}  // namespace

extern "C" int m3lb_reduce_static(int lattice, int nx, int ny, int nz, int px, int py, int pz,
                                  int op, int storage, int shifted, int forcing, double fx,
                                  double fy, double fz, const void* populations,
                                  const uint8_t* flags, long long timestep, void* stream,
                                  double* out) {
  if (!populations || !out) return fail(M3LB_ERR_INVALID, "reduce_static: null pointer");
  const Launchers* T = table(lattice, storage);
  if (!T) return fail(M3LB_ERR_INVALID, "reduce_static: bad lattice or storage");
  if (lattice == 9 && nz != 1) return fail(M3LB_ERR_INVALID, "reduce_static: D2Q9 needs nz == 1");
  if (nx < 1 || ny < 1 || nz < 1 || op < M3LB_OP_NONE || op > M3LB_OP_CM)
    return fail(M3LB_ERR_INVALID, "reduce_static: bad extent or operator");
  if (!shifted && op != M3LB_OP_NONE && (storage == M3LB_STORE_F16 || storage == M3LB_STORE_BF16))
    return fail(M3LB_ERR_UNSUPPORTED, "reduce_static: 16-bit storage holds shifted populations only");
  const long long nint = (long long)nx * ny * nz;
  if (nint > kStaticMaxNodes) {
    char buf[200];
    std::snprintf(buf, sizeof buf,
                  "reduce_static: %lld interior nodes exceed the fixed scratch, which holds "
                  "%d block partials (at most %lld nodes); use m3lb_reduce",
                  nint, kStaticBlocks, kStaticMaxNodes);
    return fail(M3LB_ERR_INVALID, buf);
  }
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;

  // Domain(nx, ny, nz, px, py, pz): halo only along non-periodic axes.
  auto halo = [](int n, int per) { return n <= 1 ? 0 : (per ? 0 : 1); };
  StepArgs a{};
  Geo& g = a.g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.px = px != 0; g.py = py != 0; g.pz = pz != 0;
  g.hx = halo(nx, g.px); g.hy = halo(ny, g.py); g.hz = halo(nz, g.pz);
  g.sx = nx + 2 * g.hx; g.sy = ny + 2 * g.hy; g.sz = nz + 2 * g.hz;
  g.nch = (g.sx + kChunk - 1) / kChunk;
  g.n_padded = (long long)g.sx * g.sy * g.sz;
  a.f = const_cast<void*>(populations);
  a.flags = flags;
  a.parity = (int)(timestep & 1);
  a.fx = forcing ? fx : 0; a.fy = forcing ? fy : 0; a.fz = forcing ? fz : 0;

  const int nblocks = (int)((nint + kReduceThreads - 1) / kReduceThreads);
  cudaError_t e = T->reduce(a, op, shifted != 0 || op == M3LB_OP_NONE, forcing != 0, scratch,
                            nblocks, out,
                            static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return fail(M3LB_ERR_CUDA, std::string("reduce_static: ") + cudaGetErrorString(e));
  return M3LB_OK;
}
