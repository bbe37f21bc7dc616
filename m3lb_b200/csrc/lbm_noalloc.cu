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
// Stage one runs as many blocks as m3lb_reduce gives the same lattice
// (reduce_blocks: one per 256 nodes, at most 4 * 148), each summing its nodes
// in the same grid-stride order, and stage two adds the partials in the same
// fixed order, so the six sums are bit-identical to m3lb_reduce's.
//
// Host code may not pass the array's name to a kernel: in host code the name
// is a host-side stand-in, not a device address.  The device address is
// looked up with cudaGetSymbolAddress, with the device current, on the first
// call made in a CUDA context, and kept for that context (keyed by the
// context's ID, ctx_cache.h): a call after cudaDeviceReset, or under another
// context, looks it up again.  Make the first call in a context before any
// stream capture.
//
// All calls share the one array and each call overwrites the partials the
// previous call left there.  Nothing in it needs clearing: the second kernel
// reads only partials the first kernel of the same call has written.  Calls
// that overlap on the GPU (different streams, or different host threads,
// without ordering between them) race on the array and give wrong sums.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/m3lb.h"
#include "ctx_cache.h"
#include "lbm_host.h"

using namespace m3lb;

namespace {

constexpr int kStaticBlocks = 16384;
constexpr long long kStaticMaxNodes = (long long)kStaticBlocks * kReduceThreads;

static __device__ __align__(256) double g_reduce_scratch[kStaticBlocks * kReduceVals];

constexpr int kMaxDevices = 64;
CtxAddrCache<kMaxDevices> g_scratch_cache;

int fail(int code, const std::string& msg) {
  set_last_error(msg.c_str());  // read back through m3lb_last_error()
  return code;
}

// ID of the context current on this thread, 0 when there is none or the
// driver offers no cuCtxGetId (the address is then looked up on every call).
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool resolved = false;
  if (!resolved) {
    void* f1 = nullptr;
    void* f2 = nullptr;
    cudaDriverEntryPointQueryResult q1, q2;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess) {
      get_current = reinterpret_cast<GetCurrent>(f1);
      get_id = reinterpret_cast<GetId>(f2);
    }
    resolved = true;
  }
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
  if (get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of the scratch array in the current context.
int scratch_for_current_context(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(M3LB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  cudaError_t le = cudaSuccess;
  auto lookup = [&](void** p) -> int {
    le = cudaGetSymbolAddress(p, g_reduce_scratch);
    return (le == cudaSuccess && *p) ? 0 : 1;
  };
  // A thread that has made no runtime call yet has no current context; the
  // first lookup binds the device's primary context, so ask for the ID after
  // it when there was none before.
  unsigned long long ctx = current_context_id();
  void* p = nullptr;
  if (ctx == 0) {
    if (lookup(&p))
      return fail(M3LB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_reduce_scratch): ") +
                                     cudaGetErrorString(le));
    ctx = current_context_id();
  }
  const int rc = g_scratch_cache.get(dev, ctx, lookup, &p);
  if (rc == -1) return fail(M3LB_ERR_INVALID, "device index out of range");
  if (rc)
    return fail(M3LB_ERR_CUDA, std::string("cudaGetSymbolAddress(g_reduce_scratch): ") +
                                   cudaGetErrorString(le));
  *out = static_cast<double*>(p);
  return M3LB_OK;
}

}  // namespace

extern "C" int m3lb_reduce_static(int lattice, int nx, int ny, int nz, int px, int py, int pz,
                                  int op, int storage, int shifted, int forcing, double fx,
                                  double fy, double fz, const void* populations,
                                  const uint8_t* flags, long long timestep, void* stream,
                                  double* out) {
  if (!populations || !out) return fail(M3LB_ERR_INVALID, "reduce_static: null pointer");
  const Launchers* T = table_for(lattice, storage);
  if (!T) return fail(M3LB_ERR_INVALID, "reduce_static: bad lattice or storage");
  if (lattice == 9 && nz != 1) return fail(M3LB_ERR_INVALID, "reduce_static: D2Q9 needs nz == 1");
  if (nx < 1 || ny < 1 || nz < 1 || op < M3LB_OP_NONE || op > M3LB_OP_CM)
    return fail(M3LB_ERR_INVALID, "reduce_static: bad extent or operator");
  if (!shifted && op != M3LB_OP_NONE && elem_bytes(storage) == 2)
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
  int rc = scratch_for_current_context(&scratch);
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

  // m3lb_reduce's block count (at most 4 * 148 <= kStaticBlocks), so the
  // partial sums and their fixed-order total are the same bit for bit
  const int nblocks = reduce_blocks(g);
  if (nblocks > kStaticBlocks) return fail(M3LB_ERR_INVALID, "reduce_static: too many blocks");
  cudaError_t e = T->reduce(a, op, shifted != 0 || op == M3LB_OP_NONE, forcing != 0, scratch,
                            nblocks, out,
                            static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return fail(M3LB_ERR_CUDA, std::string("reduce_static: ") + cudaGetErrorString(e));
  return M3LB_OK;
}
