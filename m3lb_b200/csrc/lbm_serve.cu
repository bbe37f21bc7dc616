// Serving loop: many independent lattices resident in HBM, advanced together.
//
// A request is one periodic D3Q27 Taylor-Green lattice (size N, operator,
// amplitude u0, step count).  The server admits queued requests in arrival
// order while their device footprint fits the HBM budget, keeps every
// admitted lattice resident until its last step, and advances all of them in
// scheduling rounds.  A round runs R time steps of every resident lattice
// (R = the smallest remaining step count, capped by the configured round
// length); each time step is one launch of the batched kernel per operator,
// over a device table of (lattice, first chunk) items, and the launches of a
// round are captured once into a CUDA graph and replayed while the resident
// set does not change.  Finished lattices are reduced (FP64 mass, momentum,
// energy) and, optionally, their rho and u copied out; their memory returns
// to the stream-ordered pool and the next requests are admitted.
//
// Each lattice chunk is updated by pairs_unit, the same device code as the
// single-lattice paired kernel, so a request's result does not depend on
// what else is resident: it is bit-identical alone, in any mix, and through
// the single-lattice C ABI with the same kernel.
//
// With 16-bit storage the lattices can instead go through the row kernel
// (lbm_rows.cuh, batch_rows): one persistent launch per time step and per
// (operator, row width in chunks) group, each CTA moving whole rows of
// whichever lattice of its group they belong to through shared memory by
// TMA.  The launch reads its group's row count and item table from device
// memory, and a lattice that has done its steps sits the rest of a round
// out inside the kernel, so every round runs the configured length and a
// round's launches are captured once per (groups present, length) and
// replayed from then on, whatever lattices come and go.  The row kernel's
// per-node arithmetic is the paired kernel's, so results stay bit-identical
// across the two paths.
//
// The reference has no serving loop; this file has no counterpart there.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "../../include/m3lb.h"
#include "lbm_host.h"
#include "lbm_kernels.cuh"
#include "lbm_rows.cuh"

using namespace m3lb;

namespace {

// ------------------------------------------------------------------ device
struct BatchItem {
  StepArgs a;             // geometry, populations, rates (parity set per step)
  long long first_unit;   // first chunk of this lattice in the launch
  long long t0;           // lattice time at the start of the round
};

constexpr int kBatchThreads = 128;
constexpr int kMaxItems = 1024;  // lattices in one launch (shared-memory search table)
// Batched row launches: one group per (operator, row width in chunks).
constexpr int kRowGroups = 4 * kRowsMaxChunks;
using RowItem27 = RowItem<D3Q27>;

// One time step of every lattice in `items` (all with operator OP): warp u
// of the grid updates unit u - first_unit of the item whose range holds u,
// a chunk (DENSE false) or 64 consecutive nodes (DENSE true) of pairs_unit.
// Resident 128-thread blocks per SM of the batched kernel: four (128
// registers) for every operator on 16-bit storage, where the paired kernel
// runs three for BGK / TRT and five for MRT / CM.  Measured on sets of
// resident lattices (dense mapping, N = 160 / 96 / 48): BGK 27.6 -> 29.5
// GLUPS and TRT 26.7 -> 28.3 at N = 160 (a few bytes of spills buy 16 warps
// per SM instead of 12); CM 26.2 / 26.3 / 24.6 -> 26.8-28.9 / 28.8 / 27.2
// (five blocks spill more at 102 registers; six, at 80, lose 15 %).
template <int OP, int ST>
constexpr int batch_min_blocks() {
  return (ST == kF16 || ST == kBF16 || ST == kF16C) ? 4 : pair_min_blocks<OP, ST>();
}

template <int ST, int OP, int EQ, bool DENSE>
__global__ void __launch_bounds__(kBatchThreads, batch_min_blocks<OP, ST>())
batch_step(const BatchItem* __restrict__ items, int n_items, long long n_units, int s) {
  __shared__ long long first[kMaxItems];
  for (int i = threadIdx.x; i < n_items; i += blockDim.x) first[i] = items[i].first_unit;
  __syncthreads();
  const long long u = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (u >= n_units) return;  // whole warp (uniform)
  int lo = 0, hi = n_items - 1;  // last item with first <= u
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (first[mid] <= u) lo = mid; else hi = mid - 1;
  }
  StepArgs a = items[lo].a;
  a.parity = (int)((items[lo].t0 + s) & 1);
  pairs_unit<D3Q27, ST, OP, EQ, true, false, DENSE>(a, u - first[lo], threadIdx.x & 31);
}

// Taylor-Green benchmark initial field (the analytic pressure in rho, w = 0)
// on an N^3 periodic box, in FP64, rounded to the FP32 fields the seed reads.
__global__ void tgv_field_kernel(int n, double u0, float* rho, float* ux, float* uy, float* uz) {
  const long long nn = (long long)n * n * n;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)(i / ((long long)n * n));
  const double k = 2.0 * 3.14159265358979323846 / n;
  const double X = x * k, Y = y * k, Z = z * k;
  const double dr = 3.0 * u0 * u0 / 16.0;
  rho[i] = (float)(1.0 + dr * (cos(2 * X) + cos(2 * Y)) * (cos(2 * Z) + 2.0));
  ux[i] = (float)(u0 * sin(X) * cos(Y) * cos(Z));
  uy[i] = (float)(-u0 * cos(X) * sin(Y) * cos(Z));
  uz[i] = 0.0f;
}

using BatchFn = void (*)(const BatchItem*, int, long long, int);

template <int ST, bool DENSE>
BatchFn batch_fn_st(int op) {
  switch (op) {
    case M3LB_OP_BGK: return batch_step<ST, 1, 0, DENSE>;
    case M3LB_OP_TRT: return batch_step<ST, 2, 0, DENSE>;
    case M3LB_OP_MRT: return batch_step<ST, 3, 0, DENSE>;
    case M3LB_OP_CM: return batch_step<ST, 4, 0, DENSE>;
    default: return nullptr;
  }
}
BatchFn batch_fn(int storage, int op, bool dense = false) {
  switch (storage) {
    case M3LB_STORE_F16: return dense ? batch_fn_st<kF16, true>(op) : batch_fn_st<kF16, false>(op);
    case M3LB_STORE_BF16: return dense ? batch_fn_st<kBF16, true>(op) : batch_fn_st<kBF16, false>(op);
    case M3LB_STORE_F16C: return dense ? batch_fn_st<kF16C, true>(op) : batch_fn_st<kF16C, false>(op);
    case M3LB_STORE_F32: return dense ? batch_fn_st<kF32, true>(op) : batch_fn_st<kF32, false>(op);
    default: return nullptr;
  }
}

// -------------------------------------------------------------------- host
int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  set_last_error(buf);
  return code;
}

#define SRV_TRY(call)                                                             \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(M3LB_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));        \
  } while (0)

using Clock = std::chrono::steady_clock;

struct Lattice {
  RowMaps<D3Q27> maps{};    // the row kernel's tensor maps of its populations
  m3lb_request req;
  Geo g{};
  const Launchers* L = nullptr;
  void* f = nullptr;
  size_t bytes = 0;         // admission footprint
  long long t = 0;          // time steps done
  long long units = 0;      // chunks per time step
  long long dense_units = 0;  // 64-node units per time step (dense mapping)
  double admitted = 0;
};

struct Finished {
  m3lb_result res;
  std::vector<float> fields;  // rho, ux, uy, uz (keep_fields)
};

constexpr int kOps[4] = {M3LB_OP_BGK, M3LB_OP_TRT, M3LB_OP_MRT, M3LB_OP_CM};

// A launched round: its end event and the requests whose readout it carries;
// for a round the mapping tuner measures, timing events around its launches,
// the mapping it ran and its lattice updates.
struct Inflight {
  cudaEvent_t end = nullptr;
  std::vector<size_t> finishing;  // indices into done
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  int cand = -1;                  // 0 chunks, 1 dense
  double lups = 0;
};

// Rounds the tuner measures with each mapping before it fixes the fastest,
// and its candidates: 64-slot chunks, dense 64-node strips, whole rows.
constexpr int kTuneRounds = 6;
constexpr int kCands = 3;
constexpr int kCandRows = 2;

// A captured round of batched row launches: the groups it launches and its
// length.
struct RowGraph {
  unsigned mask = 0;
  int R = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
constexpr int kRowGraphs = 8;

}  // namespace

struct m3lb_server {
  m3lb_serve_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  std::vector<m3lb_request> submitted;
  std::deque<m3lb_request> queue;   // arrived, not admitted
  std::vector<Lattice> active;
  std::vector<Finished> done;
  size_t resident = 0;              // bytes held by active lattices
  uint8_t* zero_flags = nullptr;    // all-fluid flags for seeding and readout
  long long zero_flags_bytes = 0;
  double* partials = nullptr;       // reduction scratch (one lattice at a time)
  int partial_blocks = 0;
  double* red_out = nullptr;
  BatchItem* items_dev = nullptr;   // [4][kMaxItems]
  BatchItem* items_host = nullptr;  // pinned, two of that shape: a round's table is
                                    // still to be copied while the next is built
  int flip = 0;
  int n_items[4] = {0, 0, 0, 0};
  long long n_units[4] = {0, 0, 0, 0};
  bool dense[4] = {false, false, false, false};  // unit mapping of each operator's launch
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  long long set_version = 0, graph_version = -1;
  int graph_R = -1;
  long long prev_version = -1;      // resident set and R of the previous round
  int prev_R = -1;
  int graph_map = -1, prev_map = -1;  // unit mappings (bit o: operator o dense) of both
  // M3LB_MAP_TUNE: rounds launched / measured with each mapping, their time
  // and lattice updates, the mapping of the round being built (-1: the
  // automatic rule), and the choice once made (-1 until then)
  int tune_launched[kCands] = {0, 0, 0}, tune_measured[kCands] = {0, 0, 0};
  double tune_ms[kCands] = {0, 0, 0}, tune_lups[kCands] = {0, 0, 0};
  int tune_cand = -1, tuned = -1;
  // batched row launches: device item table and per-group launch
  // descriptors, their pinned host copies (two of each, as for items_host),
  // the groups of the round being built, the captured rounds
  RowItem27* ritems_dev = nullptr;
  RowItem27* ritems_host = nullptr;
  RowBatch* rdesc_dev = nullptr;
  RowBatch* rdesc_host = nullptr;
  unsigned row_mask = 0, prev_row_mask = ~0u;
  int prev_row_R = -1;
  std::vector<RowGraph> rgraphs;
  // one stream per group of a round (its steps depend only on each other),
  // forked from and joined back to `stream`
  std::vector<cudaStream_t> row_streams;
  std::vector<cudaEvent_t> row_joins;
  cudaEvent_t row_fork = nullptr;
  std::vector<cudaEvent_t> free_timing;
  double* red_slots = nullptr;      // pinned, kReduceVals per request of a run
  int red_cap = 0;
  std::deque<Inflight> inflight;    // launched rounds not yet observed complete
  std::vector<cudaEvent_t> free_events;
  m3lb_serve_stats stats{};
};

namespace {

struct SrvGuard {
  int prev = -1;
  explicit SrvGuard(int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev) {
      prev = cur;
      cudaSetDevice(dev);
    }
  }
  ~SrvGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Device bytes a request holds while resident: populations, the FP32 seed /
// readout fields, the reduction scratch share.
size_t footprint(const m3lb_serve_config& c, int n) {
  const Geo g = make_geo(n, n, n, 1, 1, 1);
  return pop_elems(g, 27) * (size_t)elem_bytes(c.storage) + 16 * (size_t)n * n * n;
}

// Whole-row launches need 16-bit storage (their stage of 4 rows of up to 8
// chunks fits a CTA) and rows of at most 8 chunks (N <= 512, as admitted).
bool rows_eligible(const m3lb_server* s) { return elem_bytes(s->cfg.storage) == 2; }

// Whether the round being built goes through the row kernel: as configured;
// automatic: whenever eligible; tuner: its candidate or its choice.
bool use_rows(const m3lb_server* s) {
  if (!rows_eligible(s)) return false;
  if (s->cfg.mapping == M3LB_MAP_ROWS || s->cfg.mapping == M3LB_MAP_AUTO) return true;
  if (s->cfg.mapping == M3LB_MAP_TUNE) {
    const int m = s->tuned >= 0 ? s->tuned : s->tune_cand;
    return m == kCandRows;
  }
  return false;
}

double now_s(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

int ensure_zero_flags(m3lb_server* s, long long bytes) {
  if (bytes <= s->zero_flags_bytes) return M3LB_OK;
  SRV_TRY(cudaStreamSynchronize(s->stream));
  if (s->zero_flags) SRV_TRY(cudaFree(s->zero_flags));
  s->zero_flags = nullptr;
  SRV_TRY(cudaMalloc((void**)&s->zero_flags, (size_t)bytes));
  SRV_TRY(cudaMemset(s->zero_flags, 0, (size_t)bytes));
  s->zero_flags_bytes = bytes;
  return M3LB_OK;
}

int ensure_partials(m3lb_server* s, int blocks) {
  if (blocks <= s->partial_blocks) return M3LB_OK;
  SRV_TRY(cudaStreamSynchronize(s->stream));
  if (s->partials) SRV_TRY(cudaFree(s->partials));
  s->partials = nullptr;
  SRV_TRY(cudaMalloc((void**)&s->partials, ((size_t)blocks + 1) * kReduceVals * sizeof(double)));
  s->partial_blocks = blocks;
  s->red_out = s->partials + (size_t)blocks * kReduceVals;
  return M3LB_OK;
}

StepArgs lattice_args(const m3lb_server* s, const Lattice& l) {
  StepArgs a{};
  a.g = l.g;
  a.f = l.f;
  a.flags = nullptr;
  a.parity = (int)(l.t & 1);
  a.omega = l.req.omega;
  a.omega2 = l.req.omega2;
  (void)s;
  return a;
}

// Admit one request: allocate its populations from the pool and seed the
// Taylor-Green equilibrium through the single-lattice seed path.
int admit(m3lb_server* s, const m3lb_request& r, double t_now) {
  Lattice l;
  l.req = r;
  l.g = make_geo(r.n, r.n, r.n, 1, 1, 1);
  l.L = table_for(27, s->cfg.storage);
  l.bytes = footprint(s->cfg, r.n);
  l.units = (long long)l.g.ny * l.g.nz * l.g.nch;
  l.dense_units = ((long long)r.n * r.n * r.n + kChunk - 1) / kChunk;
  l.admitted = t_now;
  int rc = ensure_zero_flags(s, l.g.n_padded);
  if (rc) return rc;
  SRV_TRY(cudaMallocAsync(&l.f, pop_elems(l.g, 27) * (size_t)elem_bytes(s->cfg.storage),
                          s->stream));
  const size_t nn = (size_t)r.n * r.n * r.n;
  float* fld = nullptr;
  SRV_TRY(cudaMallocAsync((void**)&fld, 4 * nn * sizeof(float), s->stream));
  tgv_field_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s->stream>>>(r.n, r.u0, fld, fld + nn,
                                                                          fld + 2 * nn, fld + 3 * nn);
  SRV_TRY(cudaGetLastError());
  SeedArgs sa{};
  sa.g = l.g;
  sa.f = l.f;
  sa.flags = s->zero_flags;
  sa.parity = 0;
  sa.mode = 1;
  sa.rho0 = 1;
  // the seed reads fields of the arithmetic type: FP32 except for FP64 storage
  sa.rho = fld; sa.ux = fld + nn; sa.uy = fld + 2 * nn; sa.uz = fld + 3 * nn;
  SRV_TRY(l.L->seed(sa, r.op, 0, true, s->stream));
  SRV_TRY(cudaFreeAsync(fld, s->stream));
  if (elem_bytes(s->cfg.storage) == 2)
    SRV_TRY(l.L->row_maps(lattice_args(s, l), &l.maps, sizeof l.maps));
  s->resident += l.bytes;
  s->active.push_back(l);
  ++s->set_version;
  return M3LB_OK;
}

// Enqueue the readout of a finished lattice (FP64 reductions into its pinned
// slot; rho, u when kept) and the release of its memory.  The result is
// complete when the round's end event is.
int finish(m3lb_server* s, Lattice& l) {
  Finished fin;
  std::memset(&fin.res, 0, sizeof fin.res);
  fin.res.id = l.req.id;
  fin.res.arrival = l.req.arrival;
  fin.res.admitted = l.admitted;
  fin.res.n = l.req.n;
  fin.res.op = l.req.op;
  fin.res.steps = l.req.steps;
  const size_t slot = s->done.size();
  if ((int)slot >= s->red_cap) return fail(M3LB_ERR_INVALID, "serve: result slots exhausted");
  StepArgs a = lattice_args(s, l);
  const int nb = reduce_blocks(l.g);
  int rc = ensure_partials(s, nb);
  if (rc) return rc;
  SRV_TRY(l.L->reduce(a, l.req.op, true, false, s->partials, nb, s->red_out, s->stream));
  SRV_TRY(cudaMemcpyAsync(s->red_slots + slot * kReduceVals, s->red_out,
                          kReduceVals * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  const size_t nn = (size_t)l.req.n * l.req.n * l.req.n;
  if (s->cfg.keep_fields) {
    float* fld = nullptr;
    SRV_TRY(cudaMallocAsync((void**)&fld, 4 * nn * sizeof(float), s->stream));
    StepArgs m = a;
    m.flags = s->zero_flags;
    m.rho = fld; m.ux = fld + nn; m.uy = fld + 2 * nn; m.uz = fld + 3 * nn;
    SRV_TRY(l.L->macro(m, l.req.op, true, false, s->stream));
    fin.fields.resize(4 * nn);
    SRV_TRY(cudaMemcpyAsync(fin.fields.data(), fld, 4 * nn * sizeof(float),
                            cudaMemcpyDeviceToHost, s->stream));
    SRV_TRY(cudaFreeAsync(fld, s->stream));
  }
  SRV_TRY(cudaFreeAsync(l.f, s->stream));
  fin.res.node_steps = (long long)nn * l.req.steps;
  fin.res.status = M3LB_ERR_INVALID;  // until observed complete
  s->resident -= l.bytes;
  s->done.push_back(std::move(fin));
  return M3LB_OK;
}

// Wait for the oldest launched round; stamp the requests it finished.
int retire_oldest(m3lb_server* s, Clock::time_point t0) {
  Inflight f = s->inflight.front();
  s->inflight.pop_front();
  SRV_TRY(cudaEventSynchronize(f.end));
  const double t = now_s(t0);
  if (f.cand >= 0) {
    float ms = 0;
    SRV_TRY(cudaEventElapsedTime(&ms, f.t0, f.t1));
    s->tune_ms[f.cand] += ms;
    s->tune_lups[f.cand] += f.lups;
    s->tune_measured[f.cand] += 1;
    s->free_timing.push_back(f.t0);
    s->free_timing.push_back(f.t1);
    const int ncand = rows_eligible(s) ? kCands : 2;
    bool all = true;
    for (int c = 0; c < ncand; ++c) all = all && s->tune_measured[c] >= kTuneRounds;
    if (s->tuned < 0 && all) {
      // the highest rate of lattice updates per second of GPU time
      double best = -1;
      for (int c = 0; c < ncand; ++c) {
        const double r = s->tune_lups[c] / std::max(s->tune_ms[c], 1e-9);
        if (r > best) { best = r; s->tuned = c; }
      }
      static const int kMap[kCands] = {M3LB_MAP_CHUNKS, M3LB_MAP_DENSE, M3LB_MAP_ROWS};
      s->stats.tuned_mapping = kMap[s->tuned];
      s->stats.tuned_chunks_mlups = s->tune_lups[0] / std::max(s->tune_ms[0], 1e-9) * 1e-3;
      s->stats.tuned_dense_mlups = s->tune_lups[1] / std::max(s->tune_ms[1], 1e-9) * 1e-3;
      if (ncand > kCandRows)
        s->stats.tuned_rows_mlups = s->tune_lups[2] / std::max(s->tune_ms[2], 1e-9) * 1e-3;
    }
  }
  for (size_t i : f.finishing) {
    m3lb_result& r = s->done[i].res;
    const double* v = s->red_slots + i * kReduceVals;
    r.mass = v[0];
    for (int k = 0; k < 3; ++k) r.momentum[k] = v[1 + k];
    r.energy = v[4];
    r.finished = t;
    r.status = M3LB_OK;
    s->stats.node_steps += r.node_steps;
    s->stats.finished += 1;
  }
  s->free_events.push_back(f.end);
  return M3LB_OK;
}

// Item tables of the resident set, one per operator, for a round starting
// now; returns through n_items / n_units.
BatchItem* host_table(m3lb_server* s) { return s->items_host + (size_t)s->flip * 4 * kMaxItems; }

// The unit mapping of one operator's launch: as configured, or (automatic)
// dense when a lattice of it has rows that leave chunk lanes idle (N not a
// multiple of 64), chunks otherwise (the two are the same then).
void choose_mapping(m3lb_server* s) {
  if (s->cfg.mapping == M3LB_MAP_TUNE) {
    const int m = s->tuned >= 0 ? s->tuned : s->tune_cand;
    if (m == 0 || m == 1) {
      for (int o = 0; o < 4; ++o) s->dense[o] = m == 1;
      return;
    }
  }
  for (int o = 0; o < 4; ++o) s->dense[o] = s->cfg.mapping == M3LB_MAP_DENSE;
  if (s->cfg.mapping != M3LB_MAP_AUTO && s->cfg.mapping != M3LB_MAP_TUNE) return;
  for (const Lattice& l : s->active) {
    int o = 0;
    while (kOps[o] != l.req.op) ++o;
    if (l.req.n % kChunk != 0) s->dense[o] = true;
  }
}

void build_items(m3lb_server* s) {
  BatchItem* tab = host_table(s);
  choose_mapping(s);
  for (int o = 0; o < 4; ++o) {
    s->n_items[o] = 0;
    s->n_units[o] = 0;
  }
  for (const Lattice& l : s->active) {
    int o = 0;
    while (kOps[o] != l.req.op) ++o;
    BatchItem& it = tab[o * kMaxItems + s->n_items[o]++];
    it.a = lattice_args(s, l);
    it.first_unit = s->n_units[o];
    it.t0 = l.t;
    s->n_units[o] += s->dense[o] ? l.dense_units : l.units;
  }
}

int launch_round(m3lb_server* s, int R) {
  for (int step = 0; step < R; ++step)
    for (int o = 0; o < 4; ++o) {
      if (!s->n_items[o]) continue;
      BatchFn fn = batch_fn(s->cfg.storage, kOps[o], s->dense[o]);
      const long long threads = s->n_units[o] * 32;
      const unsigned blocks = (unsigned)((threads + kBatchThreads - 1) / kBatchThreads);
      void* args[4];
      const BatchItem* ip = s->items_dev + (size_t)o * kMaxItems;
      int ni = s->n_items[o];
      long long nu = s->n_units[o];
      int st = step;
      args[0] = (void*)&ip; args[1] = &ni; args[2] = &nu; args[3] = &st;
      SRV_TRY(cudaLaunchKernel((const void*)fn, dim3(blocks), dim3(kBatchThreads), args, 0,
                               s->stream));
    }
  return M3LB_OK;
}

// One round: R steps of every resident lattice.  A round whose resident set
// and R repeat the previous one's is captured into a CUDA graph (or replays
// the graph already captured for them); a round after a change launches
// directly, since its graph would be used once.
int run_round(m3lb_server* s, int R) {
  // at most two rounds are in flight and the older one has completed before
  // a new table is built, so alternating host tables never overwrites one
  // whose copy is still queued
  s->flip ^= 1;
  build_items(s);
  const BatchItem* tab = host_table(s);
  for (int o = 0; o < 4; ++o)
    if (s->n_items[o])
      SRV_TRY(cudaMemcpyAsync(s->items_dev + (size_t)o * kMaxItems, tab + (size_t)o * kMaxItems,
                              s->n_items[o] * sizeof(BatchItem), cudaMemcpyHostToDevice, s->stream));
  int map = 0;
  for (int o = 0; o < 4; ++o) map |= (s->dense[o] ? 1 : 0) << o;
  const bool cached = s->graph_exec && s->graph_version == s->set_version && s->graph_R == R &&
                      s->graph_map == map;
  const bool repeat = s->prev_version == s->set_version && s->prev_R == R && s->prev_map == map;
  s->prev_version = s->set_version;
  s->prev_R = R;
  s->prev_map = map;
  if (!cached && !repeat) {
    const int rc = launch_round(s, R);
    if (rc) return rc;
  } else {
    if (!cached) {
      if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
      if (s->graph) cudaGraphDestroy(s->graph);
      s->graph_exec = nullptr;
      s->graph = nullptr;
      SRV_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
      const int rc = launch_round(s, R);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
      if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
      }
      SRV_TRY(e);
      s->graph = g;
      SRV_TRY(cudaGraphInstantiate(&s->graph_exec, s->graph, 0));
      s->graph_version = s->set_version;
      s->graph_R = R;
      s->graph_map = map;
      s->stats.graph_captures += 1;
    }
    SRV_TRY(cudaGraphLaunch(s->graph_exec, s->stream));
    s->stats.graph_launches += 1;
  }
  for (Lattice& l : s->active) l.t += R;
  s->stats.rounds += 1;
  for (int o = 0; o < 4; ++o) {
    s->stats.launches += (long long)R * (s->n_items[o] ? 1 : 0);
    s->stats.dense_launches += (long long)R * (s->n_items[o] && s->dense[o] ? 1 : 0);
  }
  return M3LB_OK;
}

// The batched row tables of the resident set for a round: items grouped by
// (operator, row width), each group's rows numbered in item order; the
// groups present in s->row_mask.
void build_row_items(m3lb_server* s) {
  RowItem27* tab = s->ritems_host + (size_t)s->flip * kMaxItems;
  RowBatch* desc = s->rdesc_host + (size_t)s->flip * kRowGroups;
  int count[kRowGroups] = {};
  for (const Lattice& l : s->active) {
    int o = 0;
    while (kOps[o] != l.req.op) ++o;
    ++count[o * kRowsMaxChunks + l.g.nch - 1];
  }
  int first = 0;
  s->row_mask = 0;
  for (int g = 0; g < kRowGroups; ++g) {
    desc[g].first_item = first;
    desc[g].n_items = 0;
    desc[g].n_rows = 0;
    first += count[g];
    if (count[g]) s->row_mask |= 1u << g;
  }
  for (const Lattice& l : s->active) {
    int o = 0;
    while (kOps[o] != l.req.op) ++o;
    RowBatch& d = desc[o * kRowsMaxChunks + l.g.nch - 1];
    RowItem27& it = tab[d.first_item + d.n_items++];
    it.maps = l.maps;
    it.a = lattice_args(s, l);
    it.first_row = d.n_rows;
    it.t0 = l.t;
    it.t_end = l.req.steps;
    d.n_rows += (long long)l.g.ny * l.g.nz;
  }
}

// The groups' lattices are disjoint, so a group's R steps depend only on
// each other: with several groups each runs on its own stream (forked from
// the server stream after the tables' upload, joined back before the
// round's readouts), so one group's launch tail overlaps the others' work.
int ensure_row_streams(m3lb_server* s, int groups) {
  if (groups < 2) return M3LB_OK;
  if (!s->row_fork) SRV_TRY(cudaEventCreateWithFlags(&s->row_fork, cudaEventDisableTiming));
  while ((int)s->row_streams.size() < groups) {
    cudaStream_t st = nullptr;
    cudaEvent_t e = nullptr;
    SRV_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    s->row_streams.push_back(st);
    SRV_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    s->row_joins.push_back(e);
  }
  return M3LB_OK;
}

// (the streams and events exist: ensure_row_streams ran before any capture)
int launch_rows_round(m3lb_server* s, int R) {
  const Launchers* T = table_for(27, s->cfg.storage);
  const int groups = __builtin_popcount(s->row_mask);
  if (groups > 1) SRV_TRY(cudaEventRecord(s->row_fork, s->stream));
  int lane = 0;
  for (int g = 0; g < kRowGroups; ++g) {
    if (!(s->row_mask >> g & 1u)) continue;
    cudaStream_t st = groups > 1 ? s->row_streams[lane] : s->stream;
    if (groups > 1) SRV_TRY(cudaStreamWaitEvent(st, s->row_fork, 0));
    for (int step = 0; step < R; ++step)
      SRV_TRY(T->batch_rows(s->ritems_dev, s->rdesc_dev + g, kOps[g / kRowsMaxChunks],
                            g % kRowsMaxChunks + 1, step, st));
    if (groups > 1) {
      SRV_TRY(cudaEventRecord(s->row_joins[lane], st));
      SRV_TRY(cudaStreamWaitEvent(s->stream, s->row_joins[lane], 0));
    }
    ++lane;
  }
  return M3LB_OK;
}

// A round of batched row launches: the tables go to the device ahead of the
// launches; a round whose groups and length match a captured one replays it,
// a round repeating the previous round's groups and length is captured, and
// any other launches directly.
int run_round_rows(m3lb_server* s, int R) {
  s->flip ^= 1;
  build_row_items(s);
  const size_t n = s->active.size();
  if (n)
    SRV_TRY(cudaMemcpyAsync(s->ritems_dev, s->ritems_host + (size_t)s->flip * kMaxItems,
                            n * sizeof(RowItem27), cudaMemcpyHostToDevice, s->stream));
  SRV_TRY(cudaMemcpyAsync(s->rdesc_dev, s->rdesc_host + (size_t)s->flip * kRowGroups,
                          kRowGroups * sizeof(RowBatch), cudaMemcpyHostToDevice, s->stream));
  {
    const int rc = ensure_row_streams(s, __builtin_popcount(s->row_mask));
    if (rc) return rc;
  }
  RowGraph* hit = nullptr;
  for (RowGraph& g : s->rgraphs)
    if (g.mask == s->row_mask && g.R == R) hit = &g;
  const bool repeat = s->prev_row_mask == s->row_mask && s->prev_row_R == R;
  s->prev_row_mask = s->row_mask;
  s->prev_row_R = R;
  if (!hit && repeat && (int)s->rgraphs.size() < kRowGraphs) {
    RowGraph g;
    g.mask = s->row_mask;
    g.R = R;
    SRV_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = launch_rows_round(s, R);
    const cudaError_t e = cudaStreamEndCapture(s->stream, &g.graph);
    if (rc) {
      if (g.graph) cudaGraphDestroy(g.graph);
      return rc;
    }
    SRV_TRY(e);
    SRV_TRY(cudaGraphInstantiate(&g.exec, g.graph, 0));
    s->rgraphs.push_back(g);
    hit = &s->rgraphs.back();
    s->stats.graph_captures += 1;
  }
  if (hit) {
    SRV_TRY(cudaGraphLaunch(hit->exec, s->stream));
    s->stats.graph_launches += 1;
  } else {
    const int rc = launch_rows_round(s, R);
    if (rc) return rc;
  }
  for (Lattice& l : s->active) l.t = std::min<long long>(l.t + R, l.req.steps);
  s->stats.rounds += 1;
  const long long groups = __builtin_popcount(s->row_mask);
  s->stats.launches += (long long)R * groups;
  s->stats.rows_launches += (long long)R * groups;
  return M3LB_OK;
}

bool fits(const m3lb_server* s, const m3lb_request& r) {
  if (s->cfg.max_resident > 0 && (int)s->active.size() >= s->cfg.max_resident) return false;
  if ((int)s->active.size() >= kMaxItems) return false;
  return s->resident + footprint(s->cfg, r.n) <= s->cfg.hbm_budget;
}

}  // namespace

extern "C" {

int m3lb_serve_create(const m3lb_serve_config* cfg, m3lb_server** out) {
  if (!cfg || !out) return fail(M3LB_ERR_INVALID, "serve_create: null argument");
  *out = nullptr;
  if (!batch_fn(cfg->storage, M3LB_OP_CM))
    return fail(M3LB_ERR_UNSUPPORTED, "serve_create: storage %d is not served (F16, F16C, BF16, F32)",
                cfg->storage);
  if (cfg->round_steps < 1) return fail(M3LB_ERR_INVALID, "serve_create: round_steps must be >= 1");
  if (cfg->mapping < M3LB_MAP_AUTO || cfg->mapping > M3LB_MAP_ROWS)
    return fail(M3LB_ERR_INVALID,
                "serve_create: mapping must be M3LB_MAP_AUTO, _CHUNKS, _DENSE, _TUNE or _ROWS");
  if (cfg->mapping == M3LB_MAP_ROWS && elem_bytes(cfg->storage) != 2)
    return fail(M3LB_ERR_UNSUPPORTED, "serve_create: M3LB_MAP_ROWS needs 16-bit storage");
  auto* s = new m3lb_server();
  s->cfg = *cfg;
  cudaGetDevice(&s->device);
  auto bail = [&](int rc) { m3lb_serve_destroy(s); return rc; };
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(M3LB_ERR_CUDA, "serve_create: cannot create a stream"));
  if (cudaDeviceGetDefaultMemPool(&s->pool, s->device) == cudaSuccess) {
    // keep freed lattice memory in the pool for the next admissions
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (cudaMalloc((void**)&s->items_dev, 4 * kMaxItems * sizeof(BatchItem)) != cudaSuccess ||
      cudaMallocHost((void**)&s->items_host, 2 * 4 * kMaxItems * sizeof(BatchItem)) != cudaSuccess)
    return bail(fail(M3LB_ERR_MEMORY, "serve_create: cannot allocate the item tables"));
  std::memset(s->items_host, 0, 2 * 4 * kMaxItems * sizeof(BatchItem));
  if (cudaMalloc((void**)&s->ritems_dev, kMaxItems * sizeof(RowItem27)) != cudaSuccess ||
      cudaMallocHost((void**)&s->ritems_host, 2 * kMaxItems * sizeof(RowItem27)) != cudaSuccess ||
      cudaMalloc((void**)&s->rdesc_dev, kRowGroups * sizeof(RowBatch)) != cudaSuccess ||
      cudaMallocHost((void**)&s->rdesc_host, 2 * kRowGroups * sizeof(RowBatch)) != cudaSuccess)
    return bail(fail(M3LB_ERR_MEMORY, "serve_create: cannot allocate the row tables"));
  *out = s;
  return M3LB_OK;
}

int m3lb_serve_submit(m3lb_server* s, const m3lb_request* r) {
  if (!s || !r) return fail(M3LB_ERR_INVALID, "serve_submit: null argument");
  if (r->n < 2 || (r->n % 2) != 0)
    return fail(M3LB_ERR_INVALID, "serve_submit: N must be even and >= 2 (got %d)", r->n);
  if (r->steps < 0) return fail(M3LB_ERR_INVALID, "serve_submit: negative step count");
  if (!batch_fn(s->cfg.storage, r->op))
    return fail(M3LB_ERR_UNSUPPORTED, "serve_submit: operator %d is not served", r->op);
  if (footprint(s->cfg, r->n) > s->cfg.hbm_budget)
    return fail(M3LB_ERR_MEMORY, "serve_submit: N=%d needs %zu bytes, above the budget %zu",
                r->n, footprint(s->cfg, r->n), s->cfg.hbm_budget);
  s->submitted.push_back(*r);
  return M3LB_OK;
}

int m3lb_serve_run(m3lb_server* s, double time_limit) {
  if (!s) return fail(M3LB_ERR_INVALID, "serve_run: null handle");
  SrvGuard dg(s->device);
  std::vector<m3lb_request> pending = s->submitted;
  s->submitted.clear();
  std::stable_sort(pending.begin(), pending.end(),
                   [](const m3lb_request& a, const m3lb_request& b) { return a.arrival < b.arrival; });
  // pinned result slots for every request of this run (and those before)
  const int need = (int)(s->done.size() + pending.size() + s->queue.size() + s->active.size());
  if (need > s->red_cap) {
    double* p = nullptr;
    SRV_TRY(cudaStreamSynchronize(s->stream));
    SRV_TRY(cudaMallocHost((void**)&p, (size_t)std::max(need, 1) * kReduceVals * sizeof(double)));
    if (s->red_slots) {
      std::memcpy(p, s->red_slots, (size_t)s->red_cap * kReduceVals * sizeof(double));
      cudaFreeHost(s->red_slots);
    }
    s->red_slots = p;
    s->red_cap = std::max(need, 1);
  }
  size_t next = 0;
  const Clock::time_point t0 = Clock::now();
  while (next < pending.size() || !s->queue.empty() || !s->active.empty() || !s->inflight.empty()) {
    const double t = now_s(t0);
    if (time_limit > 0 && t > time_limit)
      return fail(M3LB_ERR_INVALID, "serve_run: time limit %.1f s reached with %zu queued, %zu resident",
                  time_limit, s->queue.size() + (pending.size() - next), s->active.size());
    while (next < pending.size() && pending[next].arrival <= t) s->queue.push_back(pending[next++]);
    while (!s->queue.empty() && fits(s, s->queue.front())) {
      const int rc = admit(s, s->queue.front(), t);
      if (rc) return rc;
      s->queue.pop_front();
    }
    if (s->active.empty()) {
      if (!s->inflight.empty()) {
        const int rc = retire_oldest(s, t0);
        if (rc) return rc;
      } else if (next < pending.size()) {
        const double wait = pending[next].arrival - now_s(t0);
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.005)));
      }
      continue;
    }
    // the mapping tuner alternates its candidates over its first rounds
    s->tune_cand = -1;
    if (s->cfg.mapping == M3LB_MAP_TUNE && s->tuned < 0) {
      const int ncand = rows_eligible(s) ? kCands : 2;
      int c = 0;
      for (int k = 1; k < ncand; ++k)
        if (s->tune_launched[k] < s->tune_launched[c]) c = k;
      if (s->tune_launched[c] < kTuneRounds) s->tune_cand = c;
    }
    // whole-row rounds run the configured length (a lattice that finishes
    // inside the round sits the rest out); chunk rounds end with the first
    // lattice to finish
    const bool rows = use_rows(s);
    long long R = rows ? 0 : s->cfg.round_steps;
    for (const Lattice& l : s->active) {
      if (rows) R = std::max<long long>(R, l.req.steps - l.t);
      else R = std::min<long long>(R, l.req.steps - l.t);
    }
    if (rows) R = std::min<long long>(R, s->cfg.round_steps);
    Inflight f;
    if (R > 0) {
      if (s->tune_cand >= 0) {
        for (int k = 0; k < 2; ++k) {
          if (s->free_timing.empty()) {
            cudaEvent_t e = nullptr;
            SRV_TRY(cudaEventCreate(&e));
            s->free_timing.push_back(e);
          }
          (k ? f.t1 : f.t0) = s->free_timing.back();
          s->free_timing.pop_back();
        }
        f.cand = s->tune_cand;
        for (const Lattice& l : s->active)
          f.lups += (double)l.req.n * l.req.n * l.req.n *
                    (double)std::min<long long>(R, l.req.steps - l.t);
        s->tune_launched[f.cand] += 1;
        SRV_TRY(cudaEventRecord(f.t0, s->stream));
      }
      const int rc = rows ? run_round_rows(s, (int)R) : run_round(s, (int)R);
      if (rc) return rc;
      if (f.cand >= 0) SRV_TRY(cudaEventRecord(f.t1, s->stream));
    }
    // lattices done after this round: readout and release follow it on the stream
    for (size_t i = 0; i < s->active.size();) {
      Lattice& l = s->active[i];
      if (l.t >= l.req.steps) {
        const int rc = finish(s, l);
        if (rc) return rc;
        f.finishing.push_back(s->done.size() - 1);
        s->active.erase(s->active.begin() + (long)i);
        ++s->set_version;
      } else {
        ++i;
      }
    }
    if (s->free_events.empty()) {
      cudaEvent_t e = nullptr;
      SRV_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      s->free_events.push_back(e);
    }
    f.end = s->free_events.back();
    s->free_events.pop_back();
    SRV_TRY(cudaEventRecord(f.end, s->stream));
    s->inflight.push_back(std::move(f));
    // at most two rounds queued: wait for the older one while the newer runs
    while (s->inflight.size() > 1) {
      const int rc = retire_oldest(s, t0);
      if (rc) return rc;
    }
  }
  s->stats.makespan = now_s(t0);
  return M3LB_OK;
}

int m3lb_serve_results(const m3lb_server* s, m3lb_result* out, int cap, int* count) {
  if (!s || !count) return fail(M3LB_ERR_INVALID, "serve_results: null argument");
  int n = 0;
  for (const Finished& f : s->done)
    if (f.res.status == M3LB_OK) {
      if (out && n < cap) out[n] = f.res;
      ++n;
    }
  *count = n;
  return M3LB_OK;
}

int m3lb_serve_fields(const m3lb_server* s, long long id, float* rho, float* ux, float* uy,
                      float* uz) {
  if (!s || !rho || !ux || !uy || !uz) return fail(M3LB_ERR_INVALID, "serve_fields: null argument");
  for (const Finished& f : s->done)
    if (f.res.id == id) {
      if (f.fields.empty())
        return fail(M3LB_ERR_INVALID, "serve_fields: fields of %lld were not kept", id);
      const size_t nn = f.fields.size() / 4;
      float* dst[4] = {rho, ux, uy, uz};
      for (int k = 0; k < 4; ++k) std::memcpy(dst[k], f.fields.data() + k * nn, nn * sizeof(float));
      return M3LB_OK;
    }
  return fail(M3LB_ERR_INVALID, "serve_fields: no finished request %lld", id);
}

int m3lb_serve_get_stats(const m3lb_server* s, m3lb_serve_stats* st) {
  if (!s || !st) return fail(M3LB_ERR_INVALID, "serve_stats: null argument");
  *st = s->stats;
  return M3LB_OK;
}

int m3lb_serve_destroy(m3lb_server* s) {
  if (!s) return M3LB_OK;
  SrvGuard dg(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (Lattice& l : s->active)
    if (l.f) cudaFree(l.f);
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  if (s->zero_flags) cudaFree(s->zero_flags);
  if (s->partials) cudaFree(s->partials);
  if (s->items_dev) cudaFree(s->items_dev);
  if (s->items_host) cudaFreeHost(s->items_host);
  for (RowGraph& g : s->rgraphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  if (s->ritems_dev) cudaFree(s->ritems_dev);
  if (s->ritems_host) cudaFreeHost(s->ritems_host);
  if (s->rdesc_dev) cudaFree(s->rdesc_dev);
  if (s->rdesc_host) cudaFreeHost(s->rdesc_host);
  if (s->red_slots) cudaFreeHost(s->red_slots);
  for (Inflight& f : s->inflight) {
    cudaEventDestroy(f.end);
    if (f.t0) cudaEventDestroy(f.t0);
    if (f.t1) cudaEventDestroy(f.t1);
  }
  for (cudaEvent_t e : s->free_events) cudaEventDestroy(e);
  for (cudaEvent_t e : s->free_timing) cudaEventDestroy(e);
  for (cudaStream_t st : s->row_streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  for (cudaEvent_t e : s->row_joins) cudaEventDestroy(e);
  if (s->row_fork) cudaEventDestroy(s->row_fork);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return M3LB_OK;
}

int m3lb_tgv_field(int n, double u0, float* rho, float* ux, float* uy, float* uz, void* stream) {
  if (n < 1 || !rho || !ux || !uy || !uz) return fail(M3LB_ERR_INVALID, "tgv_field: bad argument");
  const long long nn = (long long)n * n * n;
  tgv_field_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n, u0, rho, ux, uy, uz);
  SRV_TRY(cudaGetLastError());
  return M3LB_OK;
}

}  // extern "C"
