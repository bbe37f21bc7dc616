// Row kernel: one CTA updates whole x-rows, moved by the tensor-memory
// accelerator (TMA).
//
// Layout facts it relies on (lbm_common.cuh, chunked SoA): one direction of
// one padded row is nch segments of 64 elements, Q * 64 elements apart.  A
// 3-D tensor map (x: 64, direction: Q, chunk: sz * sy * nch) with a box of
// (64, span, nch) and a traversal stride s along the direction axis moves
// ceil(span / s) directions q0, q0 + s, ... of one row in a single copy.
//
// Per row (y, z) of the update, Esoteric Pull reads and writes the same 27
// lines (src/memory/EsotericPull.hpp:61-111): direction 0 and the
// directions i + P of the own row (every other direction: one strided
// copy), and direction i + 1 - P of row (y + c_iy, z + c_iz) for every odd i
// (grouped by neighbour row into strided copies of one or two lines).  For
// D3Q27 a row moves in 11 copies each way instead of 27.  Every slot of
// those lines belongs to one node of this row, which reads it and later
// writes it, so:
//   * the copies of a row land in a stage buffer (cp.async.bulk.tensor,
//     mbarrier completion) and go back after the update
//     (cp.async.bulk.tensor, bulk-group completion);
//   * the update runs in place in shared memory; the ±1 x shift of a remote
//     line is a fixed per-lane offset (periodic wrap included), so there is
//     no shuffle, no chunk-edge load or store and no address arithmetic per
//     row in the update itself;
//   * rows are independent: CTAs never exchange data, and a row's global
//     lines are read and written only by its own CTA within a step.
// Warp w of a CTA takes chunk w of the row (nch <= 4 warps, nx even,
// periodic x; lanes past nx in a partial last chunk store nothing).  Rows stream through a kRowsStages-stage ring with the
// rows ahead of the one being updated in flight.
//
// Waits on the load barriers are bounded: past the limit the CTA records a
// status in StepArgs::err, lets its copies in flight finish (bounded again)
// and leaves; the host reports it at the next m3lb_sync.
#pragma once
#include <cuda.h>

#include "lbm_stream.cuh"

namespace m3lb {

constexpr int kRowsStages = 4;
constexpr int kRowsMaxWarps = 4;  // nch <= 4 (nx <= 256)
constexpr int kRowsLine = kRowsMaxWarps * kChunk;  // shared elements reserved per line
constexpr long long kRowsWaitCycles = 4000000000LL;  // ~2 s at 2 GHz
constexpr int kRowsSmemMax = 227 * 1024;              // dynamic shared memory per CTA

// ---------------------------------------------------------------- plan
// One copy of a row: own row or neighbour row (dy, dz); its first direction
// at parity 0 (q0; at parity P it is q0 + sgn * P), the number of lines and
// their direction stride, and which tensor map (box shape) moves it.
struct RowOp {
  int own, dy, dz, q0, sgn, count, stride, map;
};

template <class L>
struct RowPlan;

template <>
struct RowPlan<D3Q27> {
  static constexpr int NOPS = 11;
  static constexpr int NMAPS = 4;
  static constexpr int map_count[NMAPS] = {1, 13, 2, 2};
  static constexpr int map_stride[NMAPS] = {1, 2, 4, 6};
  static constexpr RowOp ops[NOPS] = {
      {1, 0, 0, 0, 0, 1, 1, 0},     // direction 0
      {1, 0, 0, 1, +1, 13, 2, 1},   // i + P, i = 1, 3, ..., 25
      {0, 0, 0, 2, -1, 1, 1, 0},    // i = 1
      {0, 1, 0, 4, -1, 2, 4, 2},    // i = 3, 7
      {0, 0, 1, 6, -1, 2, 6, 3},    // i = 5, 11
      {0, -1, 0, 10, -1, 1, 1, 0},  // i = 9
      {0, 0, -1, 14, -1, 1, 1, 0},  // i = 13
      {0, 1, 1, 16, -1, 2, 4, 2},   // i = 15, 19
      {0, 1, 1, 26, -1, 1, 1, 0},   // i = 25
      {0, 1, -1, 18, -1, 2, 4, 2},  // i = 17, 21
      {0, -1, 1, 24, -1, 1, 1, 0},  // i = 23
  };
};

template <>
struct RowPlan<D2Q9> {
  static constexpr int NOPS = 5;
  static constexpr int NMAPS = 3;
  static constexpr int map_count[NMAPS] = {1, 4, 2};
  static constexpr int map_stride[NMAPS] = {1, 2, 2};
  static constexpr RowOp ops[NOPS] = {
      {1, 0, 0, 0, 0, 1, 1, 0},    // direction 0
      {1, 0, 0, 1, +1, 4, 2, 1},   // i + P, i = 1, 3, 5, 7
      {0, 0, 0, 2, -1, 1, 1, 0},   // i = 1
      {0, 1, 0, 4, -1, 2, 2, 2},   // i = 3, 5
      {0, -1, 0, 8, -1, 1, 1, 0},  // i = 7
  };
};

// Where the kernel's value q lives: value 0 is direction 0, value i (odd) is
// the own direction i + P, value i + 1 the remote direction i + 1 - P.
template <class L>
struct RowSlots {
  using Pl = RowPlan<L>;
  static __host__ __device__ constexpr int op_of(int q) {
    if (q == 0) return 0;
    if (q % 2 == 1) return 1;
    for (int o = 2; o < Pl::NOPS; ++o)
      for (int j = 0; j < Pl::ops[o].count; ++j)
        if (Pl::ops[o].q0 + j * Pl::ops[o].stride == q) return o;
    return -1;
  }
  static __host__ __device__ constexpr int j_of(int q) {
    if (q == 0) return 0;
    if (q % 2 == 1) return (q - 1) / 2;
    const int o = op_of(q);
    for (int j = 0; j < Pl::ops[o].count; ++j)
      if (Pl::ops[o].q0 + j * Pl::ops[o].stride == q) return j;
    return -1;
  }
  // first shared element of a copy's block: blocks in op order, each
  // count * kRowsLine elements (the row's [nch][count][64] at its start)
  static __host__ __device__ constexpr int base_of(int o) {
    int b = 0;
    for (int p = 0; p < o; ++p) b += Pl::ops[p].count * kRowsLine;
    return b;
  }
  // every value has a copy, every copy of a neighbour row is that value's
  static __host__ __device__ constexpr bool consistent() {
    int lines = 0;
    for (int o = 0; o < Pl::NOPS; ++o) {
      lines += Pl::ops[o].count;
      if (Pl::map_count[Pl::ops[o].map] != Pl::ops[o].count) return false;
      if (Pl::map_stride[Pl::ops[o].map] != Pl::ops[o].stride) return false;
    }
    if (lines != L::Q) return false;
    if (Pl::ops[1].count != (L::Q - 1) / 2 || Pl::ops[1].stride != 2) return false;
    for (int i = 1; i < L::Q; i += 2) {
      const int o = op_of(i + 1);
      if (o < 2) return false;
      if (Pl::ops[o].dy != L::cy[i] || Pl::ops[o].dz != L::cz[i]) return false;
    }
    return true;
  }
};
static_assert(RowSlots<D3Q27>::consistent(), "row copy plan does not cover D3Q27");
static_assert(RowSlots<D2Q9>::consistent(), "row copy plan does not cover D2Q9");

template <class L>
struct RowMaps {
  CUtensorMap m[RowPlan<L>::NMAPS];
};

template <class L, int ST>
struct RowsCfg {
  using E = typename WordOps<ST>::E;
  static constexpr int STAGE_BYTES = L::Q * kRowsLine * (int)sizeof(E);
  static constexpr int SMEM = kRowsStages * STAGE_BYTES + 64;  // + barriers, counters
  static __host__ __device__ int row_bytes(int nch) { return L::Q * nch * kChunk * (int)sizeof(E); }
};

// ------------------------------------------------------------- primitives
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, int bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, int parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of a barrier; false if the limit passed.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, int parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > kRowsWaitCycles) return false;
  }
}
// One copy: the box of `map` at (x 0, direction q, chunk c), into dst.
__device__ __forceinline__ void tma_load_box(uint32_t dst, const CUtensorMap* map, int q, int c,
                                             uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(dst),
      "l"(map), "r"(0), "r"(q), "r"(c), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_store_box(const CUtensorMap* map, int q, int c, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(map),
               "r"(0), "r"(q), "r"(c), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// First chunk index (tensor coordinate) of padded row (py, pz).
__device__ __forceinline__ int row_chunk(const Geo& g, int py, int pz) {
  return (pz * g.sy + py) * g.nch;
}

// Interior row cursor: row r = (yi, zi), advanced by the grid's CTA count.
struct RowCursor {
  long long r;
  int yi, zi;
  __device__ __forceinline__ void start(long long r0, int ny) {
    r = r0;
    yi = (int)(r0 % ny);
    zi = (int)(r0 / ny);
  }
  __device__ __forceinline__ void advance(long long dr, int dy, int dz, int ny) {
    r += dr;
    yi += dy;
    if (yi >= ny) { yi -= ny; ++zi; }
    zi += dz;
  }
};

// The copies of one row by the calling thread.  LOAD: global -> stage
// (completion on `bar`, whose expected bytes the caller has set); else
// stage -> global, in one bulk group of this thread.
template <class L, int ST, bool LOAD>
__device__ __forceinline__ void rows_copy(const Geo& g, const RowMaps<L>& maps, int P,
                                          const RowCursor& rc, uint32_t stage, uint32_t bar) {
  using Pl = RowPlan<L>;
  using E = typename WordOps<ST>::E;
  const int py = rc.yi + g.hy, pz = rc.zi + g.hz;
  static_for<0, Pl::NOPS>([&](auto O) {
    constexpr int o = decltype(O)::value;
    constexpr RowOp op = Pl::ops[o];
    int ry = py + op.dy, rz = pz + op.dz;
    if constexpr (op.dy != 0) {
      if (ry < 0) ry += g.ny; else if (ry >= g.sy) ry -= g.ny;
    }
    if constexpr (op.dz != 0) {
      if (rz < 0) rz += g.nz; else if (rz >= g.sz) rz -= g.nz;
    }
    const int q = op.q0 + op.sgn * P;
    const uint32_t dst = stage + (uint32_t)(RowSlots<L>::base_of(o) * (int)sizeof(E));
    if constexpr (LOAD) tma_load_box(dst, &maps.m[op.map], q, row_chunk(g, ry, rz), bar);
    else tma_store_box(&maps.m[op.map], q, row_chunk(g, ry, rz), dst);
  });
  if constexpr (!LOAD) bulk_commit();
}

// BGK/TRT keep more values live than the moment operators (as in the paired
// kernel): let them use more registers at fewer resident CTAs.
template <int OP, int ST>
constexpr int rows_min_blocks() {
  return (OP == 1 || OP == 2 || ST == kF64) ? 1 : 4;
}

// Rows stream through a ring of kRowsStages stage buffers; stage s holds
// rows j = s, s + kRowsStages, ... of this CTA.  There is no CTA-wide
// barrier per row: each warp, when done with row j, counts itself in
// done[s]; the last warp to finish moves the row (stores it, waits until the
// stores have read the stage, then loads row j + kRowsStages into it).
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE>
__global__ void __launch_bounds__(kRowsMaxWarps * 32, rows_min_blocks<OP, ST>())
step_rows(StepArgs a, const __grid_constant__ RowMaps<L> maps) {
  using WO = WordOps<ST>;
  using W = typename WO::W;
  using H = typename WO::H;
  using E = typename WO::E;
  using V = typename WO::V;
  using S = typename Lanes<V>::S;
  using Cfg = RowsCfg<L, ST>;
  using Pl = RowPlan<L>;
  using Sl = RowSlots<L>;
  using XW = XWord<ST>;
  constexpr int Q = L::Q;
  const Geo& g = a.g;

  extern __shared__ __align__(128) unsigned char rows_smem[];
  const int lane = threadIdx.x & 31;
  const int k = threadIdx.x >> 5;  // chunk of the row
  const int nw = blockDim.x >> 5;  // == nch
  const int P = a.parity;
  const long long nrows = (long long)g.ny * g.nz;
  const int rbytes = Cfg::row_bytes(g.nch);
  uint64_t* bars = reinterpret_cast<uint64_t*>(rows_smem + kRowsStages * Cfg::STAGE_BYTES);
  int* done = reinterpret_cast<int*>(bars + kRowsStages);  // warps finished with the stage's row
  int* issued = done + kRowsStages;                        // loads issued into the stage
  const uint32_t stage0 = smem_addr(rows_smem);
  const uint32_t bar0 = smem_addr(bars);
  const int dyr = (int)(gridDim.x % g.ny), dzr = (int)(gridDim.x / g.ny);

  RowCursor cur;
  cur.start(blockIdx.x, g.ny);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kRowsStages; ++s) {
      mbar_init(bar0 + 8 * s, 1);
      done[s] = 0;
      issued[s] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    // prologue: this CTA's first kRowsStages rows in flight
    RowCursor c = cur;
    for (int s = 0; s < kRowsStages && c.r < nrows; ++s) {
      mbar_expect_tx(bar0 + 8 * s, rbytes);
      rows_copy<L, ST, true>(g, maps, P, c, stage0 + s * Cfg::STAGE_BYTES, bar0 + 8 * s);
      issued[s] += 1;
      c.advance(gridDim.x, dyr, dzr, g.ny);
    }
  }
  __syncthreads();

  // Per-lane element offsets of an x position inside a copy's block of
  // `count` lines ([chunk][count][64]): (x >> 6) * count * 64 + (x & 63).
  // The pair's word at x0, the words at x0 + 2 and x0 - 2 and the element
  // at x0 - 1 (periodic wrap), for the block shapes the plan uses.
  // A lane past the end of a partial last chunk (x0 >= nx) takes lane 0's
  // positions, so its shared-memory reads stay inside the row, and counts as
  // solid, so it stores nothing.
  const bool lane_ok = k * kChunk + 2 * lane < g.nx;
  const int x0 = lane_ok ? k * kChunk + 2 * lane : 0;
  const int xn = (x0 + 2 == g.nx) ? 0 : x0 + 2;
  const int xm = (x0 == 0) ? g.nx - 2 : x0 - 2;
  const int xe = (x0 == 0) ? g.nx - 1 : x0 - 1;
  auto posc = [](int x, int c) { return (x >> 6) * c * kChunk + (x & 63); };
  const int p0_1 = x0, pn_1 = xn, pm_1 = xm, pe_1 = xe;
  const int p0_2 = posc(x0, 2), pn_2 = posc(xn, 2), pm_2 = posc(xm, 2), pe_2 = posc(xe, 2);
  constexpr int COWN = Pl::ops[1].count;
  const int p0_own = posc(x0, COWN);
  const CollideParams<S> prm{(S)a.omega, (S)a.omega2, (S)a.fx, (S)a.fy, (S)a.fz};

  RowCursor ahead = cur;  // row j + kRowsStages, the next one for this stage
  for (int t = 0; t < kRowsStages; ++t) ahead.advance(gridDim.x, dyr, dzr, g.ny);
  bool failed = false;
  for (int j = 0; cur.r < nrows; ++j) {
    const int s = j % kRowsStages;
    if (!mbar_wait_bounded(bar0 + 8 * s, (j / kRowsStages) & 1)) {
      failed = true;
      break;
    }
    E* sl = reinterpret_cast<E*>(rows_smem + s * Cfg::STAGE_BYTES);

    // ---- the pair's 27 values from the shared blocks
    W w[Q];
    w[0] = *reinterpret_cast<const W*>(sl + Sl::base_of(0) + p0_1);
    static_for<1, Q, 2>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::cx[i];
      constexpr int ro = Sl::op_of(i + 1);
      constexpr int rc = Pl::ops[ro].count;
      static_assert(rc == 1 || rc == 2, "remote copies hold one or two lines");
      const E* ol = sl + Sl::base_of(1) + Sl::j_of(i) * kChunk;
      const E* rl = sl + Sl::base_of(ro) + Sl::j_of(i + 1) * kChunk;
      const int r0 = rc == 1 ? p0_1 : p0_2;
      w[i] = *reinterpret_cast<const W*>(ol + p0_own);
      if constexpr (cx == 0) {
        w[i + 1] = *reinterpret_cast<const W*>(rl + r0);
      } else if constexpr (cx > 0) {
        // elements (x0 + 1, x0 + 2)
        const int rn = rc == 1 ? pn_1 : pn_2;
        w[i + 1] = XW::join(*reinterpret_cast<const W*>(rl + r0), *reinterpret_cast<const W*>(rl + rn));
      } else {
        // elements (x0 - 1, x0)
        const int rm = rc == 1 ? pm_1 : pm_2;
        w[i + 1] = XW::join(*reinterpret_cast<const W*>(rl + rm), *reinterpret_cast<const W*>(rl + r0));
      }
    });

    bool solid0 = !lane_ok, solid1 = !lane_ok;
    if (a.flags) {
      const uint16_t fl = *reinterpret_cast<const uint16_t*>(
          a.flags + ((long long)(cur.zi + g.hz) * g.sy + (cur.yi + g.hy)) * g.sx + x0);
      solid0 = solid0 || (fl & 0xffu) != 0;
      solid1 = solid1 || (fl >> 8) != 0;
    }
    Macro<V> m;
    if constexpr (OP != 0) {
      V f[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) f[q] = WO::unpack(w[q]);
      if constexpr (FORCE) {  // the force per node of the pair (Boussinesq)
        CollideParams<S, V> pv{prm.omega, prm.omega2, bc<V>(prm.fx), bc<V>(prm.fy), bc<V>(prm.fz)};
        if (a.temp) {
          const S* T = reinterpret_cast<const S*>(a.temp);
          const size_t kk = ((size_t)cur.zi * g.ny + cur.yi) * g.nx + x0;
          buoyant_force<V>(a, pack2v(load_pair2(T, kk)), pv.fx, pv.fy, pv.fz);
        }
        m = collide<L, OP, EQ, SH, FORCE>(f, pv);
      } else {
        m = collide<L, OP, EQ, SH, FORCE>(f, prm);
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) w[q] = WO::pack(f[q]);
    } else {  // pure streaming reports rest: rho 1, u 0 (the no-collision mock)
      m.dens = m.rho = bc<V>(1);
      m.ux = m.uy = m.uz = bc<V>(0);
    }

    // ---- write back in place: f_{i+1}' to the own slot, f_i' to the
    // remote slot; solid / excluded nodes leave their slots as read
    // (halfway bounce-back, EsotericPull.hpp:27-33).  Each slot belongs to
    // one lane, so lanes never write what another lane still reads.
    const bool any_solid = __any_sync(0xffffffffu, solid0 || solid1);
    auto put = [&](E* at, W v) {  // the pair's word
      if (!any_solid) {
        *reinterpret_cast<W*>(at) = v;
      } else {
        if (!solid0) *reinterpret_cast<H*>(at) = WO::lo(v);
        if (!solid1) *reinterpret_cast<H*>(at + 1) = WO::hi(v);
      }
    };
    put(sl + Sl::base_of(0) + p0_1, w[0]);
    static_for<1, Q, 2>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::cx[i];
      constexpr int ro = Sl::op_of(i + 1);
      constexpr int rc = Pl::ops[ro].count;
      E* ol = sl + Sl::base_of(1) + Sl::j_of(i) * kChunk;
      E* rl = sl + Sl::base_of(ro) + Sl::j_of(i + 1) * kChunk;
      const int r0 = rc == 1 ? p0_1 : p0_2;
      put(ol + p0_own, w[i + 1]);
      if constexpr (cx == 0) {
        put(rl + r0, w[i]);
      } else if constexpr (cx > 0) {
        // elements x0 + 1 (inside the pair's word) and x0 + 2
        const int rn = rc == 1 ? pn_1 : pn_2;
        if (!solid0) *reinterpret_cast<H*>(rl + r0 + 1) = WO::lo(w[i]);
        if (!solid1) *reinterpret_cast<H*>(rl + rn) = WO::hi(w[i]);
      } else {
        // elements x0 - 1 and x0
        const int re = rc == 1 ? pe_1 : pe_2;
        if (!solid0) *reinterpret_cast<H*>(rl + re) = WO::lo(w[i]);
        if (!solid1) *reinterpret_cast<H*>(rl + r0) = WO::hi(w[i]);
      }
    });

    {
      if (a.rho)
        store_macro_pair<S>(a, ((size_t)cur.zi * g.ny + cur.yi) * g.nx + x0, m, solid0, solid1);
    }

    // ---- row done for this warp: make its writes visible to the copy
    // engine, count it; the last warp moves the row
    fence_async_smem();
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      const int before = atomicAdd(&done[s], 1);
      if (before == nw - 1) {
        atomicExch(&done[s], 0);
        __threadfence_block();
        rows_copy<L, ST, false>(g, maps, P, cur, stage0 + s * Cfg::STAGE_BYTES, 0);
        if (ahead.r < nrows) {
          bulk_wait_read<0>();  // this thread's stores no longer read the stage
          mbar_expect_tx(bar0 + 8 * s, rbytes);
          rows_copy<L, ST, true>(g, maps, P, ahead, stage0 + s * Cfg::STAGE_BYTES, bar0 + 8 * s);
          issued[s] += 1;
        }
      }
    }
    cur.advance(gridDim.x, dyr, dzr, g.ny);
    ahead.advance(gridDim.x, dyr, dzr, g.ny);
  }

  if (failed && lane == 0 && a.err) atomicExch(a.err, 1);
  if (lane == 0) bulk_wait_all();  // this thread's stores have landed
  // every warp is out of the loop (all waits are bounded); after a failure,
  // loads that were issued but never consumed land (bounded again) before
  // the CTA's shared memory is released
  if (__syncthreads_or(failed) && threadIdx.x == 0) {
    for (int s = 0; s < kRowsStages; ++s)
      if (issued[s] > 0) mbar_wait_bounded(bar0 + 8 * s, (issued[s] - 1) & 1);
  }
}

}  // namespace m3lb
