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
// A CTA is nch update warps (warp k takes chunk k of the row; nx even,
// periodic x; lanes past nx in a partial last chunk store nothing) and, for
// rows of 3 chunks or more, one copy warp that moves the rows through a
// ring of kRowsStages stages: it loads the rows ahead, and once every update
// warp has marked a row done it stores the row and reloads the stage.  Rows
// of 1-2 chunks have no copy warp: the update warp that finishes a row last
// moves it, through a ring of 3 stages, so twice as many CTAs are resident.
// The stage is sized for LW chunks (2, 3, 4 or 8), the smallest that holds
// the row, so short rows keep more CTAs resident.
//
// Waits are bounded: past the limit a warp records a status in
// StepArgs::err and raises the CTA's abort flag, the copies in flight
// finish (bounded again) and the CTA leaves; the host reports the status at
// the next m3lb_sync.
#pragma once
#include <cuda.h>

#include "lbm_stream.cuh"

namespace m3lb {

constexpr int kRowsStages = 4;
constexpr int kRowsMaxChunks = 8;  // nch <= 8 (nx <= 512)
constexpr long long kRowsWaitCycles = 4000000000LL;  // ~2 s at 2 GHz
constexpr uint32_t kRowsSuspendNs = 20000;            // longest suspension per barrier test
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
  // first shared element of a copy's block in a stage of LW-chunk lines:
  // blocks in op order, each count * LW * 64 elements (the row's
  // [nch][count][64] at its start)
  static __host__ __device__ constexpr int base_of(int o, int lw) {
    int b = 0;
    for (int p = 0; p < o; ++p) b += Pl::ops[p].count * lw * kChunk;
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

// One lattice of a batched launch (the serving loop): its tensor maps, step
// arguments, first row in the launch's numbering and time at the start of
// the round.
template <class L>
struct RowItem {
  RowMaps<L> maps;
  StepArgs a;
  long long first_row;
  long long t0;     // the lattice's time at step 0 of the launch
  long long t_end;  // its last time: steps from t_end on leave its rows alone
};
// A batched launch: items first_item .. first_item + n_items of the table
// (one operator, one row width), n_rows rows in all.
struct RowBatch {
  int first_item, n_items;
  long long n_rows;
};

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

// What the copies of a row need of its lattice, held in registers (read
// through a pointer into global memory, the fields would be reloaded after
// every copy, each of which clobbers memory).
struct RowGeo {
  int ny, nz, sy, sz, hy, hz, nch;
  __device__ __forceinline__ static RowGeo of(const Geo& g) {
    return RowGeo{g.ny, g.nz, g.sy, g.sz, g.hy, g.hz, g.nch};
  }
};

// A row in a stage: its lattice's copy geometry, maps and parity, its (y, z)
// there, and (batched launches) its item, -1 for a lattice sitting out.
template <class L>
struct RowHeld {
  RowGeo g;
  const RowMaps<L>* maps;
  int parity, yi, zi, item;
};

// Shared memory of a CTA: NS stages of Q lines of LW chunks, then the
// barriers (full[s]: the stage's loads landed; empty[s]: every update warp
// is done with the stage's row), the abort flag, per stage the row's item
// (batched launches) or whether it has a non-fluid node, and per stage the
// RowHeld of its row.  Without a copy warp the empty barriers' words hold,
// per stage, the count of update warps done with the row and the count of
// loads issued into it.
template <class L, int ST, int LW, int NS = kRowsStages>
struct RowsCfg {
  using E = typename WordOps<ST>::E;
  static constexpr int STAGE_BYTES = L::Q * LW * kChunk * (int)sizeof(E);
  static constexpr int HELD_OFF = (NS * STAGE_BYTES + 2 * NS * 8 + 4 + 4 * NS + 15) / 16 * 16;
  static constexpr int SMEM = HELD_OFF + NS * (int)sizeof(RowHeld<L>);
  static __host__ __device__ int row_bytes(int nch) { return L::Q * nch * kChunk * (int)sizeof(E); }
};
// Line width (chunks per stage line) for a row of nch chunks: 2, 3, 4 or 8.
__host__ __device__ constexpr int rows_lw(int nch) {
  return nch <= 2 ? 2 : (nch == 3 ? 3 : (nch <= 4 ? 4 : 8));
}

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
// Whether phase `parity` of a barrier has completed, without waiting.
__device__ __forceinline__ bool mbar_test(uint32_t bar, int parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
  return ok != 0;
}
// The same test, letting the hardware suspend the warp until the phase
// completes or kRowsSuspendNs pass, so a waiting warp issues no spin loop.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t bar, int parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(bar), "r"(parity), "r"(kRowsSuspendNs) : "memory");
  return ok != 0;
}
// Bounded wait for phase `parity` of a barrier: true once the phase has
// completed, false when `limit` clock cycles passed first (after a first
// test that never waits).
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, int parity,
                                                  long long limit = kRowsWaitCycles) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (clock64() - t0 < limit)
    if (mbar_try_wait_sleep(bar, parity)) return true;
  return false;
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

// The copies of one row (interior row yi, zi).  LOAD: global -> stage
// (completion on `bar`, whose expected bytes the caller has set); else stage
// -> global, in one bulk group of the issuing thread.  Every calling thread
// computes the coordinates; only where `issue` holds are the copies issued.
// A whole warp calling with the same arguments keeps the arithmetic on
// warp-uniform values, and one branch around the copies leaves them
// straight-line: the copy thread's latency per row is on the path that
// recycles a stage.
template <class L, int ST, int LW, bool LOAD>
__device__ __forceinline__ void rows_copy(const RowGeo g, const RowMaps<L>* maps, int P, int yi,
                                          int zi, uint32_t stage, uint32_t bar, bool issue) {
  using Pl = RowPlan<L>;
  using E = typename WordOps<ST>::E;
  const int py = yi + g.hy, pz = zi + g.hz;
  int qs[Pl::NOPS], cs[Pl::NOPS];
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
    qs[o] = op.q0 + op.sgn * P;
    cs[o] = (rz * g.sy + ry) * g.nch;
  });
  if (!issue) return;
  static_for<0, Pl::NOPS>([&](auto O) {
    constexpr int o = decltype(O)::value;
    constexpr RowOp op = Pl::ops[o];
    const uint32_t dst = stage + (uint32_t)(RowSlots<L>::base_of(o, LW) * (int)sizeof(E));
    if constexpr (LOAD) tma_load_box(dst, &maps->m[op.map], qs[o], cs[o], bar);
    else tma_store_box(&maps->m[op.map], qs[o], cs[o], dst);
  });
  if constexpr (!LOAD) bulk_commit();
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool flag_set(const int* f) {
  return *reinterpret_cast<const volatile int*>(f) != 0;
}
// A bounded barrier wait that also gives up once the CTA's abort flag is set.
__device__ __forceinline__ bool rows_wait(uint32_t bar, int parity, long long limit,
                                          const int* abort_flag) {
  if (mbar_test(bar, parity)) return true;
  const long long t0 = clock64();
  while (clock64() - t0 < limit) {
    if (mbar_try_wait_sleep(bar, parity)) return true;
    if (flag_set(abort_flag)) return false;
  }
  return false;
}

// Resident CTAs per SM the launch bounds ask for.  With a copy warp (rows of
// 3 to 8 chunks, and the batched kernel): the moment operators fit their
// registers at the occupancy the stage size allows (16-bit storage, LW 2: 8
// CTAs of 27.6 KB fit, registers allow 6; LW 3: 5 CTAs of 41.5 KB; LW 4: 4
// CTAs of 55 KB; LW 8: 2 of 110 KB); BGK/TRT keep more values live (as in
// the paired kernel) and take their registers at fewer resident CTAs.  Without a copy warp (the
// single-lattice kernel's rows of up to 4 chunks, 3 stages): 16-bit LW 4
// stages of 41.5 KB fit 5 CTAs of 4 warps, LW 2 stages of 20.8 KB 10 CTAs of
// 2 warps, both at up to 96 registers.
template <int OP, int ST, int LW, bool CW = true>
constexpr int rows_min_blocks() {
  if (ST == kF64) return 1;
  if (!CW) {
    if (ST == kF32) return LW == 2 ? 5 : 2;
    if (OP == 1 || OP == 2) return LW == 2 ? 6 : 3;
    return LW == 2 ? 10 : 5;
  }
  if (OP == 1 || OP == 2) return LW == 2 ? 4 : (LW == 3 ? 3 : (LW == 4 ? 2 : 1));
  if (ST == kF32) return LW <= 3 ? 2 : 1;
  return LW == 2 ? 6 : (LW == 3 ? 5 : (LW == 4 ? 4 : 2));
}
// Stages of the ring: 4 with a copy warp, 3 without (the warp that finishes
// a row last moves it, so a stage is busy only while its row is stored and
// the next one loads).
template <bool CW>
__host__ __device__ constexpr int rows_stages() { return CW ? kRowsStages : 3; }

// The rows a CTA loads, in order (row j of the CTA at its j-th call of
// next()).  BATCH: global row r belongs to the item whose row range holds
// it; the lattice the cursor is in is cached while consecutive rows of the
// CTA (gridDim.x apart) stay in it: its rows [c_first, c_end), copy
// geometry, parity, whether it steps, and the cursor's (y, z) with the grid
// stride's (y, z) parts for an incremental advance.  The item table is
// searched only when the cursor leaves the lattice.
template <class L, bool BATCH>
struct RowLoader {
  RowCursor ld;  // next row to load
  int c_item, c_yi, c_zi, c_dy, c_dz, c_par;
  long long c_first, c_end;
  bool c_live;
  RowGeo c_g;
  int flag;  // with cell flags: the summary of row ld, read one row ahead
  __device__ __forceinline__ static int row_flag(const StepArgs& a, const RowCursor& c,
                                                 long long nrows) {
    if (BATCH || !a.flags || c.r >= nrows) return 0;
    const Geo& g = a.g;
    return a.row_flags ? a.row_flags[(c.zi + g.hz) * g.sy + (c.yi + g.hy)] : 1;
  }
  __device__ __forceinline__ void init(const RowCursor& start, const StepArgs& a, long long nrows) {
    const Geo& g = a.g;
    ld = start;
    flag = row_flag(a, ld, nrows);
    c_item = -1;
    c_yi = c_zi = c_dy = c_dz = c_par = 0;
    c_first = c_end = 0;
    c_live = true;
    c_g = RowGeo::of(g);
  }
  // The RowHeld of row ld (which the caller has checked is < nrows); ld
  // moves to the CTA's next row.
  __device__ __forceinline__ RowHeld<L> next(const StepArgs& a, const RowMaps<L>& maps,
                                             const RowItem<L>* __restrict__ items, int n_items,
                                             int step, int dyr, int dzr, long long nrows) {
    if constexpr (BATCH) {
      const long long r = ld.r;
      if (c_item >= 0 && r >= c_first && r < c_end) {
        c_yi += c_dy;
        if (c_yi >= c_g.ny) { c_yi -= c_g.ny; ++c_zi; }
        c_zi += c_dz;
      } else {
        int lo = 0, hi = n_items - 1;  // last item with first_row <= r
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (items[mid].first_row <= r) lo = mid; else hi = mid - 1;
        }
        const RowItem<L>& it = items[lo];
        c_item = lo;
        c_g = RowGeo::of(it.a.g);
        c_first = it.first_row;
        c_end = c_first + (long long)c_g.ny * c_g.nz;
        c_par = (int)((it.t0 + step) & 1);
        c_live = it.t0 + step < it.t_end;
        const long long local = r - c_first;
        c_yi = (int)(local % c_g.ny);
        c_zi = (int)(local / c_g.ny);
        c_dy = (int)(gridDim.x % (unsigned)c_g.ny);
        c_dz = (int)(gridDim.x / (unsigned)c_g.ny);
      }
      ld.r += gridDim.x;
      // a lattice that has done its steps sits this step out: its row is
      // neither loaded nor stored, the update warps see item -1
      return RowHeld<L>{c_g, &items[c_item].maps, c_par, c_yi, c_zi, c_live ? c_item : -1};
    } else {
      const RowHeld<L> h{RowGeo::of(a.g), &maps, a.parity, ld.yi, ld.zi, 0};
      ld.advance(gridDim.x, dyr, dzr, a.g.ny);
      flag = row_flag(a, ld, nrows);
      return h;
    }
  }
};

// One CTA.  Row j of the CTA sits in stage j % NS; its load completes phase
// (j / NS) & 1 of full[s].
//
// CW (copy warp): warps 0 .. nch-1 update chunk k of each of the CTA's
// rows, warp nch (lane 0) moves them.  The update warps' arrivals on
// empty[s] (one per warp) complete the row's phase there, after which the
// copy warp stores the row, waits until the stores have read the stage, and
// loads row j + NS into it.
//
// Without a copy warp: the nch warps update the rows, and the warp that
// finishes a row last (a per-stage count in shared memory) stores it, waits
// until the stores have read the stage and loads row j + NS into it; every
// other warp goes on to the next row at once.  No warp waits for another
// except through the full barriers, so fewer warps per CTA buy more
// resident CTAs.  The last warps of consecutive rows take turns: the last
// warp of row j + 1 can only finish it after leaving row j's copies, so the
// copies are issued in row order, one thread at a time.  Lane 0 of every
// warp runs its own RowLoader one row after another, so whichever warp
// turns out last holds the cursor of the row to load.
//
// A lattice with cell flags: whoever loads a row also records in the
// stage's slot of `meta` whether the row has a non-fluid node (the per-row
// summary row_flags), and the update warps load the flags of those rows
// only.
//
// BATCH: the rows of many lattices of one operator and one row width (the
// serving loop): global row r belongs to the item whose range holds it
// (items sorted by first_row), each item carrying its own step arguments,
// tensor maps and time.  Whoever loads a row records its item in the
// stage's slot of `meta` and its RowHeld beside it; the update warps read
// the item there and take the lattice's x extent and rates when it changes,
// and the row's RowHeld tells whoever stores it where it goes.  Batched
// lattices are periodic boxes with no cell flags, buoyancy or macroscopic
// output.
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE, int LW, bool CW, bool BATCH>
__device__ __forceinline__ void rows_body(const StepArgs& a, const RowMaps<L>& maps,
                                          const RowItem<L>* __restrict__ items, int n_items,
                                          long long batch_rows, int step) {
  using WO = WordOps<ST>;
  using W = typename WO::W;
  using H = typename WO::H;
  using E = typename WO::E;
  using V = typename WO::V;
  using S = typename Lanes<V>::S;
  constexpr int NS = rows_stages<CW>();
  using Cfg = RowsCfg<L, ST, LW, NS>;
  using Pl = RowPlan<L>;
  using Sl = RowSlots<L>;
  using XW = XWord<ST>;
  using Held = RowHeld<L>;
  constexpr int Q = L::Q;
  const Geo& g = a.g;

  extern __shared__ __align__(128) unsigned char rows_smem[];
  const int lane = threadIdx.x & 31;
  const int k = threadIdx.x >> 5;  // chunk of the row; == nch for the copy warp
  const int nch = BATCH ? items[0].a.g.nch : g.nch;
  const long long nrows = BATCH ? batch_rows : (long long)g.ny * g.nz;
  uint64_t* bars = reinterpret_cast<uint64_t*>(rows_smem + NS * Cfg::STAGE_BYTES);
  int* abort_flag = reinterpret_cast<int*>(bars + 2 * NS);
  int* meta = abort_flag + 1;  // per stage: BATCH the row's item, else whether it has flags
  Held* held = reinterpret_cast<Held*>(rows_smem + Cfg::HELD_OFF);  // per stage (no copy warp)
  // without a copy warp, in the words of the empty barriers: per stage the
  // update warps done with its row, and the loads issued into it
  int* done = reinterpret_cast<int*>(bars + NS);
  int* issued = done + NS;
  const uint32_t stage0 = smem_addr(rows_smem);
  const uint32_t full0 = smem_addr(bars), empty0 = full0 + 8 * NS;
  const int dyr = BATCH ? 0 : (int)(gridDim.x % g.ny), dzr = BATCH ? 0 : (int)(gridDim.x / g.ny);
  const int rbytes = Cfg::row_bytes(nch);
  // Load row `ld` of the loader into stage s (a sitting-out row only
  // completes the stage's phase), record its item or flag summary in meta[s]
  // (published to the update warps by the barrier arrival) and, without a
  // copy warp, its RowHeld in held[s]; returns the RowHeld.
  auto load_row = [&](RowLoader<L, BATCH>& lo, int s, bool issue) -> Held {
    const int flag = lo.flag;
    const Held h = lo.next(a, maps, items, n_items, step, dyr, dzr, nrows);
    if (issue) {
      meta[s] = BATCH ? h.item : flag;
      if constexpr (!CW) held[s] = h;
    }
    if (h.item >= 0) {
      if (issue) mbar_expect_tx(full0 + 8 * s, rbytes);
      rows_copy<L, ST, LW, true>(h.g, h.maps, h.parity, h.yi, h.zi,
                                 stage0 + s * Cfg::STAGE_BYTES, full0 + 8 * s, issue);
    } else if (issue) {
      mbar_arrive(full0 + 8 * s);
    }
    return h;
  };

  RowCursor cur;
  if constexpr (BATCH) cur.r = blockIdx.x;
  else cur.start(blockIdx.x, g.ny);

  // without a copy warp: lane 0 of every warp runs the loader, NS rows
  // ahead of the warp's own row
  RowLoader<L, BATCH> ahead;
  if (!CW && lane == 0) ahead.init(cur, a, nrows);

  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      mbar_init(full0 + 8 * s, 1);
      if constexpr (CW) {
        mbar_init(empty0 + 8 * s, nch);
      } else {
        done[s] = 0;
        issued[s] = 0;
      }
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    if constexpr (!CW) {
      // prologue: the CTA's first NS rows in flight
      for (int s = 0; s < NS && ahead.ld.r < nrows; ++s) {
        load_row(ahead, s, true);
        issued[s] = 1;
      }
    }
  }
  if (!CW && lane == 0 && threadIdx.x != 0) {
    // the other warps' loaders skip the prologue's rows (no copies)
    for (int s = 0; s < NS && ahead.ld.r < nrows; ++s)
      ahead.next(a, maps, items, n_items, step, dyr, dzr, nrows);
  }
  __syncthreads();

  // ------------------------------------------------------------ copy warp
  // The whole warp runs the loop on warp-uniform values; lane 0 issues the
  // copies, the barrier arrivals and the bulk-group waits.
  if (CW && k == nch) {
    const bool l0 = lane == 0;
    Held hs[NS];
    RowLoader<L, BATCH> lo;
    lo.init(cur, a, nrows);
    int nl = 0, nst = 0;  // rows loaded, rows stored
    bool failed = false;
    while (nl < NS && lo.ld.r < nrows) {
      hs[nl] = load_row(lo, nl, l0);
      ++nl;
    }
    while (nst < nl) {
      const int s = nst % NS;
      // lane 0's view of the wait decides for the warp
      const bool ok = __shfl_sync(0xffffffffu,
                                  rows_wait(empty0 + 8 * s, (nst / NS) & 1, kRowsWaitCycles,
                                            abort_flag), 0);
      if (!ok) {
        failed = true;
        break;
      }
      const Held h = hs[s];
      if (h.item >= 0)
        rows_copy<L, ST, LW, false>(h.g, h.maps, h.parity, h.yi, h.zi,
                                    stage0 + s * Cfg::STAGE_BYTES, 0, l0);
      ++nst;
      if (lo.ld.r < nrows) {
        if (l0) bulk_wait_read<0>();  // the stores no longer read the stage
        __syncwarp();
        hs[s] = load_row(lo, s, l0);
        ++nl;
      }
    }
    if (l0) {
      bulk_wait_all();  // every store has landed
      if (failed || flag_set(abort_flag)) {
        atomicExch(abort_flag, 1);
        if (a.err) atomicExch(a.err, 1);
        // loads issued for rows not stored yet land before the CTA's shared
        // memory is released (bounded; the abort flag is not consulted here)
        for (int r = nst; r < nl; ++r)
          mbar_wait_bounded(full0 + 8 * (r % NS), (r / NS) & 1);
      }
    }
    return;
  }

  // ---------------------------------------------------------- update warps
  // Per-lane element offsets of an x position inside a copy's block of
  // `count` lines ([chunk][count][64]): (x >> 6) * count * 64 + (x & 63).
  // The pair's word at x0, the words at x0 + 2 and x0 - 2 and the element
  // at x0 - 1 (periodic wrap), for the block shapes the plan uses.
  // A lane past the end of a partial last chunk (x0 >= nx) takes lane 0's
  // positions, so its shared-memory reads stay inside the row, and counts as
  // solid, so it stores nothing.
  auto posc = [](int x, int c) { return (x >> 6) * c * kChunk + (x & 63); };
  constexpr int COWN = Pl::ops[1].count;
  bool lane_ok;
  int x0, p0_1, pn_1, pm_1, pe_1, p0_2, pn_2, pm_2, pe_2, p0_own;
  CollideParams<S> prm;
  auto set_lattice = [&](const StepArgs& la) {
    const int nx = la.g.nx;
    lane_ok = k * kChunk + 2 * lane < nx;
    x0 = lane_ok ? k * kChunk + 2 * lane : 0;
    const int xn = (x0 + 2 == nx) ? 0 : x0 + 2;
    const int xm = (x0 == 0) ? nx - 2 : x0 - 2;
    const int xe = (x0 == 0) ? nx - 1 : x0 - 1;
    p0_1 = x0; pn_1 = xn; pm_1 = xm; pe_1 = xe;
    p0_2 = posc(x0, 2); pn_2 = posc(xn, 2); pm_2 = posc(xm, 2); pe_2 = posc(xe, 2);
    p0_own = posc(x0, COWN);
    prm = CollideParams<S>{(S)la.omega, (S)la.omega2, (S)la.fx, (S)la.fy, (S)la.fz};
  };
  int cur_item = -1;
  if constexpr (!BATCH) set_lattice(a);
  const long long consume_limit = BATCH ? kRowsWaitCycles
                                        : (a.wait_cycles > 0 ? a.wait_cycles : kRowsWaitCycles);
  // ---- row done for this warp: its shared-memory writes become visible to
  // the copy engine; then one arrival on the stage's empty barrier, or (no
  // copy warp) the count of warps done, the last of which stores the row
  // and loads row j + NS into the stage.  Lane 0 of every warp moves its
  // loader on by one row either way.
  auto row_done = [&](int s) {
    fence_async_smem();
    __syncwarp();
    if (lane != 0) return;
    if constexpr (CW) {
      mbar_arrive(empty0 + 8 * s);
    } else {
      __threadfence_block();
      if (atomicAdd(&done[s], 1) == nch - 1) {
        // every update warp is done with the row: no warp touches the count
        // again before the stage's next load lands
        done[s] = 0;
        __threadfence_block();
        const Held h = held[s];
        if (h.item >= 0)
          rows_copy<L, ST, LW, false>(h.g, h.maps, h.parity, h.yi, h.zi,
                                      stage0 + s * Cfg::STAGE_BYTES, 0, true);
        if (ahead.ld.r < nrows) {
          bulk_wait_read<0>();  // this thread's stores no longer read the stage
          load_row(ahead, s, true);
          issued[s] += 1;
        }
      } else if (ahead.ld.r < nrows) {
        ahead.next(a, maps, items, n_items, step, dyr, dzr, nrows);
      }
    }
  };

  bool failed = false;
  for (int j = 0; cur.r < nrows; ++j) {
    const int s = j % NS;
    if (!rows_wait(full0 + 8 * s, (j / NS) & 1, consume_limit, abort_flag)) {
      failed = true;
      break;
    }
    E* sl = reinterpret_cast<E*>(rows_smem + s * Cfg::STAGE_BYTES);
    if constexpr (BATCH) {
      const int item = meta[s];
      if (item < 0) {  // a finished lattice's row: nothing to update
        row_done(s);
        cur.r += gridDim.x;
        continue;
      }
      if (item != cur_item) {
        cur_item = item;
        set_lattice(items[item].a);
      }
    }

    // ---- the pair's 27 values from the shared blocks.  An x-shifted remote
    // pair straddles two words: the collision operators decode it from both
    // directly; pure streaming joins the two halves into one word.
    W w[Q];
    V f[Q];
    auto rd = [](const E* at) { return *reinterpret_cast<const W*>(at); };
    w[0] = rd(sl + Sl::base_of(0, LW) + p0_1);
    static_for<1, Q, 2>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::cx[i];
      constexpr int ro = Sl::op_of(i + 1);
      constexpr int rc = Pl::ops[ro].count;
      static_assert(rc == 1 || rc == 2, "remote copies hold one or two lines");
      const E* ol = sl + Sl::base_of(1, LW) + Sl::j_of(i) * kChunk;
      const E* rl = sl + Sl::base_of(ro, LW) + Sl::j_of(i + 1) * kChunk;
      const int r0 = rc == 1 ? p0_1 : p0_2;
      w[i] = rd(ol + p0_own);
      if constexpr (cx == 0) {
        w[i + 1] = rd(rl + r0);
      } else {
        // elements (x0 + 1, x0 + 2), or (x0 - 1, x0)
        const W a0 = cx > 0 ? rd(rl + r0) : rd(rl + (rc == 1 ? pm_1 : pm_2));
        const W b0 = cx > 0 ? rd(rl + (rc == 1 ? pn_1 : pn_2)) : rd(rl + r0);
        if constexpr (OP == 0) w[i + 1] = XW::join(a0, b0);
        else f[i + 1] = WO::unpack_join(a0, b0);
      }
    });

    bool solid0 = !lane_ok, solid1 = !lane_ok;
    if (!BATCH && a.flags && meta[s]) {
      const uint16_t fl = *reinterpret_cast<const uint16_t*>(
          a.flags + ((long long)(cur.zi + g.hz) * g.sy + (cur.yi + g.hy)) * g.sx + x0);
      solid0 = solid0 || (fl & 0xffu) != 0;
      solid1 = solid1 || (fl >> 8) != 0;
    }
    Macro<V> m;
    if constexpr (OP != 0) {
      static_for<0, Q>([&](auto QQ) {
        constexpr int q = decltype(QQ)::value;
        if constexpr (q == 0 || (q % 2) == 1 || L::cx[q - 1] == 0) f[q] = WO::unpack(w[q]);
      });
      if constexpr (FORCE) {  // the force per node of the pair (Boussinesq)
        CollideParams<S, V> pv{prm.omega, prm.omega2, bc<V>(prm.fx), bc<V>(prm.fy), bc<V>(prm.fz)};
        if (!BATCH && a.temp) {
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
    // one lane, so lanes never write what another lane still reads.  A warp
    // with no solid lane (the common case) stores without per-node tests.
    auto store_all = [&](auto GUARD) {
      constexpr bool G = decltype(GUARD)::value;
      auto put = [&](E* at, W v) {  // the pair's word
        if constexpr (!G) {
          *reinterpret_cast<W*>(at) = v;
        } else {
          if (!solid0) *reinterpret_cast<H*>(at) = WO::lo(v);
          if (!solid1) *reinterpret_cast<H*>(at + 1) = WO::hi(v);
        }
      };
      auto put_h = [&](E* at, H v, bool solid) {  // one node's element
        if (!G || !solid) *reinterpret_cast<H*>(at) = v;
      };
      put(sl + Sl::base_of(0, LW) + p0_1, w[0]);
      static_for<1, Q, 2>([&](auto I) {
        constexpr int i = decltype(I)::value;
        constexpr int cx = L::cx[i];
        constexpr int ro = Sl::op_of(i + 1);
        constexpr int rc = Pl::ops[ro].count;
        E* ol = sl + Sl::base_of(1, LW) + Sl::j_of(i) * kChunk;
        E* rl = sl + Sl::base_of(ro, LW) + Sl::j_of(i + 1) * kChunk;
        const int r0 = rc == 1 ? p0_1 : p0_2;
        put(ol + p0_own, w[i + 1]);
        if constexpr (cx == 0) {
          put(rl + r0, w[i]);
        } else if constexpr (cx > 0) {
          // elements x0 + 1 (inside the pair's word) and x0 + 2
          put_h(rl + r0 + 1, WO::lo(w[i]), solid0);
          put_h(rl + (rc == 1 ? pn_1 : pn_2), WO::hi(w[i]), solid1);
        } else {
          // elements x0 - 1 and x0
          put_h(rl + (rc == 1 ? pe_1 : pe_2), WO::lo(w[i]), solid0);
          put_h(rl + r0, WO::hi(w[i]), solid1);
        }
      });
    };
    if (__any_sync(0xffffffffu, solid0 || solid1)) store_all(IC<1>{});
    else store_all(IC<0>{});

    if (!BATCH && a.rho)
      store_macro_pair<S>(a, ((size_t)cur.zi * g.ny + cur.yi) * g.nx + x0, m, solid0, solid1);

    row_done(s);
    if constexpr (BATCH) cur.r += gridDim.x;
    else cur.advance(gridDim.x, dyr, dzr, g.ny);
  }
  if (failed && lane == 0) {
    atomicExch(abort_flag, 1);
    if (a.err) atomicExch(a.err, 1);
  }
  if constexpr (!CW) {
    if (lane == 0) bulk_wait_all();  // this thread's stores have landed
    // every warp is out of the loop (all waits are bounded); after a
    // failure, loads issued but never consumed land (bounded again, the
    // abort flag not consulted) before the CTA's shared memory is released
    if (__syncthreads_or(failed || flag_set(abort_flag)) && threadIdx.x == 0) {
      for (int s = 0; s < NS; ++s)
        if (issued[s] > 0) mbar_wait_bounded(full0 + 8 * s, (issued[s] - 1) & 1);
    }
  }
}

// The single-lattice row kernel; CW: with a copy warp (LW 8), else the
// update warps move the rows themselves (LW 2, 4).
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE, int LW, bool CW>
__global__ void __launch_bounds__((LW + (CW ? 1 : 0)) * 32, rows_min_blocks<OP, ST, LW, CW>())
step_rows(StepArgs a, const __grid_constant__ RowMaps<L> maps) {
  rows_body<L, ST, OP, EQ, SH, FORCE, LW, CW, false>(a, maps, nullptr, 0, 0, 0);
}

// One time step of the rows of a batch (launch descriptor read from device
// memory, so a captured launch serves any resident set of its group); with
// a copy warp for rows of 3 chunks or more, as the single-lattice kernel.
template <class L, int ST, int OP, int EQ, int LW>
__global__ void __launch_bounds__((LW + (LW != 2 ? 1 : 0)) * 32,
                                  rows_min_blocks<OP, ST, LW, (LW != 2)>())
batch_rows(const RowItem<L>* __restrict__ items, const RowBatch* __restrict__ desc, int step) {
  const RowBatch d = *desc;
  if (d.n_items <= 0 || d.n_rows <= 0) return;
  const RowItem<L>* it = items + d.first_item;
  rows_body<L, ST, OP, EQ, true, false, LW, (LW != 2), true>(it[0].a, it[0].maps, it, d.n_items,
                                                             d.n_rows, step);
}

}  // namespace m3lb
