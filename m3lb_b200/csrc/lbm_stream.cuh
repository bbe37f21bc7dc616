// Persistent, software-pipelined step kernel for periodic-x lattices on
// sm_100a.
//
// Same update as step_pairs (lbm_kernels.cuh): one warp per 64-node chunk,
// two x-adjacent nodes per lane, paired FP32 arithmetic, ±1 x shift by warp
// shuffle.  What changes is the schedule:
//   * the grid is persistent (the resident blocks of every SM) and warp w
//     takes chunks w, w + T, w + 2T, ... (T warps in the grid), advancing its
//     row/chunk cursor by additions instead of the divisions of step_pairs;
//     at any moment the grid works on one contiguous window of the lattice;
//   * every warp owns a ring of STAGES chunk buffers in shared memory and
//     keeps the words of its next STAGES - 1 chunks in flight with
//     asynchronous global->shared copies (cp.async) while it collides the
//     current one, so DRAM reads stay outstanding without holding registers
//     (the collision needs all of them).
// Each lane copies, and later reads, only its own words (word q of lane l
// sits at stage[q * 32 + l]); the chunk-edge word of a shifted direction is
// copied by the one lane that needs it.  So completion of the lane's own copy
// groups (cp.async.wait_group) is the only synchronisation.
// Race freedom in global memory is Esoteric Pull's own: every slot is read and
// written by the same node, so the copies of later chunks never see a slot
// that an earlier chunk's stores change.
#pragma once
#include "lbm_kernels.cuh"

namespace m3lb {

// Index of an odd direction among those with c_x != 0 (each has a chunk-edge
// word in the stage buffer), or -1.
template <class L>
__host__ __device__ constexpr int xshift_index(int i) {
  int k = 0;
  for (int j = 1; j < L::Q; j += 2) {
    if (j == i) return L::cx[j] != 0 ? k : -1;
    if (L::cx[j] != 0) ++k;
  }
  return -1;
}
template <class L>
__host__ __device__ constexpr int xshift_count() {
  int k = 0;
  for (int j = 1; j < L::Q; j += 2) k += L::cx[j] != 0;
  return k;
}

// Word recombination for the ±1 x shift.  join(a, b) is the word holding
// the hi element of a and the lo element of b.  For 16-bit storage a word is
// one 32-bit register: whole words are shuffled and joined with one byte
// permute.  For wider storage only the element that is used is shuffled.
template <int ST>
struct XWord {
  using WO = WordOps<ST>;
  using W = typename WO::W;
  static constexpr bool kPacked = sizeof(W) == 4;
  static __device__ __forceinline__ W join(W a, W b) {
    if constexpr (kPacked) return __byte_perm(a, b, 0x5432);
    else return WO::make(WO::hi(a), WO::lo(b));
  }
  // word of lane src whose lo element is valid
  static __device__ __forceinline__ W shfl_lo(W w, int src) {
    if constexpr (kPacked) return __shfl_sync(0xffffffffu, w, src);
    else return WO::make(shfl_h(WO::lo(w), src), WO::hi(w));
  }
  // word of lane src whose hi element is valid
  static __device__ __forceinline__ W shfl_hi(W w, int src) {
    if constexpr (kPacked) return __shfl_sync(0xffffffffu, w, src);
    else return WO::make(WO::lo(w), shfl_h(WO::hi(w), src));
  }
};

// Shared-memory ring of the streamed kernel, per warp: STAGES buffers of
// (Q + NX) * 32 words: word q of lane l at [q * 32 + l], then the lane's
// chunk-edge word of x-shifted direction e at [(Q + e) * 32 + l].
template <class L, int ST>
struct StreamCfg {
  using W = typename WordOps<ST>::W;
  static constexpr int WARPS = kPairThreads / 32;
  static constexpr int STAGES = 2;
  static constexpr int NX = xshift_count<L>();
  static constexpr int STAGE_WORDS = (L::Q + NX) * 32;
  static constexpr int WARP_BYTES = STAGES * STAGE_WORDS * (int)sizeof(W);
  static constexpr int SMEM = WARPS * WARP_BYTES;
};

// Chunk cursor: chunk k of interior row (yi, zi), linear index u.
struct Cursor {
  long long u;
  int k, yi, zi;
  __device__ __forceinline__ void start(long long u0, int nch, int ny) {
    u = u0;
    const long long row = u0 / nch;
    k = (int)(u0 - row * nch);
    yi = (int)(row % ny);
    zi = (int)(row / ny);
  }
  // advance by a stride decomposed as (dz planes, dy rows, dk chunks),
  // dk < nch and dy < ny
  __device__ __forceinline__ void advance(long long du, int dk, int dy, int dz, int nch, int ny) {
    u += du;
    k += dk;
    if (k >= nch) { k -= nch; ++yi; }
    yi += dy;
    if (yi >= ny) { yi -= ny; ++zi; }
    zi += dz;
  }
};

// Position of one lane in chunk k of a row: its node pair and how the ±1 x
// shift reaches the neighbouring pairs (lane shuffle inside the chunk, or an
// element of the adjacent chunk at the chunk edge and the periodic wrap).
// FULL (nx a multiple of 64, at least two chunks per row: every chunk is
// full and only lanes 31 and 0 cross a chunk edge) fixes all but the two
// edge offsets at compile time.
template <bool FULL>
struct LaneX {
  int x0;
  int nxt_off;      // element offset from this lane's word to x0 + 2 (wrapped), same direction
  int prv_off;      // element offset from this lane's word to x0 - 1 (wrapped)
  int nxt_src, prv_src;
  bool active, nxt_in, prv_in;

  __device__ __forceinline__ void set(int Q, int nx, int nch, int k, int lane) {
    x0 = k * kChunk + 2 * lane;
    if constexpr (FULL) {
      active = true;
      nxt_in = lane != 31;
      prv_in = lane != 0;
      nxt_src = (lane + 1) & 31;
      prv_src = (lane + 31) & 31;
      // lane 31 -> element 0 of chunk k + 1 (or of chunk 0), lane 0 -> element
      // 63 of chunk k - 1 (or of chunk nch - 1); other lanes do not use them
      nxt_off = (k == nch - 1 ? -(nch - 1) * Q * kChunk : Q * kChunk) - 62;
      prv_off = (k == 0 ? (nch - 1) * Q * kChunk : -Q * kChunk) + 63;
    } else {
      active = x0 < nx;
      int xn = x0 + 2; if (xn >= nx) xn -= nx;
      int xp = x0 - 2; if (xp < 0) xp += nx;
      nxt_in = (xn >> 6) == k;
      prv_in = (xp >> 6) == k;
      nxt_src = nxt_in ? ((xn & 63) >> 1) : lane;
      prv_src = prv_in ? ((xp & 63) >> 1) : lane;
      int xm = x0 - 1; if (xm < 0) xm += nx;
      nxt_off = chunk_delta(Q, x0, xn);
      prv_off = chunk_delta(Q, x0, xm);
    }
  }
};

// Slot pointers of one chunk for one lane: own slot of direction i at
// own + i * 64, remote slot (node + c_i, direction i + 1 - P) at
// rem[cz + 1][cy + 1] + i * 64, so every access is a register plus an
// immediate offset.  Rows are addressed by their 32-bit index z * sy + y
// times the elements of one row (below 2^31, checked by the launcher): one
// wide multiply-add per pointer.
template <class L, int ST>
struct ChunkPtrs {
  using E = typename WordOps<ST>::E;
  E* own;
  E* rem[3][3];

  // Al: the populations plus this lane's element offset 2 * lane.  An
  // interior row's neighbours are padded rows on a non-periodic axis (the
  // halo), so only a periodic axis wraps.
  __device__ __forceinline__ void set(const Geo& g, E* Al, int P, const Cursor& c) {
    constexpr int Q = L::Q;
    const int py = c.yi + g.hy, pz = c.zi + g.hz;
    const unsigned rowel = (unsigned)g.nch * (unsigned)(Q * kChunk);
    E* kb = Al + c.k * (Q * kChunk);
    int ym = py - 1, yp = py + 1;
    if (ym < 0) ym += g.ny;
    if (yp >= g.sy) yp -= g.ny;
    const int yy[3] = {ym, py, yp};
    int zs[3];
    zs[1] = pz * g.sy;
    if constexpr (L::D == 3) {
      int zm = pz - 1, zp = pz + 1;
      if (zm < 0) zm += g.nz;
      if (zp >= g.sz) zp -= g.nz;
      zs[0] = zm * g.sy;
      zs[2] = zp * g.sy;
    } else {
      zs[0] = zs[2] = zs[1];
    }
    own = kb + (size_t)(unsigned)(zs[1] + py) * rowel + P * kChunk;
    E* kb1 = kb + (1 - P) * kChunk;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
        rem[dz][dy] = kb1 + (size_t)(unsigned)(zs[dz] + yy[dy]) * rowel;
  }
};

// Asynchronous global->shared copy of one word, to dst + DOFF from src +
// SOFF bytes (immediate offsets, so one base register serves a whole row of
// directions); src_bytes = 0 fills zeros and reads nothing.
template <int BYTES, int DOFF, int SOFF>
__device__ __forceinline__ void copy_async(uint32_t dst, const void* src, int src_bytes) {
  if constexpr (BYTES == 16) {
    asm volatile("cp.async.cg.shared.global [%0+%3], [%1+%4], 16, %2;\n" ::"r"(dst), "l"(src),
                 "r"(src_bytes), "n"(DOFF), "n"(SOFF) : "memory");
  } else {
    asm volatile("cp.async.ca.shared.global [%0+%4], [%1+%5], %2, %3;\n" ::"r"(dst), "l"(src),
                 "n"(BYTES), "r"(src_bytes), "n"(DOFF), "n"(SOFF) : "memory");
  }
}
// The same, issued only where `pred` holds (a predicated copy, no branch).
template <int BYTES, int DOFF>
__device__ __forceinline__ void copy_async_if(bool pred, uint32_t dst, const void* src) {
  if constexpr (BYTES == 16) {
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %2, 0;\n"
                 " @p cp.async.cg.shared.global [%0+%3], [%1], 16;\n}\n" ::"r"(dst), "l"(src),
                 "r"((int)pred), "n"(DOFF) : "memory");
  } else {
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %2, 0;\n"
                 " @p cp.async.ca.shared.global [%0+%4], [%1], %3;\n}\n" ::"r"(dst), "l"(src),
                 "r"((int)pred), "n"(BYTES), "n"(DOFF) : "memory");
  }
}
__device__ __forceinline__ void copy_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void copy_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Global store of one word or element at base + OFF bytes where `pred`
// holds: a predicated store instruction, never a branch around it.
template <int OFF>
__device__ __forceinline__ void st_if(bool pred, void* base, uint32_t v) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %0, 0;\n @p st.global.b32 [%1+%3], %2;\n}\n"
               ::"r"((int)pred), "l"(base), "r"(v), "n"(OFF) : "memory");
}
template <int OFF>
__device__ __forceinline__ void st_if(bool pred, void* base, uint16_t v) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %0, 0;\n @p st.global.b16 [%1+%3], %2;\n}\n"
               ::"r"((int)pred), "l"(base), "h"(v), "n"(OFF) : "memory");
}
template <int OFF>
__device__ __forceinline__ void st_if(bool pred, void* base, float v) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %0, 0;\n @p st.global.f32 [%1+%3], %2;\n}\n"
               ::"r"((int)pred), "l"(base), "f"(v), "n"(OFF) : "memory");
}
template <int OFF>
__device__ __forceinline__ void st_if(bool pred, void* base, float2 v) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %0, 0;\n"
               " @p st.global.v2.f32 [%1+%4], {%2, %3};\n}\n"
               ::"r"((int)pred), "l"(base), "f"(v.x), "f"(v.y), "n"(OFF) : "memory");
}
template <int OFF>
__device__ __forceinline__ void st_if(bool pred, void* base, double v) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %0, 0;\n @p st.global.f64 [%1+%3], %2;\n}\n"
               ::"r"((int)pred), "l"(base), "d"(v), "n"(OFF) : "memory");
}
template <int OFF>
__device__ __forceinline__ void st_if(bool pred, void* base, double2 v) {
  asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %0, 0;\n"
               " @p st.global.v2.f64 [%1+%4], {%2, %3};\n}\n"
               ::"r"((int)pred), "l"(base), "d"(v.x), "d"(v.y), "n"(OFF) : "memory");
}

template <int OP, int ST>
constexpr int stream_min_blocks() {
  return ST == kF64 ? 2 : pair_min_blocks<OP, ST>();
}

template <class L, int ST, int OP, int EQ, bool SH, bool FORCE, bool FULL>
__global__ void __launch_bounds__(kPairThreads, stream_min_blocks<OP, ST>())
step_stream(StepArgs a) {
  using WO = WordOps<ST>;
  using W = typename WO::W;
  using H = typename WO::H;
  using E = typename WO::E;
  using V = typename WO::V;
  using S = typename Lanes<V>::S;
  using Cfg = StreamCfg<L, ST>;
  using XW = XWord<ST>;
  constexpr int Q = L::Q;
  constexpr int NS = Cfg::STAGES;
  constexpr int WB = (int)sizeof(W);
  constexpr int EB = (int)sizeof(E);
  const Geo& g = a.g;

  extern __shared__ __align__(16) unsigned char stream_smem[];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const long long nunits = (long long)g.ny * g.nz * g.nch;
  const long long tw = (long long)gridDim.x * Cfg::WARPS;
  const long long gw = (long long)blockIdx.x * Cfg::WARPS + wib;
  if (gw >= nunits) return;  // whole warp idle (uniform)
  // the grid stride as (planes, rows, chunks)
  const int dk = (int)(tw % g.nch);
  const long long trow = tw / g.nch;
  const int dy = (int)(trow % g.ny);
  const int dz = (int)(trow / g.ny);

  E* Al = reinterpret_cast<E*>(a.f) + 2 * lane;
  const int P = a.parity;
  const CollideParams<S> prm{(S)a.omega, (S)a.omega2, (S)a.fx, (S)a.fy, (S)a.fz};

  unsigned char* ring = stream_smem + wib * Cfg::WARP_BYTES;
  // this lane's word 0 of stage 0, in the shared window
  const uint32_t ring_s = (uint32_t)__cvta_generic_to_shared(ring) + (uint32_t)(lane * WB);

  // Copy one chunk into stage buffer `st`: the lane's Q words, and the
  // neighbouring chunk's word of each x-shifted direction (the word holding
  // element x0 + 2, or x0 - 1), read only on the chunk-edge lane; every
  // other copy of an edge word, and every copy on a lane past the end of a
  // partial chunk, reads nothing and fills zeros.
  auto issue = [&](const Cursor& cu, int st) {
    LaneX<FULL> lx;
    lx.set(Q, g.nx, g.nch, cu.k, lane);
    ChunkPtrs<L, ST> cp;
    cp.set(g, Al, P, cu);
    const uint32_t sb = ring_s + (uint32_t)(st * Cfg::STAGE_WORDS * WB);
    const int nb = lx.active ? WB : 0;
    const int nbn = (lx.active && !lx.nxt_in) ? WB : 0;
    const int nbp = (lx.active && !lx.prv_in) ? WB : 0;
    copy_async<WB, 0, 0>(sb, cp.own - P * kChunk, nb);
    static_for<1, Q, 2>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
      const E* rp = cp.rem[cz + 1][cy + 1];
      copy_async<WB, i * 32 * WB, i * kChunk * EB>(sb, cp.own, nb);
      copy_async<WB, (i + 1) * 32 * WB, i * kChunk * EB>(sb, rp, nb);
      constexpr int ed = (Q + (xshift_index<L>(i) < 0 ? 0 : xshift_index<L>(i))) * 32 * WB;
      if constexpr (cx > 0) {
        copy_async<WB, ed, i * kChunk * EB>(sb, rp + lx.nxt_off, nbn);
      } else if constexpr (cx < 0) {
        copy_async<WB, ed, i * kChunk * EB>(sb, rp + lx.prv_off - 1, nbp);
      }
    });
  };

  // prologue: the first NS - 1 chunks in flight (one copy group each, empty
  // groups past the end keep the group count uniform)
  Cursor cur, nxt;
  cur.start(gw, g.nch, g.ny);
  nxt = cur;
#pragma unroll
  for (int s = 0; s < NS - 1; ++s) {
    if (nxt.u < nunits) issue(nxt, s);
    copy_commit();
    nxt.advance(tw, dk, dy, dz, g.nch, g.ny);
  }

  for (int st = 0; cur.u < nunits; st = (st + 1 == NS) ? 0 : st + 1) {
    // refill the buffer the previous chunk used with chunk + NS - 1 (all its
    // words were read into registers one iteration ago)
    {
      const int sn = (st == 0) ? NS - 1 : st - 1;
      if (nxt.u < nunits) issue(nxt, sn);
      copy_commit();
      nxt.advance(tw, dk, dy, dz, g.nch, g.ny);
    }
    // this chunk's copies (the oldest pending group) have landed
    copy_wait<NS - 1>();
    const W* sw = reinterpret_cast<const W*>(ring + st * Cfg::STAGE_WORDS * WB) + lane;
    W w[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) w[q] = sw[q * 32];

    LaneX<FULL> lx;
    lx.set(Q, g.nx, g.nch, cur.k, lane);
    // ±1 x shift of the remote words (shuffle, or the chunk-edge word)
    static_for<1, Q, 2>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::cx[i];
      if constexpr (cx != 0) {
        const W ew = sw[(Q + xshift_index<L>(i)) * 32];
        if constexpr (cx > 0) {
          const W nw = XW::shfl_lo(w[i + 1], lx.nxt_src);
          w[i + 1] = XW::join(w[i + 1], lx.nxt_in ? nw : ew);
        } else {
          const W pw = XW::shfl_hi(w[i + 1], lx.prv_src);
          w[i + 1] = XW::join(lx.prv_in ? pw : ew, w[i + 1]);
        }
      }
    });

    bool solid0 = false, solid1 = false;
    Macro<V> m;
    if constexpr (OP != 0) {
      V f[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) f[q] = WO::unpack(w[q]);
      if constexpr (FORCE) {  // the force per node of the pair (Boussinesq)
        CollideParams<S, V> pv{prm.omega, prm.omega2, bc<V>(prm.fx), bc<V>(prm.fy), bc<V>(prm.fz)};
        if (a.temp) {
          const S* T = reinterpret_cast<const S*>(a.temp);
          const size_t kk = ((size_t)cur.zi * g.ny + cur.yi) * g.nx + lx.x0;
          buoyant_force<V>(a, lx.active ? pack2v(load_pair2(T, kk)) : bc<V>(S(0)), pv.fx, pv.fy, pv.fz);
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
    ChunkPtrs<L, ST> cp;
    cp.set(g, Al, P, cur);
    if (a.flags) {
      const int py = cur.yi + g.hy, pz = cur.zi + g.hz;
      const uint16_t fl = lx.active ? *reinterpret_cast<const uint16_t*>(
          a.flags + ((long long)pz * g.sy + py) * g.sx + lx.x0) : 0;
      solid0 = (fl & 0xffu) != 0;
      solid1 = (fl >> 8) != 0;
      if (__any_sync(0xffffffffu, solid0 || solid1)) {
        // solid / excluded nodes write back what they read: re-read this
        // chunk's slots (not yet written) and reflect each pair
        auto pick = [&](W vin, W vout) -> W {
          return WO::make(solid0 ? WO::lo(vin) : WO::lo(vout), solid1 ? WO::hi(vin) : WO::hi(vout));
        };
        const E* rest = cp.own - P * kChunk;
        w[0] = pick(lx.active ? *reinterpret_cast<const W*>(rest) : W{}, w[0]);
        static_for<1, Q, 2>([&](auto I) {
          constexpr int i = decltype(I)::value;
          constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
          const E* rp = cp.rem[cz + 1][cy + 1] + i * kChunk;
          const W ro = lx.active ? *reinterpret_cast<const W*>(cp.own + i * kChunk) : W{};
          W rr = lx.active ? *reinterpret_cast<const W*>(rp) : W{};
          if constexpr (cx > 0) {
            H nlo = shfl_h(WO::lo(rr), lx.nxt_src);
            if (lx.active && !lx.nxt_in) nlo = *reinterpret_cast<const H*>(rp + lx.nxt_off);
            rr = WO::make(WO::hi(rr), nlo);
          } else if constexpr (cx < 0) {
            H phi = shfl_h(WO::hi(rr), lx.prv_src);
            if (lx.active && !lx.prv_in) phi = *reinterpret_cast<const H*>(rp + lx.prv_off);
            rr = WO::make(phi, WO::lo(rr));
          }
          // bounce-back: f_i' = f_{i+1}, f_{i+1}' = f_i, so the stores land in place
          w[i] = pick(rr, w[i]);
          w[i + 1] = pick(ro, w[i + 1]);
        });
      }
    }

    // ---- store: f_{i+1}' to the own slot, f_i' to the remote slot; the
    // shifted remote words are recombined across lanes, and the element that
    // belongs to the adjacent chunk goes out on its own
    const bool st_w_n = lx.active && lx.nxt_in, st_h_n = lx.active && !lx.nxt_in;
    const bool st_w_p = lx.active && lx.prv_in, st_h_p = lx.active && !lx.prv_in;
    if (lx.active) *reinterpret_cast<W*>(cp.own - P * kChunk) = w[0];
    static_for<1, Q, 2>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
      const W oi = w[i], oj = w[i + 1];
      if (lx.active) *reinterpret_cast<W*>(cp.own + i * kChunk) = oj;
      E* rp = cp.rem[cz + 1][cy + 1] + i * kChunk;
      if constexpr (cx == 0) {
        if (lx.active) *reinterpret_cast<W*>(rp) = oi;
      } else if constexpr (cx > 0) {
        const W pw = XW::shfl_hi(oi, lx.prv_src);
        if (st_w_p) *reinterpret_cast<W*>(rp) = XW::join(pw, oi);
        if (st_h_p) *reinterpret_cast<H*>(rp + 1) = WO::lo(oi);
        if (st_h_n) *reinterpret_cast<H*>(rp + lx.nxt_off) = WO::hi(oi);
      } else {
        const W nw = XW::shfl_lo(oi, lx.nxt_src);
        if (st_w_n) *reinterpret_cast<W*>(rp) = XW::join(oi, nw);
        if (st_h_n) *reinterpret_cast<H*>(rp) = WO::hi(oi);
        if (st_h_p) *reinterpret_cast<H*>(rp + lx.prv_off) = WO::lo(oi);
      }
    });

    {
      if (a.rho && lx.active)
        store_macro_pair<S>(a, ((size_t)cur.zi * g.ny + cur.yi) * g.nx + lx.x0, m, solid0, solid1);
    }
    cur.advance(tw, dk, dy, dz, g.nch, g.ny);
  }
  copy_wait<0>();  // no copy outlives the warp (the tail groups are empty)
}

}  // namespace m3lb
