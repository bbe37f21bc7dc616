// Kernels of the M3LB lattice-Boltzmann step on sm_100a.
//
// Streaming is Esoteric Pull on one population array (src/memory/
// EsotericPull.hpp:1-111): for every opposite pair (i, i+1), i odd, node n
// reads and writes exactly two slots, its own slot of direction i+P and the
// slot of direction i+1-P at node n + c_i (P = t % 2):
//     f_i     <- own,      f_{i+1} <- remote      (load_pair  :88-91)
//     remote  <- f_i',     own     <- f_{i+1}'    (store_pair :92-96)
// Every slot has one reader and one writer, the same node, so the update is in
// place and race free.  The parity only decides which of the two direction
// rows is "own": it is folded into two base offsets, so one kernel serves
// both parities with no per-node cost.
//
// Solid and excluded cells do nothing (implicit halfway bounce-back,
// EsotericPull.hpp:27-33): the paired kernel writes their slots back
// unchanged, the one-node kernel skips them.
#pragma once
#include "lbm_collide.cuh"

namespace m3lb {

constexpr int kPairThreads = 128;
constexpr int kNodeThreads = 128;

// ------------------------------------------------------- FP64 node pairs
struct d2 { double x, y; };
__device__ __forceinline__ d2 add(d2 a, d2 b) { return {__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)}; }
__device__ __forceinline__ d2 mul(d2 a, d2 b) { return {__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)}; }
__device__ __forceinline__ d2 fma(d2 a, d2 b, d2 c) { return {__fma_rn(a.x, b.x, c.x), __fma_rn(a.y, b.y, c.y)}; }
__device__ __forceinline__ d2 sub(d2 a, d2 b) { return {__fma_rn(b.x, -1.0, a.x), __fma_rn(b.y, -1.0, a.y)}; }
__device__ __forceinline__ d2 neg(d2 a) { return {-a.x, -a.y}; }
__device__ __forceinline__ d2 rcp(d2 a) { return {__drcp_rn(a.x), __drcp_rn(a.y)}; }
template <> struct Lanes<d2> { using S = double; static constexpr int N = 2; };
__device__ __forceinline__ f2 pack2(float a, float b) { return mk(a, b); }
__device__ __forceinline__ d2 pack2(double a, double b) { return d2{a, b}; }

// BoussinesqGuo::at (Forcing.hpp:113-117) for one node or a node pair at
// temperature T: F = (fx, fy, fz) + g b, b = rho0 beta (T - T0), rounded op
// by op so that paired and one-node kernels agree bit for bit.
template <class V>
__device__ __forceinline__ void buoyant_force(const StepArgs& a, V T, V& fx, V& fy, V& fz) {
  using S = typename Lanes<V>::S;
  const V b = mul(bc<V>(S(a.brho0) * S(a.bbeta)), sub(T, bc<V>(S(a.bT0))));
  fx = add(bc<V>(S(a.fx)), mul(bc<V>(S(a.bgx)), b));
  fy = add(bc<V>(S(a.fy)), mul(bc<V>(S(a.bgy)), b));
  fz = add(bc<V>(S(a.fz)), mul(bc<V>(S(a.bgz)), b));
}
// Collision parameters of one node (interior index k) in the one-node kernels.
template <bool FORCE, class R>
__device__ __forceinline__ CollideParams<R> node_params(const StepArgs& a, size_t k) {
  CollideParams<R> p{(R)a.omega, (R)a.omega2, (R)a.fx, (R)a.fy, (R)a.fz};
  if constexpr (FORCE)
    if (a.temp) buoyant_force<R>(a, reinterpret_cast<const R*>(a.temp)[k], p.fx, p.fy, p.fz);
  return p;
}
template <> __device__ __forceinline__ d2 bc<d2>(double a) { return {a, a}; }
__device__ __forceinline__ double lane_of(d2 a, int k) { return k ? a.y : a.x; }
__device__ __forceinline__ f2 pack2v(float2 v) { return pack2(v.x, v.y); }
__device__ __forceinline__ d2 pack2v(double2 v) { return pack2(v.x, v.y); }

// Two adjacent elements (x0, x0 + 1; x0 even, so the pair is one aligned
// 8- or 16-byte word when the array is aligned) of a per-node array.
template <class R> struct Vec2;
template <> struct Vec2<float> { using T = float2; };
template <> struct Vec2<double> { using T = double2; };
template <class R>
__device__ __forceinline__ bool pair_aligned(const void* p) {
  return (reinterpret_cast<uintptr_t>(p) & (2 * sizeof(R) - 1)) == 0;
}
template <class R>
__device__ __forceinline__ typename Vec2<R>::T load_pair2(const R* p, size_t k) {
  if (pair_aligned<R>(p)) return *reinterpret_cast<const typename Vec2<R>::T*>(p + k);
  return typename Vec2<R>::T{p[k], p[k + 1]};
}
// rho, u of a node pair into the macroscopic arrays at interior index kk
// (even); a solid node of the pair keeps its value.
template <class R, class V>
__device__ __forceinline__ void store_macro_pair(const StepArgs& a, size_t kk, const Macro<V>& m,
                                                 bool solid0, bool solid1) {
  R* dst[4] = {reinterpret_cast<R*>(a.rho), reinterpret_cast<R*>(a.ux), reinterpret_cast<R*>(a.uy),
               reinterpret_cast<R*>(a.uz)};
  const V val[4] = {m.rho, m.ux, m.uy, m.uz};
  const bool whole = !solid0 && !solid1 && pair_aligned<R>(a.rho) && pair_aligned<R>(a.ux) &&
                     pair_aligned<R>(a.uy) && pair_aligned<R>(a.uz);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    if (whole) {
      *reinterpret_cast<typename Vec2<R>::T*>(dst[f] + kk) =
          typename Vec2<R>::T{(R)lane_of(val[f], 0), (R)lane_of(val[f], 1)};
    } else {
      if (!solid0) dst[f][kk] = (R)lane_of(val[f], 0);
      if (!solid1) dst[f][kk + 1] = (R)lane_of(val[f], 1);
    }
  }
}

// ------------------------------------------------------------ word traits
// A word holds one direction of two x-adjacent nodes (lo = even x).
// unpack(w) decodes the two elements of a word; unpack_join(a, b) decodes
// the pair (hi element of a, lo element of b), the x-shifted pair that
// straddles two words, without first joining them.
template <int ST> struct WordOps;
template <> struct WordOps<kF32> {
  using W = float2; using H = float; using V = f2; using E = float;
  static __device__ __forceinline__ V unpack(W w) { return f2{w}; }
  static __device__ __forceinline__ V unpack_join(W a, W b) { return f2{make_float2(a.y, b.x)}; }
  static __device__ __forceinline__ W pack(V v) { return v.v; }
  static __device__ __forceinline__ H lo(W w) { return w.x; }
  static __device__ __forceinline__ H hi(W w) { return w.y; }
  static __device__ __forceinline__ W make(H l, H h) { return make_float2(l, h); }
};
template <> struct WordOps<kF64> {
  using W = double2; using H = double; using V = d2; using E = double;
  static __device__ __forceinline__ V unpack(W w) { return {w.x, w.y}; }
  static __device__ __forceinline__ V unpack_join(W a, W b) { return {a.y, b.x}; }
  static __device__ __forceinline__ W pack(V v) { return make_double2(v.x, v.y); }
  static __device__ __forceinline__ H lo(W w) { return w.x; }
  static __device__ __forceinline__ H hi(W w) { return w.y; }
  static __device__ __forceinline__ W make(H l, H h) { return make_double2(l, h); }
};
template <> struct WordOps<kF16> {
  using W = uint32_t; using H = uint16_t; using V = f2; using E = __half;
  static __device__ __forceinline__ V unpack(W w) { return unpack_f16(w); }
  static __device__ __forceinline__ V unpack_join(W a, W b) {
    return f2{make_float2(__half2float(__ushort_as_half((unsigned short)(a >> 16))),
                          __half2float(__ushort_as_half((unsigned short)(b & 0xffffu))))};
  }
  static __device__ __forceinline__ W pack(V v) { return pack_f16(v); }
  static __device__ __forceinline__ H lo(W w) { return (H)(w & 0xffffu); }
  static __device__ __forceinline__ H hi(W w) { return (H)(w >> 16); }
  static __device__ __forceinline__ W make(H l, H h) { return (W)l | ((W)h << 16); }
};
template <> struct WordOps<kF16C> {
  using W = uint32_t; using H = uint16_t; using V = f2; using E = f16c;
  static __device__ __forceinline__ V unpack(W w) { return unpack_f16c(w); }
  static __device__ __forceinline__ V unpack_join(W a, W b) {
    const float lo = __uint_as_float(f16c_hi_bits(a)), hi = __uint_as_float(f16c_hi_bits(b << 16));
    return f2{mul2_rn(make_float2(lo, hi), make_float2(kF16CUp, kF16CUp))};
  }
  static __device__ __forceinline__ W pack(V v) { return pack_f16c(v); }
  static __device__ __forceinline__ H lo(W w) { return (H)(w & 0xffffu); }
  static __device__ __forceinline__ H hi(W w) { return (H)(w >> 16); }
  static __device__ __forceinline__ W make(H l, H h) { return (W)l | ((W)h << 16); }
};
template <> struct WordOps<kBF16> {
  using W = uint32_t; using H = uint16_t; using V = f2; using E = __nv_bfloat16;
  static __device__ __forceinline__ V unpack(W w) { return unpack_bf16(w); }
  static __device__ __forceinline__ V unpack_join(W a, W b) {
    return f2{make_float2(__uint_as_float(a & 0xffff0000u), __uint_as_float(b << 16))};
  }
  static __device__ __forceinline__ W pack(V v) { return pack_bf16(v); }
  static __device__ __forceinline__ H lo(W w) { return (H)(w & 0xffffu); }
  static __device__ __forceinline__ H hi(W w) { return (H)(w >> 16); }
  static __device__ __forceinline__ W make(H l, H h) { return (W)l | ((W)h << 16); }
};

template <class H>
__device__ __forceinline__ H shfl_h(H v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <>
__device__ __forceinline__ uint16_t shfl_h<uint16_t>(uint16_t v, int src) {
  return (uint16_t)__shfl_sync(0xffffffffu, (unsigned)v, src);
}

// Element offset of slot (x, y, z, q) in the chunked layout.
template <int Q>
__device__ __forceinline__ size_t slot(const Geo& g, int x, int y, int z, int q) {
  return ((((size_t)((long long)z * g.sy + y) * g.nch + (x >> 6)) * Q + q) << 6) + (size_t)(x & 63);
}

// ---------------------------------------------------- paired step kernel
// Requires a periodic x axis (no x halo) and even nx.  Warp w owns chunk
// (row, k) of the interior rows; lane l the node pair x0 = 64k + 2l,
// x0 + 1.  A direction with c_x = +-1 needs an element of the neighbouring
// pair: it comes from the adjacent lane by a shuffle, or, across a chunk
// edge, from one extra element load; the shifted stores are recombined the
// same way, so every bulk access is an aligned word of a 64-node segment.
template <class L, int ST>
struct PairCtx {
  using WO = WordOps<ST>;
  using W = typename WO::W;
  using H = typename WO::H;
  using E = typename WO::E;
  static constexpr int Q = L::Q;
  E* own;           // &A[row, chunk, dir 0 + P, x0 % 64]
  E* rem[3][3];     // [dz+1][dy+1]: &A[row + (dy,dz), chunk, dir 1 - P, x0 % 64]
  int nxt_off;      // element offset from this lane's word to x0 + 2 (wrapped), same direction
  int prv_off;      // element offset from this lane's word to x0 - 1 (wrapped)
  int nxt_src, prv_src;
  bool nxt_in, prv_in, active;

  template <int I>
  __device__ __forceinline__ void load_pair(W& o, W& r) const {
    constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
    o = active ? *reinterpret_cast<const W*>(own + I * kChunk) : W{};
    const E* rp = rem[cz + 1][cy + 1] + I * kChunk;
    const W w = active ? *reinterpret_cast<const W*>(rp) : W{};
    if constexpr (cx == 0) {
      r = w;
    } else if constexpr (cx > 0) {
      // elements (x0+1, x0+2): own hi and the next pair's lo
      H nlo = shfl_h(WO::lo(w), nxt_src);
      if (active && !nxt_in) nlo = *reinterpret_cast<const H*>(rp + nxt_off);
      r = WO::make(WO::hi(w), nlo);
    } else {
      // elements (x0-1, x0): the previous pair's hi and own lo
      H phi = shfl_h(WO::hi(w), prv_src);
      if (active && !prv_in) phi = *reinterpret_cast<const H*>(rp + prv_off);
      r = WO::make(phi, WO::lo(w));
    }
  }

  // f_i' to the remote slot, f_{i+1}' to the own slot.
  template <int I>
  __device__ __forceinline__ void store_pair(W out_i, W out_j) const {
    constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
    if (active) *reinterpret_cast<W*>(own + I * kChunk) = out_j;
    E* rp = rem[cz + 1][cy + 1] + I * kChunk;
    if constexpr (cx == 0) {
      if (active) *reinterpret_cast<W*>(rp) = out_i;
    } else if constexpr (cx > 0) {
      // outputs of (x0, x0+1) land on (x0+1, x0+2)
      const H phi = shfl_h(WO::hi(out_i), prv_src);
      if (active) {
        if (prv_in) *reinterpret_cast<W*>(rp) = WO::make(phi, WO::lo(out_i));
        else *reinterpret_cast<H*>(rp + 1) = WO::lo(out_i);
        if (!nxt_in) *reinterpret_cast<H*>(rp + nxt_off) = WO::hi(out_i);
      }
    } else {
      // outputs of (x0, x0+1) land on (x0-1, x0)
      const H nlo = shfl_h(WO::lo(out_i), nxt_src);
      if (active) {
        if (nxt_in) *reinterpret_cast<W*>(rp) = WO::make(WO::hi(out_i), nlo);
        else *reinterpret_cast<H*>(rp) = WO::hi(out_i);
        if (!prv_in) *reinterpret_cast<H*>(rp + prv_off) = WO::lo(out_i);
      }
    }
  }
};

// Element offset, within one direction, from chunk-local position xa of chunk
// ca to position xb of chunk cb.
__device__ __forceinline__ int chunk_delta(int Q, int xa, int xb) {
  return ((xb >> 6) - (xa >> 6)) * Q * kChunk + ((xb & 63) - (xa & 63));
}

// Resident 128-thread blocks per SM the register allocation must allow:
// four (<= 128 registers) for the moment operators, three for BGK/TRT, whose
// per-pair equilibria keep more values live, and for 32-bit pure streaming,
// two for FP64 pairs, which need twice the registers per value.
template <int OP, int ST>
constexpr int pair_min_blocks() {
  return ST == kF64 ? 2 : ((OP == 1 || OP == 2 || (OP == 0 && ST == kF32)) ? 3 : (OP >= 3 && ST != kF32 ? 5 : 4));
}

// One unit of 64 nodes by one warp.  Shared by the paired kernel and the
// batched kernel of the serving loop, so a lattice gets the same arithmetic
// in both.  Two mappings of units to nodes:
//   * chunks (DENSE false): unit `warp` is chunk (row, k) of the lattice's
//     ny * nz * nch chunks; lane l holds x0 = 64 k + 2 l, idle past nx;
//   * dense: unit `warp` is interior nodes 64 warp ... 64 warp + 63 in x-fastest
//     order, rows of any even length packed back to back, so every lane
//     works whatever nx is; a warp spans parts of several rows, each lane
//     addresses its own row, and the x neighbour of a row's last pair (its
//     first pair, periodic wrap) comes by shuffle when that pair is in the
//     same warp, else from memory.
// The per-node arithmetic, and so the result, is the same in both.
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE, bool DENSE = false>
__device__ __forceinline__ void pairs_unit(const StepArgs& a, long long warp, int lane) {
  using WO = WordOps<ST>;
  using W = typename WO::W;
  using E = typename WO::E;
  using V = typename WO::V;
  using S = typename Lanes<V>::S;
  constexpr int Q = L::Q;
  const Geo& g = a.g;

  int x0, yi, zi, k;
  bool ok;
  int nx_ = 0, px_ = 0;  // x0 + 2 and x0 - 2, wrapped
  bool nxt_in, prv_in;
  int nxt_src, prv_src;
  if constexpr (DENSE) {
    const long long nodes = (long long)g.nx * g.ny * g.nz;
    const long long f0 = warp * kChunk;  // first node of the unit
    ok = f0 + 2 * lane < nodes;
    const long long fs = f0 < nodes ? f0 : 0;  // (a unit past the end addresses node 0)
    const long long row0 = fs / g.nx;
    const int xs = (int)(fs - row0 * g.nx);  // x of the unit's first node
    int x = xs + 2 * lane, dr = 0;
    while (x >= g.nx) { x -= g.nx; ++dr; }  // at most 64 / nx + 1 rows
    const long long row = ok ? row0 + dr : row0;
    yi = (int)(row % g.ny);
    zi = (int)(row / g.ny);
    x0 = ok ? x : 0;
    k = x0 >> 6;
    nx_ = x0 + 2; if (nx_ >= g.nx) nx_ -= g.nx;
    px_ = x0 - 2; if (px_ < 0) px_ += g.nx;
    // position inside the unit of an x of this lane's row
    const int rs = dr * g.nx - xs;
    const int pn = rs + nx_, pp = rs + px_;
    nxt_in = pn >= 0 && pn < kChunk;
    prv_in = pp >= 0 && pp < kChunk;
    nxt_src = nxt_in ? (pn >> 1) : lane;
    prv_src = prv_in ? (pp >> 1) : lane;
  } else {
    const long long nrows = (long long)g.ny * g.nz;
    const bool warp_ok = warp < nrows * g.nch;
    const long long wsafe = warp_ok ? warp : 0;
    const int row = (int)(wsafe / g.nch);
    k = (int)(wsafe - (long long)row * g.nch);
    x0 = k * kChunk + 2 * lane;
    yi = row % g.ny;
    zi = row / g.ny;
    ok = warp_ok && x0 < g.nx;
    nx_ = x0 + 2; if (nx_ >= g.nx) nx_ -= g.nx;
    px_ = x0 - 2; if (px_ < 0) px_ += g.nx;
    nxt_in = (nx_ >> 6) == k;
    prv_in = (px_ >> 6) == k;
    nxt_src = nxt_in ? ((nx_ & 63) >> 1) : lane;
    prv_src = prv_in ? ((px_ & 63) >> 1) : lane;
  }
  const int py = yi + g.hy, pz = zi + g.hz;

  PairCtx<L, ST> c;
  c.active = ok;
  {
    c.nxt_in = nxt_in;
    c.prv_in = prv_in;
    c.nxt_src = nxt_src;
    c.prv_src = prv_src;
    int xn = x0 + 2; if (xn >= g.nx) xn -= g.nx;
    int xp = x0 - 1; if (xp < 0) xp += g.nx;
    c.nxt_off = chunk_delta(Q, x0, xn);
    c.prv_off = chunk_delta(Q, x0, xp);
    E* A = reinterpret_cast<E*>(a.f);
    const int P = a.parity;
    int yy[3], zz[3];
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      yy[d + 1] = shift_coord(py + d, g.hy, g.ny, g.sy, g.py);
      zz[d + 1] = (L::D == 3) ? shift_coord(pz + d, g.hz, g.nz, g.sz, g.pz) : pz;
    }
    const int xl = x0 & 63;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
        c.rem[dz][dy] = A + slot<Q>(g, k * kChunk, yy[dy], zz[dz], 1 - P) + xl;
    c.own = A + slot<Q>(g, k * kChunk, py, pz, P) + xl;
  }
  E* rest = c.own - a.parity * kChunk;

  // ---- load
  W w[Q];
  w[0] = c.active ? *reinterpret_cast<const W*>(rest) : W{};
  static_for<1, Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    c.template load_pair<i>(w[i], w[i + 1]);
  });

  bool solid0 = false, solid1 = false;
  Macro<V> m;
  if constexpr (OP != 0) {
    V f[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) f[q] = WO::unpack(w[q]);

    // ---- collide
    if constexpr (FORCE) {  // the force as one value per node of the pair
      CollideParams<S, V> prm{(S)a.omega, (S)a.omega2, bc<V>((S)a.fx), bc<V>((S)a.fy),
                              bc<V>((S)a.fz)};
      if (a.temp) {
        const S* T = reinterpret_cast<const S*>(a.temp);
        const size_t kk = ((size_t)zi * g.ny + yi) * g.nx + x0;
        buoyant_force<V>(a, c.active ? pack2v(load_pair2(T, kk)) : bc<V>(S(0)), prm.fx, prm.fy, prm.fz);
      }
      m = collide<L, OP, EQ, SH, FORCE>(f, prm);
    } else {
      const CollideParams<S> prm{(S)a.omega, (S)a.omega2, (S)a.fx, (S)a.fy, (S)a.fz};
      m = collide<L, OP, EQ, SH, FORCE>(f, prm);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) w[q] = WO::pack(f[q]);
  } else {  // pure streaming reports rest: rho 1, u 0 (the no-collision mock)
    m.dens = m.rho = bc<V>(1);
    m.ux = m.uy = m.uz = bc<V>(0);
  }

  // ---- solid / excluded nodes write back what they read (the identity)
  if (a.flags) {
    const uint16_t fl = c.active ? *reinterpret_cast<const uint16_t*>(
        a.flags + ((long long)pz * g.sy + py) * g.sx + x0) : 0;
    solid0 = (fl & 0xffu) != 0;
    solid1 = (fl >> 8) != 0;
    if (__any_sync(0xffffffffu, solid0 || solid1)) {
      auto pick = [&](W vin, W vout) -> W {
        return WO::make(solid0 ? WO::lo(vin) : WO::lo(vout), solid1 ? WO::hi(vin) : WO::hi(vout));
      };
      w[0] = pick(c.active ? *reinterpret_cast<const W*>(rest) : W{}, w[0]);
      static_for<1, Q, 2>([&](auto I) {
        constexpr int i = decltype(I)::value;
        W wo, wr;
        c.template load_pair<i>(wo, wr);
        // bounce-back: f_i' = f_{i+1}, f_{i+1}' = f_i, so the stores land in place
        w[i] = pick(wr, w[i]);
        w[i + 1] = pick(wo, w[i + 1]);
      });
    }
  }

  // ---- store
  if (c.active) *reinterpret_cast<W*>(rest) = w[0];
  static_for<1, Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    c.template store_pair<i>(w[i], w[i + 1]);
  });

  {
    if (a.rho && c.active)
      store_macro_pair<S>(a, ((size_t)zi * g.ny + yi) * g.nx + x0, m, solid0, solid1);
  }
}

template <class L, int ST, int OP, int EQ, bool SH, bool FORCE>
__global__ void __launch_bounds__(kPairThreads, pair_min_blocks<OP, ST>())
step_pairs(StepArgs a) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  pairs_unit<L, ST, OP, EQ, SH, FORCE>(a, warp, threadIdx.x & 31);
}

// -------------------------------------------------- one-node step kernel
// Any geometry: one node per thread, neighbours by the wrap / clamp of
// Domain::fill_neighbours (Domain.hpp:82-101).  Used where the paired kernel
// does not apply (non-periodic x, odd nx).  NodeNb holds the neighbour
// coordinates (boundary pass); the per-node kernels below address slots
// through per-axis offsets instead (AxisSteps).
template <class L>
struct NodeNb {
  int x, y, z;
  int nb[L::Q][3];  // neighbour coordinates for odd i
};
template <class L>
__device__ __forceinline__ void node_neighbours(const Geo& g, int x, int y, int z, NodeNb<L>& nb) {
  nb.x = x; nb.y = y; nb.z = z;
  static_for<1, L::Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    nb.nb[i][0] = shift_coord(x + cx, g.hx, g.nx, g.sx, g.px);
    nb.nb[i][1] = shift_coord(y + cy, g.hy, g.ny, g.sy, g.py);
    nb.nb[i][2] = shift_coord(z + cz, g.hz, g.nz, g.sz, g.pz);
  });
}
// Access::load(nb, i) (EsotericPull.hpp:69-77): slot holding the population of
// direction i about to arrive at the node.
template <class L>
__device__ __forceinline__ size_t load_slot(const Geo& g, const NodeNb<L>& nb, int par, int i) {
  if (i == 0) return slot<L::Q>(g, nb.x, nb.y, nb.z, 0);
  if (i & 1) return slot<L::Q>(g, nb.x, nb.y, nb.z, par == 0 ? i : i + 1);
  const int* m = nb.nb[i - 1];
  return slot<L::Q>(g, m[0], m[1], m[2], par == 0 ? i : i - 1);
}

// The same slots without per-direction coordinate arithmetic.  A slot is
// ((z sy + y) nch + x/64) Q 64 + q 64 + x%64, so the slot of direction q at
// the neighbour along c is the node's own slot of direction 0, plus q 64,
// plus one precomputed offset per nonzero component of c: the element offset
// to the same slot one step down [0] or up [1] each axis (the wrap or clamp
// of shift_coord folded in).
template <int Q>
struct AxisSteps {
  long long x[2], y[2], z[2];
};
template <int Q>
__device__ __forceinline__ long long x_part(int v) {
  return ((long long)(v >> 6) * Q << 6) + (v & 63);
}
template <int Q>
__device__ __forceinline__ AxisSteps<Q> axis_steps(const Geo& g, int x, int y, int z) {
  AxisSteps<Q> s;
  const long long row = (long long)g.nch * Q * kChunk, plane = row * g.sy;
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int d = 2 * u - 1;
    s.x[u] = x_part<Q>(shift_coord(x + d, g.hx, g.nx, g.sx, g.px)) - x_part<Q>(x);
    s.y[u] = (long long)(shift_coord(y + d, g.hy, g.ny, g.sy, g.py) - y) * row;
    s.z[u] = (long long)(shift_coord(z + d, g.hz, g.nz, g.sz, g.pz) - z) * plane;
  }
  return s;
}
// Offset to the neighbour at x + c_I.
template <class L, int I>
__device__ __forceinline__ long long nb_offset(const AxisSteps<L::Q>& s) {
  constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
  long long o = 0;
  if constexpr (cx != 0) o += s.x[cx > 0];
  if constexpr (cy != 0) o += s.y[cy > 0];
  if constexpr (cz != 0) o += s.z[cz > 0];
  return o;
}
// load_slot of direction I from the node's slot of direction 0.
template <class L, int I>
__device__ __forceinline__ size_t load_slot_at(size_t own, const AxisSteps<L::Q>& s, int par) {
  if constexpr (I == 0) return own;
  else if constexpr ((I & 1) != 0) return own + (size_t)((par == 0 ? I : I + 1) * kChunk);
  else return own + nb_offset<L, I - 1>(s) + (long long)((par == 0 ? I : I - 1) * kChunk);
}
// The node's logical populations (Access::load at parity par) as reals.
template <class L, class E, class R>
__device__ __forceinline__ void load_node(const E* A, const Geo& g, int x, int y, int z, int par, R* f) {
  const size_t own = slot<L::Q>(g, x, y, z, 0);
  const AxisSteps<L::Q> st = axis_steps<L::Q>(g, x, y, z);
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    f[i] = to_real(A[load_slot_at<L, i>(own, st, par)]);
  });
}

// Per-node kernels other than the paired ones run a 2-D grid: blockIdx.x the
// x segment, blockIdx.y the row (y + ny z), striding by gridDim.y, so a
// node's coordinates come from additions, not 64-bit divisions.
struct RowWalk {
  int y, z, dy, dz, ny;
  __device__ __forceinline__ explicit RowWalk(int ny_) : ny(ny_) {
    y = (int)(blockIdx.y % (unsigned)ny_);
    z = (int)(blockIdx.y / (unsigned)ny_);
    dy = (int)(gridDim.y % (unsigned)ny_);
    dz = (int)(gridDim.y / (unsigned)ny_);
  }
  __device__ __forceinline__ void next() {
    y += dy;
    z += dz;
    if (y >= ny) { y -= ny; ++z; }
  }
};
inline dim3 node_grid(int nx, long long rows, int threads) {
  return dim3((unsigned)((nx + threads - 1) / threads),
              (unsigned)(rows < 65535 ? (rows > 0 ? rows : 1) : 65535));
}

// ------------------------------------------------------- specular walls
// Free-slip cell types (src/boundary/Flags.hpp:20-32): a SpecWall node is a
// ghost that reflects its whole incoming set about one axis and does not
// collide; a SpecNode is a fluid node whose unknown directions take their
// mirror images before it collides.  Both only permute values among the Q
// slots the node already reads and writes, so they need no extra buffer.

// Direction whose velocity is c_i with the components in `flip` (bit a =
// axis a) negated: the axis mirrors of src/boundary/Specular.hpp:104-118,
// composed as mirror_unknowns_faces (:263-278) composes them.
template <class L>
__host__ __device__ constexpr int mirror_of(int i, int flip) {
  const int j = dir_of<L>((flip & 1) ? -L::cx[i] : L::cx[i], (flip & 2) ? -L::cy[i] : L::cy[i],
                          (flip & 4) ? -L::cz[i] : L::cz[i]);
  return j < 0 ? i : j;
}
template <class L>
__host__ __device__ constexpr bool mirrors_are_permutations() {  // Specular.hpp:356-375
  for (int a = 0; a < 3; ++a)
    for (int i = 0; i < L::Q; ++i) {
      const int j = mirror_of<L>(i, 1 << a);
      if (mirror_of<L>(j, 1 << a) != i) return false;
      const int c[3] = {L::cx[i], L::cy[i], L::cz[i]}, d[3] = {L::cx[j], L::cy[j], L::cz[j]};
      for (int b = 0; b < 3; ++b)
        if (d[b] != (b == a ? -c[b] : c[b])) return false;
    }
  return true;
}
static_assert(mirrors_are_permutations<D2Q9>() && mirrors_are_permutations<D3Q27>(),
              "axis mirrors must permute the velocity set");
// Axes a velocity has a nonzero component on (bit a = axis a).
template <class L>
__host__ __device__ constexpr int moving_axes(int i) {
  return (L::cx[i] != 0 ? 1 : 0) | (L::cy[i] != 0 ? 2 : 0) | (L::cz[i] != 0 ? 4 : 0);
}

// mirror_axis (Specular.hpp:124-128): 0 for +-x, 1 for +-y, 2 otherwise.
__device__ __forceinline__ int spec_axis(unsigned code) {
  return (code == 1 || code == 2) ? 0 : ((code == 3 || code == 4) ? 1 : 2);
}

// SpecWall: f_i <- f_{m(i)} about one axis (FluidSolver.hpp:745-757).
template <class L, class R>
__device__ __forceinline__ void spec_wall_permute(R* f, int ax) {
  R h[L::Q];
#pragma unroll
  for (int i = 0; i < L::Q; ++i) h[i] = f[i];
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    f[i] = ax == 0 ? h[mirror_of<L>(i, 1)] : (ax == 1 ? h[mirror_of<L>(i, 2)] : h[mirror_of<L>(i, 4)]);
  });
}

// SpecNode: mirror_unknowns_faces (Specular.hpp:263-278).  A direction
// pointing into the domain across a masked face (c_ia * face_sign(a) < 0)
// takes the value of its image over every such axis; the others are kept.
template <class L, class R>
__device__ __forceinline__ void spec_node_mirror(R* f, unsigned faces) {
  int sg[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)  // face_sign (:238-243): +x wins if both were set
    sg[a] = ((faces >> (2 * a)) & 1u) ? 1 : (((faces >> (2 * a + 1)) & 1u) ? -1 : 0);
  R h[L::Q];
#pragma unroll
  for (int i = 0; i < L::Q; ++i) h[i] = f[i];
  static_for<1, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    const int flip = (sg[0] * cx < 0 ? 1 : 0) | (sg[1] * cy < 0 ? 2 : 0) | (sg[2] * cz < 0 ? 4 : 0);
    R v = h[i];
    static_for<1, 8>([&](auto M) {
      constexpr int m = decltype(M)::value;
      if constexpr ((m & moving_axes<L>(i)) == m)
        if (flip == m) v = h[mirror_of<L>(i, m)];
    });
    f[i] = v;
  });
}

// Raw moments of a SpecNode after its mirror (compute_macroscopic,
// FluidSolver.hpp:1061-1080): populations unshifted, rho = sum f_i, u =
// sum f_i c_i / rho, no force correction.
template <class L, int OP, bool SH, class R>
__device__ __forceinline__ Macro<R> spec_node_moments(R* f) {
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if constexpr (SH && OP != 0) f[i] += R(weight<L, i>());
  });
  R sm = 0, mx = 0, my = 0, mz = 0;
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    sm += f[i];
    if constexpr (cx != 0) mx += cx > 0 ? f[i] : -f[i];
    if constexpr (cy != 0) my += cy > 0 ? f[i] : -f[i];
    if constexpr (cz != 0) mz += cz > 0 ? f[i] : -f[i];
  });
  const R ir = R(1) / sm;
  Macro<R> m;
  m.dens = sm; m.rho = sm; m.ux = mx * ir; m.uy = my * ir; m.uz = mz * ir;
  return m;
}

// One interior node of step_nodes.
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE>
__device__ __forceinline__ void node_step(const StepArgs& a, int xi, int yi, int zi) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const Geo& g = a.g;
  const long long k = ((long long)zi * g.ny + yi) * g.nx + xi;
  const int x = xi + g.hx, y = yi + g.hy, z = zi + g.hz;
  // Solid and Excluded skip (bounce-back is the identity on this storage);
  // wall nodes are left to the boundary pass
  if (a.flags && a.flags[((long long)z * g.sy + y) * g.sx + x] != 0) return;
  const AxisSteps<Q> st = axis_steps<Q>(g, x, y, z);
  E* own = reinterpret_cast<E*>(a.f) + slot<Q>(g, x, y, z, 0);
  const int P = a.parity;
  // direction i (odd) at slot i + P of the node, i + 1 at slot i + 1 - P of
  // the neighbour along c_i
  E* up = own + P * kChunk;
  E* dn = own + (1 - P) * kChunk;
  R f[Q];
  f[0] = to_real(own[0]);
  static_for<1, Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    f[i] = to_real(up[i * kChunk]);
    f[i + 1] = to_real(dn[nb_offset<L, i>(st) + i * kChunk]);
  });
  const CollideParams<R> prm = node_params<FORCE, R>(a, (size_t)k);
  const Macro<R> mc = collide<L, OP, EQ, SH, FORCE>(f, prm);
  own[0] = from_real<E>(f[0]);
  static_for<1, Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    dn[nb_offset<L, i>(st) + i * kChunk] = from_real<E>(f[i]);
    up[i * kChunk] = from_real<E>(f[i + 1]);
  });
  if (a.rho) {
    reinterpret_cast<R*>(a.rho)[k] = mc.rho;
    reinterpret_cast<R*>(a.ux)[k] = mc.ux;
    reinterpret_cast<R*>(a.uy)[k] = mc.uy;
    reinterpret_cast<R*>(a.uz)[k] = mc.uz;
  }
}

template <class L, int ST, int OP, int EQ, bool SH, bool FORCE>
__global__ void __launch_bounds__(kNodeThreads)
step_nodes(StepArgs a) {
  const Geo& g = a.g;
  const int xi = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (xi >= g.nx) return;
  for (RowWalk rw(g.ny); rw.z < g.nz; rw.next()) node_step<L, ST, OP, EQ, SH, FORCE>(a, xi, rw.y, rw.z);
}

// ------------------------------------------------------- initialisation
// seed_value (BGK.hpp:95-99, TRT.hpp:129-133, MomentCollision.hpp:320-330)
// evaluated in the reference's operation order, one rounding per operation.
template <class L, int OP, int EQ, bool SH, class R>
__device__ __forceinline__ void seed_all(R rho, R ux, R uy, R uz, R* out) {
  if constexpr (OP == 0) {
#pragma unroll
    for (int i = 0; i < L::Q; ++i) out[i] = rho;
  } else if constexpr (OP == 1 || OP == 2) {
    static_for<0, L::Q>([&](auto I) {
      constexpr int i = decltype(I)::value;
      constexpr int icx = L::cx[i], icy = L::cy[i], icz = L::cz[i], iwn = L::wn[i];
      const R cx = (R)icx, cy = (R)icy, cz = (R)icz;
      R phi;
      if constexpr (EQ == 0) {
        const R ics2 = R(3);
        const R cu = add(add(mul(cx, ux), mul(cy, uy)), mul(cz, uz));
        const R uu = add(add(mul(ux, ux), mul(uy, uy)), mul(uz, uz));
        phi = sub(add(mul(ics2, cu), mul(mul(R(4.5), cu), cu)), mul(R(1.5), uu));
      } else if constexpr (L::D == 2) {
        const R cs2v = R(1) / R(3);
        const R ax = sub(mul(cx, cx), cs2v), ay = sub(mul(cy, cy), cs2v);
        const R o1 = add(mul(cx, ux), mul(cy, uy)) / cs2v;
        const R o2 = add(add(mul(mul(ax, ux), ux), mul(mul(ay, uy), uy)),
                         mul(mul(mul(mul(R(2), cx), cy), ux), uy)) /
                     mul(mul(R(2), cs2v), cs2v);
        const R o3 = add(mul(mul(mul(mul(ax, cy), ux), ux), uy),
                         mul(mul(mul(mul(ay, cx), ux), uy), uy)) /
                     mul(mul(mul(R(2), cs2v), cs2v), cs2v);
        const R o4 = mul(mul(mul(mul(mul(ax, ay), ux), ux), uy), uy) /
                     mul(mul(mul(mul(R(4), cs2v), cs2v), cs2v), cs2v);
        phi = add(add(add(o1, o2), o3), o4);
      } else {
        constexpr int c3[3] = {icx, icy, icz};
        const R u3[3] = {ux, uy, uz};
        R ch[3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
          ch[a] = c3[a] == 0 ? sub(R(1), mul(mul(R(1.5), u3[a]), u3[a]))
                             : add(R(1), mul(mul(R(3), u3[a]), add((R)c3[a], u3[a])));
        phi = sub(mul(mul(ch[0], ch[1]), ch[2]), R(1));
      }
      const R w = (R)iwn / (R)L::WDEN;
      if constexpr (SH) {
        const R drho = sub(rho, R(1));
        out[i] = mul(w, add(drho, mul(add(R(1), drho), phi)));
      } else {
        out[i] = mul(mul(w, rho), add(R(1), phi));
      }
    });
  } else {
    // inverse transform of the equilibrium moments at u_b = 0
    constexpr int D = L::D;
    constexpr int NM = D == 3 ? 27 : 9;
    const R du[3] = {ux, uy, uz};
    R k[27];
#pragma unroll
    for (int n = 0; n < NM; ++n) {
      const int p = D == 3 ? n / 9 : n / 3, q = D == 3 ? (n / 3) % 3 : n % 3, r = D == 3 ? n % 3 : 0;
      const R Qx = p == 0 ? R(1) : (p == 1 ? du[0] : mul(du[0], du[0]));
      const R Qy = q == 0 ? R(1) : (q == 1 ? du[1] : mul(du[1], du[1]));
      const R Qz = r == 0 ? R(1) : (r == 1 ? du[2] : mul(du[2], du[2]));
      R e = mul(mul(rho, Qx), Qy);
      if (D == 3) e = mul(e, Qz);
      const R wv = (n == 0) ? R(1) : R(0);
      k[n] = SH ? sub(e, wv) : e;
    }
    const R cs2v = R(1) / R(3);
    auto inv0 = [&](R& a0, R& b0, R& c0) {
      const R m0 = a0, m1 = b0, m2 = c0;
      const R s1 = m1;
      const R s2 = sub(m2, mul(sub(R(0), cs2v), m0));
      a0 = mul(R(0.5), sub(s2, s1));
      b0 = sub(m0, s2);
      c0 = mul(R(0.5), add(s2, s1));
    };
    if constexpr (D == 3) {
#pragma unroll
      for (int qr = 0; qr < 9; ++qr) inv0(k[qr], k[9 + qr], k[18 + qr]);
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int r = 0; r < 3; ++r) inv0(k[a * 9 + r], k[a * 9 + 3 + r], k[a * 9 + 6 + r]);
#pragma unroll
      for (int ab = 0; ab < 9; ++ab) inv0(k[ab * 3], k[ab * 3 + 1], k[ab * 3 + 2]);
      static_for<0, 27>([&](auto NN) {
        constexpr int n = decltype(NN)::value;
        out[dir_of<L>(n / 9 - 1, (n / 3) % 3 - 1, n % 3 - 1)] = k[n];
      });
    } else {
#pragma unroll
      for (int q = 0; q < 3; ++q) inv0(k[q], k[3 + q], k[6 + q]);
#pragma unroll
      for (int a = 0; a < 3; ++a) inv0(k[a * 3], k[a * 3 + 1], k[a * 3 + 2]);
      static_for<0, 9>([&](auto NN) {
        constexpr int n = decltype(NN)::value;
        out[dir_of<L>(n / 3 - 1, n % 3 - 1, 0)] = k[n];
      });
    }
  }
}

// Does node coordinate v own slot target t = shift(v + c) when several nodes
// map onto t?  Only the clamped (non-periodic) axes can collide; the
// reference's sequential scatter leaves the value of the highest node index,
// i.e. the largest preimage on every axis.
__device__ __forceinline__ bool axis_winner(int v, int c, int t, int per, int s) {
  if (per || c == 0) return true;
  if (c > 0) return v == ((t == s - 1) ? s - 1 : t - 1);
  return v == ((t == 0) ? min(1, s - 1) : t + 1);
}


// One padded node of seed_kernel.
template <class L, int ST, int OP, int EQ, bool SH>
__device__ __forceinline__ void seed_node(const SeedArgs& a, int x, int y, int z) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const Geo& g = a.g;
  const long long n = ((long long)z * g.sy + y) * g.sx + x;
  // RegWall and SpecNode are fluid nodes and seed as such (FluidSolver.hpp:553-579)
  const bool fluid = a.flags[n] == 0 || a.flags[n] == kRegWall || a.flags[n] == kSpecNode;
  R rho = (R)a.rho0, ux = 0, uy = 0, uz = 0;
  if (a.mode == 0) {
    if (fluid) { ux = (R)a.ux0; uy = (R)a.uy0; uz = (R)a.uz0; }
  } else if (a.mode == 1) {
    rho = R(1);
    if (fluid) {
      const size_t k = ((size_t)(z - g.hz) * g.ny + (y - g.hy)) * g.nx + (x - g.hx);
      rho = reinterpret_cast<const R*>(a.rho)[k];
      ux = reinterpret_cast<const R*>(a.ux)[k];
      uy = reinterpret_cast<const R*>(a.uy)[k];
      uz = reinterpret_cast<const R*>(a.uz)[k];
    }
  }
  // neighbour coordinate one step down [0] / up [1] each axis
  int xn[2], yn[2], zn[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    xn[u] = shift_coord(x + 2 * u - 1, g.hx, g.nx, g.sx, g.px);
    yn[u] = shift_coord(y + 2 * u - 1, g.hy, g.ny, g.sy, g.py);
    zn[u] = shift_coord(z + 2 * u - 1, g.hz, g.nz, g.sz, g.pz);
  }
  const size_t own = slot<Q>(g, x, y, z, 0);
  const AxisSteps<Q> st = axis_steps<Q>(g, x, y, z);
  E* A = reinterpret_cast<E*>(a.f);
  const int P = a.parity;
  R sv[Q];
  if (a.mode != 2) seed_all<L, OP, EQ, SH, R>(rho, ux, uy, uz, sv);
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    if constexpr (i > 0 && (i & 1) == 0) {
      constexpr int cx = L::cx[i - 1], cy = L::cy[i - 1], cz = L::cz[i - 1];
      const int mx = cx == 0 ? x : xn[cx > 0], my = cy == 0 ? y : yn[cy > 0];
      const int mz = cz == 0 ? z : zn[cz > 0];
      if (!axis_winner(x, cx, mx, g.px, g.sx) || !axis_winner(y, cy, my, g.py, g.sy) ||
          !axis_winner(z, cz, mz, g.pz, g.sz))
        return;
    }
    const size_t s = load_slot_at<L, i>(own, st, P);
    if (a.mode == 2) {
      if (a.pops) A[s] = from_real<E>(a.pops[n * Q + i]);
      else A[s] = reinterpret_cast<const E*>(a.raw)[n * Q + i];
    } else {
      A[s] = from_real<E>(sv[i]);
    }
  });
}

template <class L, int ST, int OP, int EQ, bool SH>
__global__ void seed_kernel(SeedArgs a) {
  const Geo& g = a.g;
  const int x = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (x >= g.sx) return;
  for (RowWalk rw(g.sy); rw.z < g.sz; rw.next()) seed_node<L, ST, OP, EQ, SH>(a, x, rw.y, rw.z);
}

// gather_populations (FluidSolver.hpp:620-624, 1243-1253): logical
// populations of every padded node, as double or as raw storage elements.
template <class L, int ST>
__global__ void gather_kernel(Geo g, const void* f, int parity, double* out, void* raw) {
  using E = typename StoreT<ST>::elem;
  constexpr int Q = L::Q;
  const int x = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (x >= g.sx) return;
  const E* A = reinterpret_cast<const E*>(f);
  for (RowWalk rw(g.sy); rw.z < g.sz; rw.next()) {
    const int y = rw.y, z = rw.z;
    const long long n = ((long long)z * g.sy + y) * g.sx + x;
    const size_t own = slot<Q>(g, x, y, z, 0);
    const AxisSteps<Q> st = axis_steps<Q>(g, x, y, z);
    static_for<0, Q>([&](auto I) {
      constexpr int i = decltype(I)::value;
      const E e = A[load_slot_at<L, i>(own, st, parity)];
      if (out) out[n * Q + i] = (double)to_real(e);
      else reinterpret_cast<E*>(raw)[n * Q + i] = e;
    });
  }
}

// compute_macroscopic (FluidSolver.hpp:1041-1179): rho, u of every interior
// node at the current parity; non-fluid nodes report zeros.  One node:
template <class L, int ST, int OP, bool SH, bool FORCE>
__device__ __forceinline__ void macro_node(const StepArgs& a, int xi, int yi, int zi) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const Geo& g = a.g;
  const long long k = ((long long)zi * g.ny + yi) * g.nx + xi;
  const int x = xi + g.hx, y = yi + g.hy, z = zi + g.hz;
  R* rho = reinterpret_cast<R*>(a.rho);
  R* ux = reinterpret_cast<R*>(a.ux);
  R* uy = reinterpret_cast<R*>(a.uy);
  R* uz = reinterpret_cast<R*>(a.uz);
  const long long pn = ((long long)z * g.sy + y) * g.sx + x;
  const unsigned fl = a.flags ? a.flags[pn] : 0u;
  const bool spec_node = fl == kSpecNode && a.spec;
  if (fl != 0 && !spec_node) {
    rho[k] = ux[k] = uy[k] = uz[k] = R(0);
    return;
  }
  R f[Q];
  load_node<L>(reinterpret_cast<const E*>(a.f), g, x, y, z, a.parity, f);
  Macro<R> m;
  if (spec_node) {
    spec_node_mirror<L>(f, a.spec[pn]);
    m = spec_node_moments<L, OP, SH>(f);
  } else {
    m = macroscopic<L, OP, SH, FORCE>(f, node_params<FORCE, R>(a, (size_t)k));
  }
  rho[k] = m.rho; ux[k] = m.ux; uy[k] = m.uy; uz[k] = m.uz;
}

template <class L, int ST, int OP, bool SH, bool FORCE>
__global__ void macro_kernel(StepArgs a) {
  const Geo& g = a.g;
  const int xi = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (xi >= g.nx) return;
  for (RowWalk rw(g.ny); rw.z < g.nz; rw.next()) macro_node<L, ST, OP, SH, FORCE>(a, xi, rw.y, rw.z);
}

// ------------------------------------------------------------ reductions
// Global sums in FP64 (total_mass / total_momentum, FluidSolver.hpp:601-606,
// 1205-1229, plus kinetic energy and the sum over every stored slot).
// Stage 1 writes one partial per block into a scratch array, stage 2 sums
// the partials in a fixed order: no atomics, deterministic for a fixed grid.

__device__ __forceinline__ double block_sum(double v, double* sh) {
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

// Sum in FP64 of every stored slot (all padded rows and chunks, all
// directions, x < sx), this thread's share: 16-byte words t0, t0 + stride,
// ... of the population array in that order, each word's elements in lane
// order.  A word lies inside one 64-element segment (direction q of chunk ch
// of a row); its position advances by the stride's parts with carries.
template <int Q, class E>
__device__ __forceinline__ double slot_sum_part(const E* A, const Geo& g, long long t0,
                                                long long stride) {
  constexpr int EPW = 16 / (int)sizeof(E);  // elements per word
  constexpr int WPS = kChunk / EPW;         // words per segment
  const long long nw = (long long)g.sz * g.sy * g.nch * Q * WPS;
  const long long seg0 = t0 / WPS, sseg = stride / WPS;
  int sub = (int)(t0 % WPS), q = (int)(seg0 % Q), ch = (int)(seg0 / Q % g.nch);
  const int ss = (int)(stride % WPS), sq = (int)(sseg % Q), sc = (int)(sseg / Q % g.nch);
  const uint4* W = reinterpret_cast<const uint4*>(A);
  double acc = 0;
#pragma unroll 4
  for (long long w = t0; w < nw; w += stride) {
    const uint4 v = W[w];
    const E* e = reinterpret_cast<const E*>(&v);
    const int x0 = ch * kChunk + sub * EPW;
#pragma unroll
    for (int j = 0; j < EPW; ++j)
      if (x0 + j < g.sx) acc += (double)to_real(e[j]);
    sub += ss;
    const int c0 = sub >= WPS;
    sub -= c0 * WPS;
    q += sq + c0;
    const int c1 = q >= Q;
    q -= c1 * Q;
    ch += sc + c1;
    if (ch >= g.nch) ch -= g.nch;
  }
  return acc;
}

template <class L, int ST, int OP, bool SH, bool FORCE>
__global__ void __launch_bounds__(kReduceThreads)
reduce_kernel(StepArgs a, double* partials) {
  using E = typename StoreT<ST>::elem;
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  __shared__ double sh[kReduceThreads / 32];
  const Geo& g = a.g;
  const E* A = reinterpret_cast<const E*>(a.f);
  double acc[kReduceVals] = {0, 0, 0, 0, 0, 0};
  const long long nint = (long long)g.nx * g.ny * g.nz;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const CollideParams<R> prm{(R)a.omega, (R)a.omega2, (R)a.fx, (R)a.fy, (R)a.fz};
  // thread t sums nodes t, t + stride, ... in that order; the coordinates
  // advance by the stride's (x, y, z) parts with carries
  const long long k0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nxy = (long long)g.nx * g.ny;
  int xi = (int)(k0 % g.nx), yi = (int)((k0 / g.nx) % g.ny), zi = (int)(k0 / nxy);
  const int sxs = (int)(stride % g.nx), sys = (int)((stride / g.nx) % g.ny);
  const int szs = (int)(stride / nxy);
  for (long long k = k0; k < nint; k += stride) {
    const int x = xi + g.hx, y = yi + g.hy, z = zi + g.hz;
    xi += sxs;
    if (xi >= g.nx) { xi -= g.nx; ++yi; }
    yi += sys;
    if (yi >= g.ny) { yi -= g.ny; ++zi; }
    zi += szs;
    const long long pn = ((long long)z * g.sy + y) * g.sx + x;
    const unsigned fl = a.flags ? a.flags[pn] : 0u;
    const bool spec_node = fl == kSpecNode && a.spec;
    // fluid-like: Fluid, RegWall and SpecNode (FluidSolver.hpp:1215)
    if (fl != 0 && !spec_node && !(fl == kRegWall && a.spec)) continue;
    R f[Q];
    load_node<L>(A, g, x, y, z, a.parity, f);
    if (spec_node) spec_node_mirror<L>(f, a.spec[pn]);  // reduce, FluidSolver.hpp:1221-1222
    const Macro<R> m = macroscopic<L, OP, SH, FORCE>(f, FORCE ? node_params<FORCE, R>(a, (size_t)k) : prm);
    const double r = (double)m.rho, u = (double)m.ux, v = (double)m.uy, w = (double)m.uz;
    acc[0] += r;
    acc[1] += r * u;
    acc[2] += r * v;
    acc[3] += r * w;
    acc[4] += 0.5 * r * (u * u + v * v + w * w);
  }
  // every stored slot (all padded rows and chunks, all directions, x < sx)
  acc[5] = slot_sum_part<Q>(A, g, k0, stride);
#pragma unroll
  for (int v = 0; v < kReduceVals; ++v) {
    const double s = block_sum(acc[v], sh);
    if (threadIdx.x == 0) partials[(size_t)blockIdx.x * kReduceVals + v] = s;
  }
}

// The partials of `nvals` interleaved sums, added by one warp in a fixed
// order: lane l takes blocks l, l + 32, ..., then a fixed shuffle tree.
__device__ __forceinline__ void warp_fixed_sums(const double* partials, int nblocks, int nvals,
                                                double* out) {
  const int lane = threadIdx.x & 31;
  for (int v = 0; v < nvals; ++v) {
    double s = 0;
    for (int b = lane; b < nblocks; b += 32) s += partials[(size_t)b * nvals + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[v] = s;
  }
}

// Launched with one warp.
static __global__ void reduce_finish(const double* partials, int nblocks, double* out) {
  if (threadIdx.x < 32) warp_fixed_sums(partials, nblocks, kReduceVals, out);
}

}  // namespace m3lb
