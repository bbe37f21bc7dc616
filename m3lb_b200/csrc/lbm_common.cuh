// Lattice descriptors, storage formats and the arithmetic vocabulary shared by
// every kernel of the M3LB lattice-Boltzmann step on sm_100a.
//
// Velocity sets keep the reference's Esoteric-Pull ordering
// (src/lattice/Lattices.hpp:75-159): rest first, then opposite directions at
// adjacent indices, opp(i) = i+1 for odd i.  The order is part of the storage
// contract (it decides which slot a population sits in), so it is the
// reference's order exactly.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace m3lb {

// ---------------------------------------------------------------- lattices
struct D2Q9 {
  static constexpr int Q = 9, D = 2, WDEN = 36, CS2D = 3;
  static constexpr int cx[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
  static constexpr int cy[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
  static constexpr int cz[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  static constexpr int wn[9] = {16, 4, 4, 4, 4, 1, 1, 1, 1};
};
struct D3Q27 {
  static constexpr int Q = 27, D = 3, WDEN = 216, CS2D = 3;
  static constexpr int cx[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1,
                                 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
  static constexpr int cy[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0,
                                 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
  static constexpr int cz[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1,
                                 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
  static constexpr int wn[27] = {64, 16, 16, 16, 16, 16, 16, 4, 4, 4, 4, 4, 4, 4,
                                 4,  4,  4,  4,  4,  1,  1,  1, 1, 1, 1, 1, 1};
};

// Scalar (advection-diffusion) lattices (src/lattice/Lattices.hpp:51-70,
// 100-121): rest, then the axis pairs; cs2 = 1 / CS2D.
struct D2Q5 {
  static constexpr int Q = 5, D = 2, WDEN = 6, CS2D = 3;
  static constexpr int cx[5] = {0, 1, -1, 0, 0};
  static constexpr int cy[5] = {0, 0, 0, 1, -1};
  static constexpr int cz[5] = {0, 0, 0, 0, 0};
  static constexpr int wn[5] = {2, 1, 1, 1, 1};
};
struct D3Q7 {
  static constexpr int Q = 7, D = 3, WDEN = 8, CS2D = 4;
  static constexpr int cx[7] = {0, 1, -1, 0, 0, 0, 0};
  static constexpr int cy[7] = {0, 0, 0, 1, -1, 0, 0};
  static constexpr int cz[7] = {0, 0, 0, 0, 0, 1, -1};
  static constexpr int wn[7] = {2, 1, 1, 1, 1, 1, 1};
};

template <class L>
__host__ __device__ constexpr int cvel(int i, int a) {
  return a == 0 ? L::cx[i] : (a == 1 ? L::cy[i] : L::cz[i]);
}
// Direction with the given velocity components (each in -1..1), or -1.
template <class L>
__host__ __device__ constexpr int dir_of(int x, int y, int z) {
  for (int i = 0; i < L::Q; ++i)
    if (L::cx[i] == x && L::cy[i] == y && L::cz[i] == z) return i;
  return -1;
}

// ---------------------------------------------------------- storage formats
// Population storage: the element type in HBM.  Arithmetic is FP32 for the
// 32- and 16-bit formats and FP64 for the 64-bit one.  kF16C is the 16-bit
// float below with one more mantissa bit than IEEE binary16.
enum Store : int { kF32 = 0, kF16 = 1, kBF16 = 2, kF64 = 3, kF16C = 4 };

// FP16C element: 1 sign bit, 4 exponent bits (bias 15), 11 mantissa bits,
// subnormals, no infinities or NaN (codec below).
struct f16c { uint16_t bits; };

template <int S> struct StoreT;
template <> struct StoreT<kF32> {
  using elem = float;  using word = float2;  using real = float;  using half_word = float;
};
template <> struct StoreT<kF64> {
  using elem = double; using word = double2; using real = double; using half_word = double;
};
template <> struct StoreT<kF16> {
  using elem = __half; using word = uint32_t; using real = float; using half_word = uint16_t;
};
template <> struct StoreT<kBF16> {
  using elem = __nv_bfloat16; using word = uint32_t; using real = float; using half_word = uint16_t;
};
template <> struct StoreT<kF16C> {
  using elem = f16c; using word = uint32_t; using real = float; using half_word = uint16_t;
};

// ------------------------------------------------------ packed arithmetic
// Two adjacent nodes are updated together with sm_100's paired FP32 ops
// (add/mul/fma .f32x2), one instruction for both lanes.  Every operation is
// an explicitly rounded IEEE op, so the paired path and the one-node path
// give bitwise identical results.  One exception had to be written around:
// a paired product whose only use is a paired add can be fused into one
// f32x2 FMA by the compiler (seen with both the __fmul2_rn / __fadd2_rn
// intrinsics and the `.rn` PTX below), one rounding instead of two, which the
// scalar __fmul_rn / __fadd_rn never are.  The one place the operators had
// that shape (the -cs2 * rho term of the second-order central moments,
// lbm_collide.cuh) is written as an explicit FMA in both paths.
struct f2 { float2 v; };

__device__ __forceinline__ unsigned long long f2_bits(float2 v) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(v.x), "f"(v.y));
  return r;
}
__device__ __forceinline__ float2 f2_of_bits(unsigned long long r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_of_bits(d);
}
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_of_bits(d);
}
__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return f2_of_bits(d);
}

__device__ __forceinline__ f2 mk(float a, float b) { return f2{make_float2(a, b)}; }
__device__ __forceinline__ f2 splat2(float a) { return f2{make_float2(a, a)}; }
__device__ __forceinline__ f2 add(f2 a, f2 b) { return f2{add2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 mul(f2 a, f2 b) { return f2{mul2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2 fma(f2 a, f2 b, f2 c) { return f2{fma2_rn(a.v, b.v, c.v)}; }
// a - b as a + (-1)*b in one fused op: exactly the IEEE difference.
__device__ __forceinline__ f2 sub(f2 a, f2 b) { return f2{fma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }
__device__ __forceinline__ f2 neg(f2 a) { return f2{make_float2(-a.v.x, -a.v.y)}; }
__device__ __forceinline__ f2 rcp(f2 a) { return f2{make_float2(__frcp_rn(a.v.x), __frcp_rn(a.v.y))}; }

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float sub(float a, float b) { return __fmaf_rn(b, -1.f, a); }
__device__ __forceinline__ float neg(float a) { return -a; }
__device__ __forceinline__ float rcp(float a) { return __frcp_rn(a); }

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double sub(double a, double b) { return __fma_rn(b, -1.0, a); }
__device__ __forceinline__ double neg(double a) { return -a; }
__device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }

template <class V> struct Lanes;
template <> struct Lanes<f2> { using S = float; static constexpr int N = 2; };
template <> struct Lanes<float> { using S = float; static constexpr int N = 1; };
template <> struct Lanes<double> { using S = double; static constexpr int N = 1; };

template <class V> __device__ __forceinline__ V bc(typename Lanes<V>::S a);
template <> __device__ __forceinline__ f2 bc<f2>(float a) { return splat2(a); }
template <> __device__ __forceinline__ float bc<float>(float a) { return a; }
template <> __device__ __forceinline__ double bc<double>(double a) { return a; }

// Lane access for the paired type (lane 0 = lower x).
__device__ __forceinline__ float lane_of(f2 a, int k) { return k ? a.v.y : a.v.x; }
__device__ __forceinline__ float lane_of(float a, int) { return a; }
__device__ __forceinline__ double lane_of(double a, int) { return a; }

// -------------------------------------------- word <-> paired conversion
// A "word" is the storage of two x-adjacent nodes of one direction.
__device__ __forceinline__ f2 unpack(float2 w) { return f2{w}; }
__device__ __forceinline__ float2 pack_f32(f2 v) { return v.v; }

__device__ __forceinline__ f2 unpack_f16(uint32_t w) {
  __half2 h = *reinterpret_cast<__half2*>(&w);
  return f2{__half22float2(h)};
}
__device__ __forceinline__ uint32_t pack_f16(f2 v) {
  __half2 h = __float22half2_rn(v.v);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ f2 unpack_bf16(uint32_t w) {
  return f2{make_float2(__uint_as_float(w << 16), __uint_as_float(w & 0xffff0000u))};
}
__device__ __forceinline__ uint32_t pack_bf16(f2 v) {
  __nv_bfloat162 h = __float22bfloat162_rn(v.v);
  return *reinterpret_cast<uint32_t*>(&h);
}

// FP16C: a 16-bit float for shifted populations that gives IEEE binary16's
// top exponent bit to the mantissa (the customised 16-bit number format of
// Lehmann et al. 2022, "Accuracy and performance of the lattice Boltzmann
// method with 64-bit, 32-bit, and customized 16-bit number formats"):
// 1 sign bit, 4 exponent bits with bias 15, 11 mantissa bits and subnormals;
// largest magnitude 2 - 2^-11, smallest normal 2^-14, subnormal step 2^-25;
// no infinities or NaN.  Shifted populations f - w stay far inside |x| < 2,
// so the range IEEE binary16 spends above 2 buys nothing here, while the
// extra mantissa bit halves every stored rounding error.  Encoding rounds to
// nearest with ties away from zero and saturates larger magnitudes (and NaN)
// at +-(2 - 2^-11).
//
// Codec through the FP32 bit pattern.  Scaled by 2^-112, a value of the
// format is exactly the FP32 number with bits  sign | code << 12  (the
// format's exponent bias 15 is FP32's 127 - 112, and its subnormals are FP32
// subnormals), so decoding is an arithmetic shift, a mask and a multiply by
// 2^112 (paired for the two values of a word), and encoding a clamp of the
// magnitude, a multiply by 2^-112, one integer multiply-add that shifts the
// code into the top half and adds the rounding bit, the sign, and one byte
// permute that packs the two codes.
constexpr float kF16CMax = 1.99951171875f;  // 2 - 2^-11
constexpr float kF16CUp = 0x1p112f;
constexpr float kF16CDown = 0x1p-112f;

// FP32 bits of the scaled value of the code in bits 31..16 of w
__device__ __forceinline__ uint32_t f16c_hi_bits(uint32_t w) {
  return (uint32_t)((int32_t)w >> 4) & 0x87fff000u;
}
// The code of the scaled magnitude bits t (FP32 bits of |x| 2^-112), rounded,
// in bits 30..16, with the sign of x in bit 31; bits 15..0 are rounding
// residue
__device__ __forceinline__ uint32_t f16c_code_hi(uint32_t t, float x) {
  return (t * 16u + 0x8000u) | (__float_as_uint(x) & 0x80000000u);
}
__device__ __forceinline__ f2 unpack_f16c(uint32_t w) {
  const float a = __uint_as_float(f16c_hi_bits(w << 16));
  const float b = __uint_as_float(f16c_hi_bits(w));
  return f2{mul2_rn(make_float2(a, b), make_float2(kF16CUp, kF16CUp))};
}
__device__ __forceinline__ uint32_t pack_f16c(f2 v) {
  const float2 m = make_float2(fminf(fabsf(v.v.x), kF16CMax), fminf(fabsf(v.v.y), kF16CMax));
  const float2 t = mul2_rn(m, make_float2(kF16CDown, kF16CDown));
  return __byte_perm(f16c_code_hi(__float_as_uint(t.x), v.v.x),
                     f16c_code_hi(__float_as_uint(t.y), v.v.y), 0x7632);
}
__device__ __forceinline__ float f16c_to_float(uint16_t c) {
  return __fmul_rn(__uint_as_float(f16c_hi_bits((uint32_t)c << 16)), kF16CUp);
}
__device__ __forceinline__ uint16_t f16c_from_float(float x) {
  const float t = __fmul_rn(fminf(fabsf(x), kF16CMax), kF16CDown);
  return (uint16_t)(f16c_code_hi(__float_as_uint(t), x) >> 16);
}

// Scalar element <-> arithmetic type.
__device__ __forceinline__ float to_real(float e) { return e; }
__device__ __forceinline__ double to_real(double e) { return e; }
__device__ __forceinline__ float to_real(__half e) { return __half2float(e); }
__device__ __forceinline__ float to_real(__nv_bfloat16 e) { return __bfloat162float(e); }
__device__ __forceinline__ float to_real(f16c e) { return f16c_to_float(e.bits); }
template <class E> __device__ __forceinline__ E from_real(float v);
template <class E> __device__ __forceinline__ E from_real(double v);
template <> __device__ __forceinline__ float from_real<float>(float v) { return v; }
template <> __device__ __forceinline__ double from_real<double>(double v) { return v; }
template <> __device__ __forceinline__ __half from_real<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_real<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <> __device__ __forceinline__ f16c from_real<f16c>(float v) { return f16c{f16c_from_float(v)}; }
template <> __device__ __forceinline__ f16c from_real<f16c>(double v) {
  return f16c{f16c_from_float((float)v)};
}
template <> __device__ __forceinline__ double from_real<double>(float v) { return (double)v; }
template <> __device__ __forceinline__ float from_real<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ __half from_real<__half>(double v) { return __double2half(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_real<__nv_bfloat16>(double v) {
  return __double2bfloat16(v);
}

// ------------------------------------------------------------ geometry
// Padded block, x fastest, with a halo only along non-periodic axes
// (src/grid/Domain.hpp:37-56).  Populations are stored in x-chunks of
// kChunk = 64 nodes: every padded row (y, z) is cut into nch chunks, and a
// chunk holds its Q direction segments one after the other:
//   element (x, y, z, q) at (((z*sy + y)*nch + x/64)*Q + q)*64 + x%64.
// One warp updates one chunk (32 lanes x 2 nodes), so each of its loads and
// stores is one contiguous segment, and every direction sits at a
// compile-time offset from the chunk start.
constexpr int kChunk = 64;

struct Geo {
  int nx, ny, nz;     // interior extents
  int hx, hy, hz;     // halo widths
  int sx, sy, sz;     // padded extents
  int px, py, pz;     // periodic flags
  int nch;            // chunks per padded row, ceil(sx / 64)
  long long n_padded; // sx*sy*sz
};

// Neighbour coordinate along one axis: periodic axes wrap inside [h, h+n),
// others clamp into the padded range (Domain.hpp:113-123).
__host__ __device__ __forceinline__ int shift_coord(int v, int h, int n, int s, int per) {
  if (per) {
    if (v < h) return v + n;
    if (v >= h + n) return v - n;
    return v;
  }
  if (v < 0) return 0;
  if (v >= s) return s - 1;
  return v;
}

// Cell types (src/boundary/Flags.hpp:20-32): 0 Fluid, 1 Solid, 2 Excluded,
// 3 RegWall (regularised on-node wall), 4 SpecWall (free-slip ghost),
// 5 SpecNode (on-node free slip).
constexpr uint8_t kRegWall = 3, kSpecWall = 4, kSpecNode = 5;

// Parameters of one step launch, passed by value.
struct StepArgs {
  Geo g;
  void* f;                 // populations
  const uint8_t* flags;    // per padded node (0 fluid); nullptr: all interior fluid
  const uint8_t* row_flags;  // per padded row (pz * sy + py): 1 when a node of the row
                             // is not fluid; nullptr: test every row's flags
  const uint8_t* spec;     // per padded node: SpecWall normal code / SpecNode face mask;
                           // nullptr: no wall nodes (flags 3, 4 and 5 then act as solid)
  void* rho;               // macroscopic outputs, per padded node, or nullptr
  void* ux;
  void* uy;
  void* uz;
  int parity;              // t % 2
  double omega, omega2;    // BGK/TRT/MRT/CM rates (TRT: omega_p, omega_m; moments: omega, bulk)
  double fx, fy, fz;       // uniform Guo body force
  int* err;                // device status word: a kernel whose bounded wait ran out sets it
  long long wait_cycles;   // limit of the row kernel's wait for a row's copies (0: ~2 s);
                           // shorter only to test the timeout path
  // Boussinesq buoyancy (BoussinesqGuo, src/forcing/Forcing.hpp:93-127): the
  // force at a node is (fx, fy, fz) + g rho0 beta (T - T0) with T per
  // interior node in the arithmetic type; temp == nullptr: (fx, fy, fz) alone
  const void* temp;
  double bgx, bgy, bgz, brho0, bbeta, bT0;
};

// ------------------------------------------------------------- wall nodes
// Regularised-wall normal codes beyond the six axis walls
// (src/boundary/Regularized.hpp:97-105) and the compact list of wall nodes
// the boundary pass updates (lbm_bound.cuh).
enum : uint8_t { kNrmCorner = 7, kNrmOutXp = 8, kNrmOutFree = 9, kNrmOutEq = 10 };
constexpr int kBndRefs = 6;
constexpr int kBndThreads = 128;

// One wall node of the list.
struct BNode {
  long long n;                 // padded index
  long long ref[kBndRefs];     // nodes this one reads (padded index), -1 unused:
                               //   outflow donor / upstream 1, 2; corner stencil 2a, 2a+1
  int ref_wall[kBndRefs];      // list position when the read is a wall node's state velocity
  int snap[kBndRefs];          // snapshot slot when the read precedes the node's update, else -1
  int c1, c2;                  // corner: list positions of the extrapolation nodes, -1 none
  uint32_t unk;                // RegWall: directions whose source is outside the fluid
  uint8_t type;                // kRegWall / kSpecWall / kSpecNode
  uint8_t code;                // RegWall normal code, SpecWall normal code, SpecNode face mask
  uint8_t onrm;                // NrmOutFree: outward normal of the donor axis
  int8_t fd_dir[3];            // corner stencil per axis: +1 / -1 one-sided, 0 centred, 2 unused
  double u[4];                 // wall state as given: ux, uy, uz, rho
  double un[3];                // per-node wall velocity field
};

// The fields of a list node that every update reads, in a separate array of
// 16-byte entries, so a warp reads those of its 32 consecutive nodes in one
// coalesced request (a BNode is 184 bytes; reading single fields of 32 of
// them touches a sector per node and field).
struct alignas(16) BHead {
  long long n;       // padded index (BNode::n)
  uint32_t unk;      // BNode::unk
  uint8_t type;      // BNode::type
  uint8_t code;      // BNode::code
  uint8_t moving;    // a bit of u[0..2] or un[0..2] is set: the wall velocity is read
  uint8_t pad;
};

struct BoundArgs {
  const BNode* nodes;
  const BHead* heads;          // one per list node, same order
  int begin, end;              // list positions of this launch
  void* wall_rho;              // arithmetic type, one per list node (corner densities)
  void* snap;                  // arithmetic type, Q per snapshot slot
  double scale;                // set_wall_velocity_scale
  double field_scale;          // set_wall_velocity_field_scale
  int field_on;                // per-node wall velocity field in use
  int fd_corners;              // corner stress from velocity gradients
  int force_bc;                // Guo corrections of the reconstruction
  int out_order;               // tangential extrapolation order at NrmOutXp
  double out_rho;              // NrmOutFree target density
};

// Scatter (Access::scatter, EsotericPull.hpp:104-111): write, for node n and
// direction i, the slot that load(n, i) reads.  mode 0: equilibrium at
// (rho0, u0) on fluid nodes and at rest elsewhere (initialize,
// FluidSolver.hpp:553-561); mode 1: per-node interior field arrays, rest at
// rho = 1 elsewhere (initialize_field :568-579); mode 2: explicit logical
// populations per padded node (seed_populations :634-637), as double or raw.
struct SeedArgs {
  Geo g;
  void* f;
  const uint8_t* flags;   // per padded node, never null here
  int parity;
  int mode;
  double rho0, ux0, uy0, uz0;
  const void* rho;        // mode 1: interior arrays of the arithmetic type
  const void* ux;
  const void* uy;
  const void* uz;
  const double* pops;     // mode 2 (double)
  const void* raw;        // mode 2 (storage elements), used when pops == nullptr
};

// Global reductions: threads per block and values per block partial (mass,
// momentum x/y/z, kinetic energy, sum of every stored slot).
constexpr int kReduceThreads = 256;
constexpr int kReduceVals = 6;

}  // namespace m3lb
