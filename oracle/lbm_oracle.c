/*
 * CPU oracle for the M3LB lattice-Boltzmann time step -- TEST INFRASTRUCTURE
 * (see lbm_oracle.h).  Build: `make -C oracle oracle` (gcc, -ffp-contract=off).
 */
#include "lbm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Velocity sets in the Esoteric-Pull ordering: rest first, then opposite
 * pairs at adjacent indices (src/lattice/Lattices.hpp:75-159).  The order is
 * part of the storage contract, so it is the reference's order exactly. */
static const int D2Q9_CX[9] = {0, 1, -1, 0, 0, 1, -1, 1, -1};
static const int D2Q9_CY[9] = {0, 0, 0, 1, -1, 1, -1, -1, 1};
static const int D2Q9_W[9] = {16, 4, 4, 4, 4, 1, 1, 1, 1}; /* / 36 */
static const int D3Q27_CX[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1,
                                 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1};
static const int D3Q27_CY[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0,
                                 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1};
static const int D3Q27_CZ[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1,
                                 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1};
static const int D3Q27_W[27] = {64, 16, 16, 16, 16, 16, 16, 4, 4, 4, 4, 4, 4, 4,
                                4,  4,  4,  4,  4,  1,  1,  1, 1, 1, 1, 1, 1}; /* / 216 */

/* The scalar lattices D2Q5 (w /6, cs2 1/3) and D3Q7 (w /8, cs2 1/4):
 * rest, then the axis pairs (src/lattice/Lattices.hpp:51-70, 100-121). */
static const int D2Q5_C[2][5] = {{0, 1, -1, 0, 0}, {0, 0, 0, 1, -1}};
static const int D2Q5_W[5] = {2, 1, 1, 1, 1};
static const int D3Q7_C[3][7] = {{0, 1, -1, 0, 0, 0, 0}, {0, 0, 0, 1, -1, 0, 0}, {0, 0, 0, 0, 0, 1, -1}};
static const int D3Q7_W[7] = {2, 1, 1, 1, 1, 1, 1};
/* Their axis mirrors: the partner of each axis pair about its own axis. */
static const int D2Q5_MIR[3][5] = {{0, 2, 1, 3, 4}, {0, 1, 2, 4, 3}, {0, 1, 2, 3, 4}};
static const int D3Q7_MIR[3][7] = {{0, 2, 1, 3, 4, 5, 6}, {0, 1, 2, 4, 3, 5, 6}, {0, 1, 2, 3, 4, 6, 5}};

/* Direction index for component indices (velocity + 1), the product-basis
 * table pi() of src/collision/ProductBasis.hpp:118-131. */
static int D2Q9_DIR[3][3];
static int D3Q27_DIR[3][3][3];
static void build_dir_tables(void) {
  for (int i = 0; i < 9; ++i) D2Q9_DIR[D2Q9_CX[i] + 1][D2Q9_CY[i] + 1] = i;
  for (int i = 0; i < 27; ++i) D3Q27_DIR[D3Q27_CX[i] + 1][D3Q27_CY[i] + 1][D3Q27_CZ[i] + 1] = i;
}

/* Mirror tables m[axis][i]: the direction whose velocity is c_i with
 * component `axis` negated, i itself when there is none
 * (src/boundary/Specular.hpp:104-118). */
static int D2Q9_MIR[3][9];
static int D3Q27_MIR[3][27];
static void build_mirror_tables(void) {
  for (int a = 0; a < 3; ++a) {
    for (int i = 0; i < 9; ++i) {
      int c[3] = {D2Q9_CX[i], D2Q9_CY[i], 0};
      c[a] = -c[a];
      D2Q9_MIR[a][i] = (c[2] == 0) ? D2Q9_DIR[c[0] + 1][c[1] + 1] : i;
    }
    for (int i = 0; i < 27; ++i) {
      int c[3] = {D3Q27_CX[i], D3Q27_CY[i], D3Q27_CZ[i]};
      c[a] = -c[a];
      D3Q27_MIR[a][i] = D3Q27_DIR[c[0] + 1][c[1] + 1][c[2] + 1];
    }
  }
}
__attribute__((constructor)) static void lbmo_init(void) {
  build_dir_tables();
  build_mirror_tables();
}

/* Normal codes beyond the six axis walls (src/boundary/Regularized.hpp:97-105). */
enum { NRM_CORNER = 7, NRM_OUTXP = 8, NRM_OUTFREE = 9, NRM_OUTEQ = 10 };
enum { SB_BULK = 0, SB_ADIABATIC = 1, SB_DIRICHLET = 2, SB_EXCLUDED = 3, SB_MOMENT = 4,
       SB_OUTFLOW = 5, SB_SPECULAR = 6 };

/* float -> bfloat16 -> float, round to nearest even (NaN kept quiet). */
static inline float lbmo_bf16_round(float v) {
  uint32_t u;
  memcpy(&u, &v, 4);
  if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu)) {
    u |= 0x00400000u;
  } else {
    u += 0x7fffu + ((u >> 16) & 1u);
  }
  u &= 0xffff0000u;
  memcpy(&v, &u, 4);
  return v;
}

/* float -> FP16C -> float: the 16-bit float of the device's M3LB_STORE_F16C
 * (1 sign, 4 exponent bits with bias 15, 11 mantissa bits, subnormals),
 * rounded exactly as the device encodes it: the magnitude is clamped to
 * 2 - 2^-11 (NaN included), scaled by 2^-112 into FP32's subnormal/low
 * range where the format's code is the FP32 pattern's bits 26..12, rounded
 * there by adding half a unit of bit 12 (to nearest, ties away from zero),
 * and truncated. */
static inline float lbmo_f16c_round(float v) {
  const float m = fminf(fabsf(v), 1.99951171875f);
  const float t = m * 0x1p-112f;
  uint32_t u;
  memcpy(&u, &t, 4);
  u = ((u + 0x800u) >> 12) << 12;
  float d;
  memcpy(&d, &u, 4);
  d = d * 0x1p112f;
  return signbit(v) ? -d : d;
}

#define R double
#define P lbmo_f64_
#include "lbm_oracle_body.h"
#include "lbm_oracle_scalar.h"
#undef R
#undef P

#define R float
#define P lbmo_f32_
#include "lbm_oracle_body.h"
#include "lbm_oracle_scalar.h"
#undef R
#undef P
