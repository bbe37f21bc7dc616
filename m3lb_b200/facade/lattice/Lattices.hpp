// Velocity sets (names of src/lattice/Lattices.hpp).  The ordering -- rest
// first, opposite directions at adjacent indices -- fixes which storage slot
// each population occupies, so it is the reference's ordering exactly.
#pragma once
#include <cstdint>

#define LBM_FN inline

namespace lbm {

LBM_FN constexpr int opp(int i) noexcept { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

namespace facade_tables {
constexpr int d2q9_c[3][9] = {{0, 1, -1, 0, 0, 1, -1, 1, -1},
                              {0, 0, 0, 1, -1, 1, -1, -1, 1},
                              {0, 0, 0, 0, 0, 0, 0, 0, 0}};
constexpr int d2q9_w[9] = {16, 4, 4, 4, 4, 1, 1, 1, 1};
constexpr int d3q27_c[3][27] = {
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1},
    {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1}};
constexpr int d3q27_w[27] = {64, 16, 16, 16, 16, 16, 16, 4, 4, 4, 4, 4, 4, 4,
                             4,  4,  4,  4,  4,  1,  1,  1, 1, 1, 1, 1, 1};
}  // namespace facade_tables

struct D2Q9 {
  static constexpr const char* name = "D2Q9";
  static constexpr int D = 2, Q = 9;
  static constexpr int cs2_num = 1, cs2_den = 3;
  static constexpr int w_den = 36;
  static constexpr bool supports_navier_stokes = true;
  LBM_FN static constexpr int cx(int i) noexcept { return facade_tables::d2q9_c[0][i]; }
  LBM_FN static constexpr int cy(int i) noexcept { return facade_tables::d2q9_c[1][i]; }
  LBM_FN static constexpr int w_num(int i) noexcept { return facade_tables::d2q9_w[i]; }
};

struct D3Q27 {
  static constexpr const char* name = "D3Q27";
  static constexpr int D = 3, Q = 27;
  static constexpr int cs2_num = 1, cs2_den = 3;
  static constexpr int w_den = 216;
  static constexpr bool supports_navier_stokes = true;
  LBM_FN static constexpr int cx(int i) noexcept { return facade_tables::d3q27_c[0][i]; }
  LBM_FN static constexpr int cy(int i) noexcept { return facade_tables::d3q27_c[1][i]; }
  LBM_FN static constexpr int cz(int i) noexcept { return facade_tables::d3q27_c[2][i]; }
  LBM_FN static constexpr int w_num(int i) noexcept { return facade_tables::d3q27_w[i]; }
};

// Scalar lattices: advection-diffusion only (no Navier-Stokes).
namespace facade_tables {
constexpr int d2q5_c[2][5] = {{0, 1, -1, 0, 0}, {0, 0, 0, 1, -1}};
constexpr int d3q7_c[3][7] = {{0, 1, -1, 0, 0, 0, 0}, {0, 0, 0, 1, -1, 0, 0}, {0, 0, 0, 0, 0, 1, -1}};
constexpr int scalar_w[7] = {2, 1, 1, 1, 1, 1, 1};
}  // namespace facade_tables
struct D2Q5 {
  static constexpr const char* name = "D2Q5";
  static constexpr int D = 2, Q = 5;
  static constexpr int cs2_num = 1, cs2_den = 3;
  static constexpr int w_den = 6;
  static constexpr bool supports_navier_stokes = false;
  LBM_FN static constexpr int cx(int i) noexcept { return facade_tables::d2q5_c[0][i]; }
  LBM_FN static constexpr int cy(int i) noexcept { return facade_tables::d2q5_c[1][i]; }
  LBM_FN static constexpr int w_num(int i) noexcept { return facade_tables::scalar_w[i]; }
};
struct D3Q7 {
  static constexpr const char* name = "D3Q7";
  static constexpr int D = 3, Q = 7;
  static constexpr int cs2_num = 1, cs2_den = 4;
  static constexpr int w_den = 8;
  static constexpr bool supports_navier_stokes = false;
  LBM_FN static constexpr int cx(int i) noexcept { return facade_tables::d3q7_c[0][i]; }
  LBM_FN static constexpr int cy(int i) noexcept { return facade_tables::d3q7_c[1][i]; }
  LBM_FN static constexpr int cz(int i) noexcept { return facade_tables::d3q7_c[2][i]; }
  LBM_FN static constexpr int w_num(int i) noexcept { return facade_tables::scalar_w[i]; }
};

template <class L, class T> LBM_FN constexpr T weight(int i) noexcept {
  return static_cast<T>(L::w_num(i)) / static_cast<T>(L::w_den);
}
template <class L, class T> LBM_FN constexpr T cs2() noexcept {
  return static_cast<T>(L::cs2_num) / static_cast<T>(L::cs2_den);
}
template <class L, class T> LBM_FN constexpr T inv_cs2() noexcept {
  return static_cast<T>(L::cs2_den) / static_cast<T>(L::cs2_num);
}
template <class L> LBM_FN constexpr int cvel(int i, int a) noexcept {
  if (a == 0) return L::cx(i);
  if (a == 1) return L::cy(i);
  if constexpr (L::D == 3) return L::cz(i);
  else return 0;
}

// Which lattices the device path runs.
template <class L> struct DeviceLattice { static constexpr int code = 0; };
template <> struct DeviceLattice<D2Q9> { static constexpr int code = 9; };
template <> struct DeviceLattice<D3Q27> { static constexpr int code = 27; };

}  // namespace lbm
