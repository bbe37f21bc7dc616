// Wall normal codes (names and values of src/boundary/Regularized.hpp:97-105).
// The B200 path takes the axis codes for free-slip ghost walls
// (set_specular_walls); the regularised velocity wall itself (RegWall) is not
// offered, so only the codes and normal_of are declared here.
#pragma once
#include <cstdint>

namespace lbm {

enum NormalCode : std::uint8_t {
  NrmNone = 0,
  NrmXp = 1,
  NrmXm = 2,
  NrmYp = 3,
  NrmYm = 4,
  NrmZp = 5,
  NrmZm = 6,
  NrmCorner = 7,
  NrmOutXp = 8,
  NrmOutFree = 9,
  NrmOutEq = 10,
};

// Outward unit normal of a code (zero for none, corner and the outflow codes
// other than NrmOutXp, whose outward normal is +x).
inline constexpr void normal_of(std::uint8_t code, int n[3]) {
  const int axis = (code >= NrmXp && code <= NrmZm) ? (code - 1) / 2 : (code == NrmOutXp ? 0 : -1);
  const int sign = (code >= NrmXp && code <= NrmZm) ? ((code & 1) ? 1 : -1) : 1;
  for (int a = 0; a < 3; ++a) n[a] = (a == axis) ? sign : 0;
}

}  // namespace lbm
