// Cell types (src/boundary/Flags.hpp).  The B200 path runs Fluid, Solid
// (halfway bounce-back) and Excluded cells; the others are rejected at
// set_geometry.
#pragma once
#include <cstdint>

namespace lbm {
enum CellType : std::uint8_t {
  Fluid = 0,
  Solid = 1,
  Excluded = 2,
  RegWall = 3,
  SpecWall = 4,
  SpecNode = 5,
};
}  // namespace lbm
