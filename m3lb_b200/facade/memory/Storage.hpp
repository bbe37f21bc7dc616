// What the population arrays hold (names of src/memory/Storage.hpp):
// RawPopulations stores f_i, ShiftedPopulations stores g_i = f_i - w_i.
#pragma once

namespace lbm {
struct RawPopulations {
  static constexpr const char* name = "raw";
  static constexpr bool shifted = false;
};
struct ShiftedPopulations {
  static constexpr const char* name = "shifted";
  static constexpr bool shifted = true;
};
}  // namespace lbm
