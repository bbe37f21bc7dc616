// Free-slip (specular) walls: the names of src/boundary/Specular.hpp, for
// host code that builds masks or checks the mirror on a population vector.
// On the device the same reflections run inside the step (SpecWall: whole
// incoming set mirrored about one axis, no collision; SpecNode: the unknown
// directions mirrored, composed over the masked faces, then collision).
#pragma once
#include <cstdint>

#include "boundary/Regularized.hpp"
#include "lattice/Lattices.hpp"

namespace lbm {

// m[a][i]: the direction whose velocity is c_i with component a negated
// (i itself where the lattice has none).
template <class L>
struct MirrorTable {
  static constexpr int Q = L::Q;
  int m[3][Q];
  constexpr MirrorTable() : m{} {
    for (int a = 0; a < 3; ++a)
      for (int i = 0; i < Q; ++i) {
        m[a][i] = i;
        for (int j = 0; j < Q; ++j) {
          bool same = true;
          for (int b = 0; b < 3; ++b)
            same = same && cvel<L>(j, b) == (b == a ? -cvel<L>(i, b) : cvel<L>(i, b));
          if (same) { m[a][i] = j; break; }
        }
      }
  }
};
template <class L>
inline constexpr MirrorTable<L> mirror_table{};

// Axis a normal code mirrors about: 0 for +-x, 1 for +-y, 2 otherwise.
inline constexpr int mirror_axis(std::uint8_t code) {
  return (code == NrmXp || code == NrmXm) ? 0 : ((code == NrmYp || code == NrmYm) ? 1 : 2);
}

enum SpecFace : std::uint8_t {
  SpecNone = 0,
  SpecXp = 1u << 0,
  SpecXm = 1u << 1,
  SpecYp = 1u << 2,
  SpecYm = 1u << 3,
  SpecZp = 1u << 4,
  SpecZm = 1u << 5,
};

// Outward sign of a mask on axis a: +1, -1, or 0 when the axis is free (the
// + face is read first; a mask with both is rejected by set_specular_nodes).
inline constexpr int face_sign(std::uint8_t faces, int a) {
  return ((faces >> (2 * a)) & 1u) ? 1 : (((faces >> (2 * a + 1)) & 1u) ? -1 : 0);
}

// The mask of a single normal code.
inline constexpr std::uint8_t faces_of_normal(std::uint8_t code) {
  int n[3];
  normal_of(code, n);
  unsigned m = 0;
  for (int a = 0; a < 3; ++a)
    m |= n[a] > 0 ? (1u << (2 * a)) : (n[a] < 0 ? (1u << (2 * a + 1)) : 0u);
  return std::uint8_t(m);
}

// Replace every direction that points into the domain across a masked face
// by its image, reflected in every masked plane it crosses; the others keep
// their values.
template <class L, class R>
inline void mirror_unknowns_faces(R* f, std::uint8_t faces) {
  R in[L::Q];
  for (int i = 0; i < L::Q; ++i) in[i] = f[i];
  for (int i = 0; i < L::Q; ++i) {
    int j = i;
    for (int a = 0; a < 3; ++a)
      if (cvel<L>(i, a) * face_sign(faces, a) < 0) j = mirror_table<L>.m[a][j];
    f[i] = in[j];
  }
}

// The single-normal form: the unknowns of one outward normal.
template <class L, class R>
inline void mirror_unknowns(R* g, std::uint8_t code) {
  mirror_unknowns_faces<L>(g, faces_of_normal(code));
}

}  // namespace lbm
