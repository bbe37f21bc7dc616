// Cartesian block (names and index rules of src/grid/Domain.hpp): halo only
// along non-periodic axes, periodic axes wrap, padded index
// idp = (pz*sy + py)*sx + px.  The rules fix which storage slots a node owns
// and what node indices passed to callbacks mean, so they are kept exactly.
#pragma once
#include <cstdio>
#include <cstdlib>

#include "core/Types.hpp"
#include "lattice/Lattices.hpp"

namespace lbm {

class Domain {
 public:
  Index nx = 1, ny = 1, nz = 1;
  Index hx = 0, hy = 0, hz = 0;
  Index sx = 1, sy = 1, sz = 1;
  Index n_padded = 1;
  bool periodic[3] = {true, true, true};

  Domain() = default;
  Domain(Index nx_, Index ny_, Index nz_ = 1, bool px = true, bool py = true, bool pz = true,
         Index mpi_halo = 0) {
    if (mpi_halo != 0) {
      std::fprintf(stderr, "Domain: mpi_halo is not offered by the B200 path\n");
      std::abort();
    }
    nx = nx_; ny = ny_; nz = nz_;
    periodic[0] = px; periodic[1] = py; periodic[2] = pz;
    hx = halo(nx, px); hy = halo(ny, py); hz = halo(nz, pz);
    sx = nx + 2 * hx; sy = ny + 2 * hy; sz = nz + 2 * hz;
    n_padded = sx * sy * sz;
  }

  Index n_interior() const { return nx * ny * nz; }
  Index idp(Index px, Index py, Index pz) const { return (pz * sy + py) * sx + px; }
  Index id(Index x, Index y, Index z = 0) const { return idp(x + hx, y + hy, z + hz); }
  void coords(Index n, Index& px, Index& py, Index& pz) const {
    px = n % sx;
    py = (n / sx) % sy;
    pz = n / (sx * sy);
  }
  bool is_interior(Index px, Index py, Index pz) const {
    return px >= hx && px < hx + nx && py >= hy && py < hy + ny && pz >= hz && pz < hz + nz;
  }

 private:
  static Index halo(Index n, bool per) { return n <= 1 ? 0 : (per ? 0 : 1); }
};

}  // namespace lbm
