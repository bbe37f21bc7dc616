// Host-side helpers shared by the C ABI translation units (lbm_capi.cu,
// lbm_serve.cu): storage sizes, geometry, launcher tables, error text.
#pragma once
#include <cstddef>

#include "lbm_launch.h"

namespace m3lb {

int elem_bytes(int storage);  // bytes per stored population, 0 if unknown
int real_bytes(int storage);  // bytes of the arithmetic type (macroscopic fields)
// Domain(nx, ny, nz, px, py, pz) geometry (src/grid/Domain.hpp:47-56, 104-108).
Geo make_geo(int nx, int ny, int nz, int px, int py, int pz);
int reduce_blocks(const Geo& g);
size_t pop_elems(const Geo& g, int Q);
const Launchers* table_for(int lattice, int storage);
// Message returned by m3lb_last_error() on the calling thread.
void set_last_error(const char* msg);

}  // namespace m3lb
