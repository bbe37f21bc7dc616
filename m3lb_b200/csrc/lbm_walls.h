// Host side of the wall nodes: the regularised-wall setup of
// FluidSolver::set_regularized_walls (FluidSolver.hpp:372-552) and the free-slip
// marks, turned into the compact device list the boundary pass runs over
// (lbm_bound.cuh).  Owned by one solver handle.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <unordered_map>
#include <vector>

#include "lbm_launch.h"

namespace m3lb {

// One RegWall node as set up (per padded node; the reference's bc_nrm,
// bc_ext, bc_unk, bc_don, bc_onrm and the node's wall state).
struct WallHost {
  uint8_t code = 0;   // normal code
  uint8_t ext = 0;    // corner: 1 + index of the extrapolation direction, 0 none
  uint8_t onrm = 0;   // NrmOutFree: outward normal code of the donor axis
  uint32_t unk = 0;   // directions whose source is outside the fluid
  long long don = 0;  // NrmOutFree donor (padded index; the node itself when none)
  double u[4] = {0, 0, 0, 1};  // ux, uy, uz, rho as given
};

class WallSet {
 public:
  // ---- host state
  std::vector<uint8_t> spec_nrm, spec_faces;       // per padded node, empty until set
  std::unordered_map<long long, WallHost> reg;     // RegWall nodes by padded index
  std::vector<double> field;                       // per-node wall velocity, 3 per interior node
  bool field_on = false;
  double scale = 1, field_scale = 1, out_rho = 1;
  int fd_corners = 1, force_bc = 1, out_order = 1;

  // ---- device list (rebuilt by build())
  BNode* nodes = nullptr;
  BHead* heads = nullptr;     // the hot fields of `nodes`, one per list node
  void* wall_rho = nullptr;   // arithmetic type, one per list node
  void* snap = nullptr;       // arithmetic type, Q per snapshot slot
  uint8_t* spec = nullptr;    // per padded node: SpecWall code / SpecNode mask
  int count = 0, nsnap = 0;
  bool corners = false;
  std::vector<int> level_end; // list positions where each level ends

  WallSet() = default;
  WallSet(const WallSet&) = delete;
  WallSet& operator=(const WallSet&) = delete;
  ~WallSet() { release(); }
  void release();

  // set_regularized_walls: codes (and states, 4 per node, or null) per
  // interior node; marks the coded nodes RegWall in `flags` (per padded
  // node).  Returns an M3LB_* status.
  int set_regularized(const Geo& g, int lattice, std::vector<uint8_t>& flags, const uint8_t* codes,
                      const double* states);
  // Rebuild the device list from the flags; uploads on `s` and waits.
  int build(const Geo& g, int lattice, int op, int storage, const std::vector<uint8_t>& flags,
            cudaStream_t s);
  BoundArgs args(int begin, int end) const;
};

}  // namespace m3lb
