// Host side of the wall nodes (lbm_walls.h): regularised-wall setup and the
// device list of wall nodes with its read order.
#include "lbm_walls.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "../../include/m3lb.h"
#include "lbm_host.h"

namespace m3lb {
namespace {

int werr(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

struct Vel {
  int Q;
  const int* c[3];
};
Vel velocities(int lattice) {
  if (lattice == 9) return {9, {D2Q9::cx, D2Q9::cy, D2Q9::cz}};
  return {27, {D3Q27::cx, D3Q27::cy, D3Q27::cz}};
}

// Interior coordinates -> padded index (Domain::id, no wrap).
inline long long idi(const Geo& g, long long x, long long y, long long z) {
  return ((z + g.hz) * g.sy + (y + g.hy)) * g.sx + (x + g.hx);
}
inline bool is_wall(uint8_t f) { return f == kRegWall || f == kSpecWall || f == kSpecNode; }

}  // namespace

void WallSet::release() {
  cudaFree(nodes);
  cudaFree(heads);
  cudaFree(wall_rho);
  cudaFree(snap);
  cudaFree(spec);
  nodes = nullptr; heads = nullptr; wall_rho = nullptr; snap = nullptr; spec = nullptr;
  count = 0; nsnap = 0;
}

int WallSet::set_regularized(const Geo& g, int lattice, std::vector<uint8_t>& flags,
                             const uint8_t* codes, const double* states) {
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  char msg[256];
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const unsigned c = codes[((size_t)z * ny + y) * nx + x];
        if (c > kNrmOutEq) {
          std::snprintf(msg, sizeof msg,
                        "set_regularized_walls: normal code %u at (%d,%d,%d) is not one of 0..10", c,
                        x, y, z);
          return werr(M3LB_ERR_INVALID, msg);
        }
        // the reference reads the upstream nodes at x-1 (and x-2 at order 2)
        if ((c == kNrmOutXp || c == kNrmOutEq) && x < (c == kNrmOutXp ? out_order : 1)) {
          std::snprintf(msg, sizeof msg,
                        "set_regularized_walls: outlet code %u at (%d,%d,%d) has no upstream node "
                        "inside the domain", c, x, y, z);
          return werr(M3LB_ERR_INVALID, msg);
        }
      }
  // FluidSolver.hpp:378-395: codes and states; the nodes become RegWall
  reg.clear();
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const size_t k = ((size_t)z * ny + y) * nx + x;
        if (!codes[k]) continue;
        const long long n = idi(g, x, y, z);
        WallHost w;
        w.code = codes[k];
        w.don = n;
        for (int a = 0; a < 4; ++a) w.u[a] = states ? states[k * 4 + a] : (a == 3 ? 1.0 : 0.0);
        reg[n] = w;
        flags[n] = kRegWall;
      }
  auto code_at = [&](long long n) -> uint8_t {
    auto it = reg.find(n);
    return it == reg.end() ? 0 : it->second.code;
  };
  // :399-423 corners: an axis direction whose next two nodes are straight walls
  static const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  // :428-468 unknown directions: source outside the domain, Excluded or Solid
  const Vel v = velocities(lattice);
  const int nn[3] = {nx, ny, nz};
  const int per[3] = {g.px, g.py, g.pz};
  // :476-512 outflow donors: the fluid neighbour opposite the leaving axis step
  static const int dd[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  static const uint8_t dcode[6] = {2, 1, 4, 3, 6, 5};
  int degenerate = 0;
  for (auto& [n, w] : reg) {
    const long long pz = n / ((long long)g.sx * g.sy), py = (n / g.sx) % g.sy, px = n % g.sx;
    const int x = (int)(px - g.hx), y = (int)(py - g.hy), z = (int)(pz - g.hz);
    if (w.code == kNrmCorner) {
      for (int k = 0; k < (nz > 1 ? 6 : 4); ++k) {
        const int x1 = x + d6[k][0], y1 = y + d6[k][1], z1 = z + d6[k][2];
        const int x2 = x + 2 * d6[k][0], y2 = y + 2 * d6[k][1], z2 = z + 2 * d6[k][2];
        if (x1 < 0 || y1 < 0 || z1 < 0 || x2 < 0 || y2 < 0 || z2 < 0) continue;
        if (x1 >= nx || y1 >= ny || z1 >= nz || x2 >= nx || y2 >= ny || z2 >= nz) continue;
        const uint8_t a = code_at(idi(g, x1, y1, z1)), b = code_at(idi(g, x2, y2, z2));
        if (a != 0 && a != kNrmCorner && b != 0 && b != kNrmCorner) {
          w.ext = (uint8_t)(k + 1);
          break;
        }
      }
    }
    uint32_t m = 0;
    for (int i = 0; i < v.Q; ++i) {
      int src[3] = {x - v.c[0][i], y - v.c[1][i], z - v.c[2][i]};
      bool outside = false;
      for (int a = 0; a < 3; ++a) {
        if (per[a]) src[a] = (src[a] + nn[a]) % nn[a];
        else if (src[a] < 0 || src[a] >= nn[a]) outside = true;
      }
      if (!outside) {
        const uint8_t sf = flags[idi(g, src[0], src[1], src[2])];
        if (sf == 2 || sf == 1) outside = true;
      }
      if (outside) m |= 1u << i;
    }
    w.unk = m;
    if (w.code == kNrmOutFree) {
      bool found = false;
      for (int k = 0; k < 6 && !found; ++k) {
        const int qx = x + dd[k][0], qy = y + dd[k][1], qz = z + dd[k][2];
        const bool leaves = (qx < 0 || qx >= nx || qy < 0 || qy >= ny || qz < 0 || qz >= nz) ||
                            flags[idi(g, qx, qy, qz)] == 1;
        if (!leaves) continue;
        const int o = k ^ 1;
        const int rx = x + dd[o][0], ry = y + dd[o][1], rz = z + dd[o][2];
        if (rx < 0 || rx >= nx || ry < 0 || ry >= ny || rz < 0 || rz >= nz) continue;
        const long long mm = idi(g, rx, ry, rz);
        if (flags[mm] != 0) continue;
        w.don = mm;
        w.onrm = dcode[k];
        found = true;
      }
      if (!found) ++degenerate;
    }
  }
  if (degenerate)
    std::printf("  [walls] %d outflow node(s) have no fluid neighbour and are inert\n", degenerate);
  scale = 1;
  return M3LB_OK;
}

BoundArgs WallSet::args(int begin, int end) const {
  BoundArgs b{};
  b.nodes = nodes;
  b.heads = heads;
  b.begin = begin;
  b.end = end;
  b.wall_rho = wall_rho;
  b.snap = snap;
  b.scale = scale;
  b.field_scale = field_scale;
  b.field_on = field_on ? 1 : 0;
  b.fd_corners = fd_corners;
  b.force_bc = force_bc;
  b.out_order = out_order;
  b.out_rho = out_rho;
  return b;
}

int WallSet::build(const Geo& g, int lattice, int op, int storage, const std::vector<uint8_t>& flags,
                   cudaStream_t s) {
  release();
  corners = false;
  level_end.clear();
  std::vector<long long> ns;
  for (long long n = 0; n < g.n_padded; ++n)
    if (is_wall(flags[n])) ns.push_back(n);
  if (ns.empty()) return M3LB_OK;
  const bool f64 = storage == M3LB_STORE_F64;
  auto rnd = [f64](double x) { return f64 ? x : (double)(float)x; };  // the arithmetic type
  std::unordered_map<long long, int> pos;
  pos.reserve(ns.size() * 2);
  for (size_t j = 0; j < ns.size(); ++j) pos[ns[j]] = (int)j;
  auto pos_of = [&](long long n) {
    auto it = pos.find(n);
    return it == pos.end() ? -1 : it->second;
  };
  const int D = lattice == 9 ? 2 : 3;
  const int nn[3] = {g.nx, g.ny, g.nz};
  const int per[3] = {g.px, g.py, g.pz};
  static const int d6[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

  std::vector<BNode> list(ns.size());
  std::vector<int> level(ns.size(), 0);
  nsnap = 0;
  for (size_t j = 0; j < ns.size(); ++j) {
    const long long n = ns[j];
    BNode& b = list[j];
    std::fill(std::begin(b.ref), std::end(b.ref), -1LL);
    std::fill(std::begin(b.ref_wall), std::end(b.ref_wall), -1);
    std::fill(std::begin(b.snap), std::end(b.snap), -1);
    b.n = n;
    b.c1 = b.c2 = -1;
    b.type = flags[n];
    b.fd_dir[0] = b.fd_dir[1] = b.fd_dir[2] = 2;
    b.u[0] = b.u[1] = b.u[2] = 0;
    b.u[3] = 1;
    b.un[0] = b.un[1] = b.un[2] = 0;
    const int x = (int)(n % g.sx) - g.hx, y = (int)((n / g.sx) % g.sy) - g.hy,
              z = (int)(n / ((long long)g.sx * g.sy)) - g.hz;
    if (b.type == kSpecWall) {
      b.code = spec_nrm.empty() ? 0 : spec_nrm[n];
      continue;
    }
    if (b.type == kSpecNode) {
      b.code = spec_faces.empty() ? 0 : spec_faces[n];
      continue;
    }
    auto it = reg.find(n);
    const WallHost w = it == reg.end() ? WallHost{} : it->second;
    b.code = w.code;
    b.unk = w.unk;
    b.onrm = w.onrm;
    for (int a = 0; a < 4; ++a) b.u[a] = rnd(w.u[a]);
    if (field_on && !field.empty()) {
      const size_t k = ((size_t)z * g.ny + y) * g.nx + x;
      for (int a = 0; a < 3; ++a) b.un[a] = rnd(field[k * 3 + a]);
    }
    if (w.code == kNrmOutFree) {
      b.ref[0] = w.don;
    } else if (w.code == kNrmOutEq) {
      b.ref[0] = idi(g, x - 1, y, z);
    } else if (w.code == kNrmOutXp) {
      b.ref[0] = idi(g, x - 1, y, z);
      if (out_order >= 2) b.ref[1] = idi(g, x - 2, y, z);
    } else if (w.code == kNrmCorner) {
      corners = true;
      if (w.ext) {
        const int* e = d6[w.ext - 1];
        b.c1 = pos_of(idi(g, x + e[0], y + e[1], z + e[2]));
        b.c2 = pos_of(idi(g, x + 2 * e[0], y + 2 * e[1], z + 2 * e[2]));
        if (b.c1 < 0 || b.c2 < 0) b.c1 = b.c2 = -1;
      }
      if (fd_corners && op != 0) {
        // FluidSolver.hpp:988-1011: one-sided at a non-periodic end, else centred
        const int ic[3] = {x, y, z};
        for (int a = 0; a < D; ++a) {
          if (nn[a] < 3) continue;
          int dir = 0;
          if (!per[a]) {
            if (ic[a] == 0) dir = 1;
            else if (ic[a] == nn[a] - 1) dir = -1;
          }
          int c1[3] = {x, y, z}, c2[3] = {x, y, z};
          if (dir != 0) {
            c1[a] += dir;
            c2[a] += 2 * dir;
          } else {
            c1[a] = (ic[a] + 1) % nn[a];
            c2[a] = (ic[a] - 1 + nn[a]) % nn[a];
          }
          b.fd_dir[a] = (int8_t)dir;
          b.ref[2 * a] = idi(g, c1[0], c1[1], c1[2]);
          b.ref[2 * a + 1] = idi(g, c2[0], c2[1], c2[2]);
        }
      }
    }
    // read order: a wall node's state is read without loading it; a later
    // node is read before its update (snapshot); an earlier wall node must
    // have been updated first (level)
    for (int k = 0; k < kBndRefs; ++k) {
      const long long m = b.ref[k];
      if (m < 0) continue;
      if (w.code == kNrmCorner && flags[m] == kRegWall) {
        b.ref_wall[k] = pos_of(m);
      } else if (m > n) {
        b.snap[k] = nsnap++;
      } else if (m < n && is_wall(flags[m])) {
        level[j] = std::max(level[j], level[pos_of(m)] + 1);
      }
    }
  }
  // order by level, index order within a level
  std::vector<int> order(ns.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return level[a] < level[b]; });
  std::vector<int> newpos(ns.size());
  for (size_t p = 0; p < order.size(); ++p) newpos[order[p]] = (int)p;
  std::vector<BNode> sorted(ns.size());
  for (size_t p = 0; p < order.size(); ++p) {
    BNode b = list[order[p]];
    if (b.c1 >= 0) { b.c1 = newpos[b.c1]; b.c2 = newpos[b.c2]; }
    for (int k = 0; k < kBndRefs; ++k)
      if (b.ref_wall[k] >= 0) b.ref_wall[k] = newpos[b.ref_wall[k]];
    sorted[p] = b;
    if (p + 1 == order.size() || level[order[p + 1]] != level[order[p]]) level_end.push_back((int)p + 1);
  }
  count = (int)ns.size();

  const size_t rb = f64 ? 8 : 4;
  std::vector<uint8_t> sp((size_t)g.n_padded, 0);
  for (long long n : ns) {
    if (flags[n] == kSpecWall && !spec_nrm.empty()) sp[n] = spec_nrm[n];
    if (flags[n] == kSpecNode && !spec_faces.empty()) sp[n] = spec_faces[n];
  }
  std::vector<BHead> hd(sorted.size());
  for (size_t p = 0; p < sorted.size(); ++p) {
    const BNode& b = sorted[p];
    BHead& h = hd[p];
    h.n = b.n;
    h.unk = b.unk;
    h.type = b.type;
    h.code = b.code;
    h.moving = 0;
    h.pad = 0;
    for (int a = 0; a < 3; ++a) {
      uint64_t u, v;
      std::memcpy(&u, &b.u[a], 8);
      std::memcpy(&v, &b.un[a], 8);
      if (u | v) h.moving = 1;
    }
  }
  if (cudaMalloc((void**)&nodes, sizeof(BNode) * count) != cudaSuccess ||
      cudaMalloc((void**)&heads, sizeof(BHead) * count) != cudaSuccess ||
      cudaMalloc(&wall_rho, rb * count) != cudaSuccess ||
      (nsnap && cudaMalloc(&snap, rb * (size_t)nsnap * (lattice == 9 ? 9 : 27)) != cudaSuccess) ||
      cudaMalloc((void**)&spec, (size_t)g.n_padded) != cudaSuccess) {
    release();
    return werr(M3LB_ERR_MEMORY, "walls: cannot allocate the wall-node list");
  }
  cudaError_t e = cudaMemcpyAsync(nodes, sorted.data(), sizeof(BNode) * count, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(heads, hd.data(), sizeof(BHead) * count, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(wall_rho, 0, rb * count, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(spec, sp.data(), sp.size(), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    release();
    return werr(M3LB_ERR_CUDA, cudaGetErrorString(e));
  }
  return M3LB_OK;
}

}  // namespace m3lb
