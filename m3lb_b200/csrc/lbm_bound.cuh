// Boundary-node pass of the lattice-Boltzmann step: regularised walls
// (RegWall) and free-slip walls (SpecWall, SpecNode).
//
// Wall nodes are a thin surface of the lattice, so they are kept out of the
// bulk kernels: every bulk kernel leaves a flagged node's slots untouched
// (Esoteric Pull's bounce-back is the identity on the storage), and this pass
// then updates the wall nodes from a compact list, one thread per node.  A
// wall node reads and writes only its own Q slots, so running it after the
// bulk sweep gives the same result as running it inside.
//
// Three branches of the reference read OTHER nodes inside its in-place sweep
// (FluidSolver.hpp:847-912, 924-986): the outflow codes read an upstream or
// donor node and the finite-difference corner reads the velocity of its
// neighbours.  Their result depends on the order of the sweep; the order this
// library reproduces is the index order of the reference's one-thread run.  A
// node read there before its own update (a later index) is copied by a
// snapshot pass ahead of the bulk sweep; a node read after its update (an
// earlier index) is read live after the bulk sweep, and when that node is
// itself in the list, the list is processed in levels so it goes first.
//
// Regularised reconstruction: src/boundary/Regularized.hpp:170-328 (Latt et
// al. 2008, Eqs. 27, 44-45), the step branch FluidSolver.hpp:792-1021, the
// corner densities :664-712 and the reported state :1081-1188.
#pragma once
#include "lbm_kernels.cuh"

namespace m3lb {

// ------------------------------------------------------------ node access
// Coordinates of a padded node index (32-bit division when the block has
// fewer than 2^31 nodes, as every lattice up to ~1290^3 does).
__device__ __forceinline__ void padded_coords(const Geo& g, long long n, int& x, int& y, int& z) {
  if (g.n_padded < (1LL << 31)) {
    const unsigned u = (unsigned)n, sx = (unsigned)g.sx, sy = (unsigned)g.sy;
    const unsigned r = u / sx;
    x = (int)(u - r * sx);
    y = (int)(r % sy);
    z = (int)(r / sy);
    return;
  }
  x = (int)(n % g.sx);
  y = (int)((n / g.sx) % g.sy);
  z = (int)(n / ((long long)g.sx * g.sy));
}

// Interior index (x fastest) of a padded node.
__device__ __forceinline__ size_t interior_index(const Geo& g, long long n) {
  int x, y, z;
  padded_coords(g, n, x, y, z);
  return ((size_t)(z - g.hz) * g.ny + (y - g.hy)) * g.nx + (x - g.hx);
}

// The Q populations about to arrive at node n (Access::load_pair, parity P):
// the node's own slot of direction 0 plus, per direction, a compile-time
// direction offset and the neighbour's per-axis offsets (AxisSteps, the wrap
// or clamp folded in), as the one-node step kernel addresses them.
template <class L, int ST, class R>
__device__ __forceinline__ void load_pops(const StepArgs& a, long long n, R* f) {
  using E = typename StoreT<ST>::elem;
  const Geo& g = a.g;
  int x, y, z;
  padded_coords(g, n, x, y, z);
  const E* own = reinterpret_cast<const E*>(a.f) + slot<L::Q>(g, x, y, z, 0);
  const AxisSteps<L::Q> st = axis_steps<L::Q>(g, x, y, z);
  const int P = a.parity;
  const E* up = own + P * kChunk;        // slot i + P of the node
  const E* dn = own + (1 - P) * kChunk;  // slot i + 1 - P, before the neighbour offset
  f[0] = to_real(own[0]);
  static_for<1, L::Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    f[i] = to_real(up[i * kChunk]);
    f[i + 1] = to_real(dn[nb_offset<L, i>(st) + i * kChunk]);
  });
}
template <class L, int ST, class R>
__device__ __forceinline__ void store_pops(const StepArgs& a, long long n, const R* f) {
  using E = typename StoreT<ST>::elem;
  const Geo& g = a.g;
  int x, y, z;
  padded_coords(g, n, x, y, z);
  E* own = reinterpret_cast<E*>(a.f) + slot<L::Q>(g, x, y, z, 0);
  const AxisSteps<L::Q> st = axis_steps<L::Q>(g, x, y, z);
  const int P = a.parity;
  E* up = own + P * kChunk;
  E* dn = own + (1 - P) * kChunk;
  own[0] = from_real<E>(f[0]);
  static_for<1, L::Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    dn[nb_offset<L, i>(st) + i * kChunk] = from_real<E>(f[i]);
    up[i * kChunk] = from_real<E>(f[i + 1]);
  });
}
// Populations of the k-th node a list node reads, unshifted when USH; from
// the snapshot inside a step (SNAP), from the array outside one.
template <class L, int ST, bool USH, bool SNAP = true, class R>
__device__ __forceinline__ void fetch_ref(const StepArgs& a, const BoundArgs& b, const BNode& nd,
                                          int k, R* g) {
  if (SNAP && nd.snap[k] >= 0) {
    const R* s = reinterpret_cast<const R*>(b.snap) + (size_t)nd.snap[k] * L::Q;
#pragma unroll
    for (int i = 0; i < L::Q; ++i) g[i] = s[i];
  } else {
    load_pops<L, ST>(a, nd.ref[k], g);
  }
  if constexpr (USH)
    static_for<0, L::Q>([&](auto I) { g[decltype(I)::value] += R(weight<L, decltype(I)::value>()); });
}
template <class L, bool USH, class R>
__device__ __forceinline__ void shift_pops(R* f, R sign) {
  if constexpr (USH)
    static_for<0, L::Q>([&](auto I) {
      f[decltype(I)::value] += sign * R(weight<L, decltype(I)::value>());
    });
}

// ------------------------------------------------- regularised reconstruction
// Outward normal of a code (Regularized.hpp:153-166).
__device__ __forceinline__ void normal_of_code(unsigned code, int n[3]) {
  n[0] = n[1] = n[2] = 0;
  if (code >= 1 && code <= 6) n[(code - 1) / 2] = (code & 1) ? 1 : -1;
  else if (code == kNrmOutXp) n[0] = 1;
}

// Raw equilibrium of direction I (Equilibrium.hpp:34-37) with the second-order
// (BEQ 0) or product-form (BEQ 1) phi (:49-124).
template <class L, int BEQ, int I, class R>
__device__ __forceinline__ R bc_feq(R rho, R ux, R uy, R uz) {
  constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
  R phi;
  if constexpr (BEQ == 0) {
    const R ics2 = R(3);
    const R cu = R(cx) * ux + R(cy) * uy + R(cz) * uz;
    const R uu = ux * ux + uy * uy + uz * uz;
    phi = ics2 * cu + R(0.5) * ics2 * ics2 * cu * cu - R(0.5) * ics2 * uu;
  } else if constexpr (L::D == 2) {
    const R cs2v = R(1) / R(3);
    const R ax = R(cx * cx) - cs2v, ay = R(cy * cy) - cs2v;
    const R o1 = (R(cx) * ux + R(cy) * uy) / cs2v;
    const R o2 = (ax * ux * ux + ay * uy * uy + R(2) * R(cx) * R(cy) * ux * uy) / (R(2) * cs2v * cs2v);
    const R o3 = (ax * R(cy) * ux * ux * uy + ay * R(cx) * ux * uy * uy) / (R(2) * cs2v * cs2v * cs2v);
    const R o4 = (ax * ay * ux * ux * uy * uy) / (R(4) * cs2v * cs2v * cs2v * cs2v);
    phi = o1 + o2 + o3 + o4;
  } else {
    auto chi = [](int c, R u) { return c == 0 ? R(1) - R(1.5) * u * u : R(1) + R(3) * u * (R(c) + u); };
    phi = chi(cx, ux) * chi(cy, uy) * chi(cz, uz) - R(1);
  }
  return R(weight<L, I>()) * rho * (R(1) + phi);
}

// Eq. (27) and its inverse (Regularized.hpp:178-206): the partition into
// populations leaving the domain (c.n > 0) and tangential ones.
template <class L, class R>
__device__ __forceinline__ void out_tang(const R* f, const int nrm[3], R& out, R& tang) {
  out = R(0); tang = R(0);
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    const int cn = cx * nrm[0] + cy * nrm[1] + cz * nrm[2];
    if (cn > 0) out += f[i];
    else if (cn == 0) tang += f[i];
  });
}
template <class L, class R>
__device__ __forceinline__ R bc_density(const R* f, const int nrm[3], const R* u) {
  R out, tang;
  out_tang<L>(f, nrm, out, tang);
  const R uperp = u[0] * R(nrm[0]) + u[1] * R(nrm[1]) + u[2] * R(nrm[2]);
  return (R(2) * out + tang) / (R(1) + uperp);
}
template <class L, class R>
__device__ __forceinline__ R bc_normal_velocity(const R* f, const int nrm[3], R rho) {
  R out, tang;
  out_tang<L>(f, nrm, out, tang);
  return (R(2) * out + tang) / rho - R(1);
}

// Q_I : Pi, off-diagonal terms twice (Regularized.hpp:226-231).
template <class L, int I, class R>
__device__ __forceinline__ R q_pi(const R* Pi) {
  constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
  const R cs2v = R(1) / R(3);
  const R d3 = L::D == 3 ? (R(cz * cz) - cs2v) * Pi[2] : R(0);
  const R off = L::D == 3 ? (R(cx * cz) * Pi[4] + R(cy * cz) * Pi[5]) : R(0);
  return (R(cx * cx) - cs2v) * Pi[0] + (R(cy * cy) - cs2v) * Pi[1] + d3 + R(2) * (R(cx * cy) * Pi[3] + off);
}

// Eq. (45) with Pi^(1) given (Regularized.hpp:219-236).
template <class L, int BEQ, class R>
__device__ __forceinline__ void bc_apply_with_stress(R* f, R rho, const R* u, const R* Pi) {
  const R cs2v = R(1) / R(3), cs4v = cs2v * cs2v;
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    f[i] = bc_feq<L, BEQ, i>(rho, u[0], u[1], u[2]) + R(weight<L, i>()) / (R(2) * cs4v) * q_pi<L, i>(Pi);
  });
}

// Eqs. (44)-(45) with the forced corrections (Regularized.hpp:262-328).
template <class L, int BEQ, class R>
__device__ __forceinline__ void bc_apply(R* f, R rho, const R* u, uint32_t unknown, const R* Fv) {
  constexpr int Q = L::Q;
  const R cs2v = R(1) / R(3), cs4v = cs2v * cs2v;
  const R hodd = R(0.5) / cs2v;
  R feq[Q];
  static_for<0, Q>([&](auto I) {
    feq[decltype(I)::value] = bc_feq<L, BEQ, decltype(I)::value>(rho, u[0], u[1], u[2]);
  });
  // scaffold: bounce-back of the off-equilibrium part for the unknowns
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int o = (i == 0) ? 0 : ((i & 1) ? i + 1 : i - 1);
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    if (unknown & (1u << i)) {
      const R cF = Fv ? (R(cx) * Fv[0] + R(cy) * Fv[1] + R(cz) * Fv[2]) : R(0);
      const R odd = R(weight<L, i>()) * hodd * cF;
      f[i] = (unknown & (1u << o)) ? feq[i] - odd : feq[i] + (f[o] - feq[o]) - R(2) * odd;
    }
  });
  R Pi[6] = {0, 0, 0, 0, 0, 0};
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    const R d = f[i] - feq[i];
    Pi[0] += d * R(cx) * R(cx); Pi[1] += d * R(cy) * R(cy); Pi[2] += d * R(cz) * R(cz);
    Pi[3] += d * R(cx) * R(cy); Pi[4] += d * R(cx) * R(cz); Pi[5] += d * R(cy) * R(cz);
  });
  static_for<0, Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    const R cF = Fv ? (R(cx) * Fv[0] + R(cy) * Fv[1] + R(cz) * Fv[2]) : R(0);
    f[i] = feq[i] - R(weight<L, i>()) * hodd * cF + R(weight<L, i>()) / (R(2) * cs4v) * q_pi<L, i>(Pi);
  });
}

// Raw moments of a population set: density and velocity (up_vel, vel_at).
template <class L, class R>
__device__ __forceinline__ R moments(const R* g, R* m) {
  R sm = 0;
  m[0] = m[1] = m[2] = R(0);
  static_for<0, L::Q>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int cx = L::cx[i], cy = L::cy[i], cz = L::cz[i];
    sm += g[i];
    m[0] += g[i] * R(cx); m[1] += g[i] * R(cy); m[2] += g[i] * R(cz);
  });
  return sm;
}

// Wall velocity of list node idx: the per-node field when set, else its
// state.  A node whose velocities are all +0 (not `moving`) gets the same
// products with +0 without reading its BNode.
template <class R>
__device__ __forceinline__ void wall_velocity(const BoundArgs& b, const BHead& h, int idx, R* uw) {
  if (!h.moving) {
    const R z = b.field_on ? R(b.field_scale) * R(0) : R(0) * R(b.scale);
    uw[0] = uw[1] = uw[2] = z;
    return;
  }
  const BNode& nd = b.nodes[idx];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    uw[a] = b.field_on ? R(b.field_scale) * R(nd.un[a]) : R(nd.u[a]) * R(b.scale);
}

// Velocity at the k-th upstream node of an outflow face (FluidSolver.hpp:896-912).
template <class L, int ST, bool USH, bool SNAP = true, class R>
__device__ __forceinline__ void up_velocity(const StepArgs& a, const BoundArgs& b, const BNode& nd,
                                            int k, R* v) {
  R g[L::Q];
  fetch_ref<L, ST, USH, SNAP>(a, b, nd, k, g);
  const R sm = moments<L>(g, v);
  const R ir = R(1) / sm;
  v[0] *= ir; v[1] *= ir; v[2] *= ir;
}

// The RegWall branch of run_step (FluidSolver.hpp:792-1021) on the loaded
// populations f.  Returns true when the node is finished (the outflow codes
// that overwrite it), false when it goes on to collide.
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE, class R>
__device__ __forceinline__ bool regwall(const StepArgs& a, const BoundArgs& b, const BHead& h,
                                        int idx, R* f) {
  const BNode& nd = b.nodes[idx];  // read only by the outflow and corner-stencil branches
  constexpr int Q = L::Q;
  constexpr bool USH = SH && OP != 0;                    // the no-collision mock runs raw
  constexpr int BEQ = OP >= 3 ? 1 : (OP == 0 ? 0 : EQ);  // EquilibriumOf (Regularized.hpp:47-57)
  shift_pops<L, USH>(f, R(1));
  const unsigned code = h.code;
  int nrm[3];
  normal_of_code(code, nrm);
  R uw[3];
  wall_velocity(b, h, idx, uw);
  // has_forcing looks for a ForcingPolicy member type, which only BGK declares
  R Fv[3] = {0, 0, 0};
  if constexpr (FORCE && OP == 1) {
    const CollideParams<R> fp = node_params<FORCE, R>(a, interior_index(a.g, h.n));
    Fv[0] = fp.fx; Fv[1] = fp.fy; Fv[2] = fp.fz;
  }
  R ur[3] = {uw[0], uw[1], uw[2]};
  R rw;
  if (code == kNrmOutFree) {                             // donor rescaled to the target density
    R g[Q];
    fetch_ref<L, ST, USH>(a, b, nd, 0, g);
    R sm = 0;
#pragma unroll
    for (int i = 0; i < Q; ++i) sm += g[i];
    if (sm > R(0)) {
      const R sc = R(b.out_rho) / sm;
#pragma unroll
      for (int i = 0; i < Q; ++i) f[i] = g[i] * sc;
    }
    shift_pops<L, USH>(f, R(-1));
    store_pops<L, ST>(a, h.n, f);
    return true;
  }
  if (code == kNrmOutEq) {                               // equilibrium at the upstream velocity
    const R rw2 = R(nd.u[3]);
    R g[Q], mu[3];
    fetch_ref<L, ST, USH>(a, b, nd, 0, g);
    const R sm = moments<L>(g, mu);
    const R ir = (sm > R(0)) ? R(1) / sm : R(0);
    mu[0] *= ir; mu[1] *= ir; mu[2] *= ir;
    static_for<0, Q>([&](auto I) {
      f[decltype(I)::value] = bc_feq<L, BEQ, decltype(I)::value>(rw2, mu[0], mu[1], mu[2]);
    });
    shift_pops<L, USH>(f, R(-1));
    store_pops<L, ST>(a, h.n, f);
    return true;
  }
  if (code == kNrmOutXp) {                               // imposed density, closure normal velocity
    rw = R(nd.u[3]);
    R ut[3];
    up_velocity<L, ST, USH>(a, b, nd, 0, ut);
    if (b.out_order >= 2) {
      R v2[3];
      up_velocity<L, ST, USH>(a, b, nd, 1, v2);
#pragma unroll
      for (int c = 0; c < 3; ++c) ut[c] = R(2) * ut[c] - v2[c];
    }
    const R un = bc_normal_velocity<L>(f, nrm, rw);
    R utn = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) utn += ut[c] * R(nrm[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) ur[c] = ut[c] + (un - utn) * R(nrm[c]);
  } else {
    rw = (code == kNrmCorner) ? reinterpret_cast<const R*>(b.wall_rho)[idx] : bc_density<L>(f, nrm, ur);
  }
  if (OP != 0 && b.fd_corners && code == kNrmCorner) {
    // Pi^(1) from finite-difference velocity gradients (Latt et al. Sec. V)
    R grad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll 1
    for (int ax = 0; ax < L::D; ++ax) {
      const int dir = nd.fd_dir[ax];
      if (dir == 2) continue;
      R u12[2][3];
#pragma unroll 1
      for (int s = 0; s < 2; ++s) {
        const int k = 2 * ax + s;
        if (nd.ref_wall[k] >= 0) {
          const BNode& w = b.nodes[nd.ref_wall[k]];
#pragma unroll
          for (int c = 0; c < 3; ++c) u12[s][c] = R(w.u[c]) * R(b.scale);
        } else {
          R g[Q];
          fetch_ref<L, ST, USH>(a, b, nd, k, g);
          const R sm = moments<L>(g, u12[s]);
          const R ir = R(1) / sm;
#pragma unroll
          for (int c = 0; c < 3; ++c) u12[s][c] *= ir;
        }
      }
#pragma unroll
      for (int c = 0; c < L::D; ++c)
        grad[ax][c] = dir != 0 ? R(dir) * (R(-1.5) * uw[c] + R(2) * u12[0][c] - R(0.5) * u12[1][c])
                               : R(0.5) * (u12[0][c] - u12[1][c]);
    }
    const R cs2v = R(1) / R(3);
    const R kk = -R(2) * cs2v * rw / R(a.omega);          // Eqs. (21)-(22), shear rate
    const R Pi[6] = {kk * grad[0][0], kk * grad[1][1], kk * grad[2][2],
                     kk * R(0.5) * (grad[0][1] + grad[1][0]), kk * R(0.5) * (grad[0][2] + grad[2][0]),
                     kk * R(0.5) * (grad[1][2] + grad[2][1])};
    bc_apply_with_stress<L, BEQ>(f, rw, ur, Pi);
  } else {
    bc_apply<L, BEQ>(f, rw, ur, h.unk, b.force_bc ? Fv : (const R*)nullptr);
  }
  shift_pops<L, USH>(f, R(-1));
  return false;
}

// ------------------------------------------------------------------ kernels
// Copies of the nodes read before their own update (later in index order).
template <class L, int ST>
__global__ void __launch_bounds__(kBndThreads) bnd_snapshot(StepArgs a, BoundArgs b) {
  using R = typename StoreT<ST>::real;
  const int i = b.begin + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= b.end) return;
  const BNode& nd = b.nodes[i];
#pragma unroll 1
  for (int k = 0; k < kBndRefs; ++k) {
    if (nd.snap[k] < 0) continue;
    R g[L::Q];
    load_pops<L, ST>(a, nd.ref[k], g);
    R* s = reinterpret_cast<R*>(b.snap) + (size_t)nd.snap[k] * L::Q;
#pragma unroll
    for (int q = 0; q < L::Q; ++q) s[q] = g[q];
  }
}

// corner_density pass 1 (FluidSolver.hpp:675-694): the closure density of
// every straight RegWall node at the parity the sweep is about to read.
template <class L, int ST, bool USH>
__global__ void __launch_bounds__(kBndThreads) bnd_wall_rho(StepArgs a, BoundArgs b) {
  using R = typename StoreT<ST>::real;
  const int i = b.begin + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= b.end) return;
  const BHead h = b.heads[i];
  if (h.type != kRegWall || h.code == kNrmCorner || h.code == 0) return;
  R f[L::Q], uw[3];
  load_pops<L, ST>(a, h.n, f);
  shift_pops<L, USH>(f, R(1));
  int nrm[3];
  normal_of_code(h.code, nrm);
  wall_velocity(b, h, i, uw);
  R* rho = reinterpret_cast<R*>(b.wall_rho);
  rho[i] = (h.code == kNrmOutXp || h.code == kNrmOutEq) ? R(b.nodes[i].u[3])
         : (h.code == kNrmOutFree) ? R(b.out_rho) : bc_density<L>(f, nrm, uw);
}
// pass 2 (:696-711): corners extrapolated along a wall, 1 without a stencil.
template <class R>
__global__ void __launch_bounds__(kBndThreads) bnd_corner_rho(BoundArgs b) {
  const int i = b.begin + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= b.end) return;
  const BHead h = b.heads[i];
  if (h.type != kRegWall || h.code != kNrmCorner) return;
  const BNode& nd = b.nodes[i];
  R* rho = reinterpret_cast<R*>(b.wall_rho);
  rho[i] = nd.c1 < 0 ? R(1) : R(2) * rho[nd.c1] - rho[nd.c2];
}

// The wall nodes' update: SpecWall mirror, SpecNode mirror + collision,
// RegWall reconstruction + collision (or the outflow overwrite).
template <class L, int ST, int OP, int EQ, bool SH, bool FORCE>
__global__ void __launch_bounds__(kBndThreads) bnd_step(StepArgs a, BoundArgs b) {
  using R = typename StoreT<ST>::real;
  const int i = b.begin + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= b.end) return;
  const BHead h = b.heads[i];
  R f[L::Q];
  load_pops<L, ST>(a, h.n, f);
  if (h.type == kSpecWall) {
    spec_wall_permute<L>(f, spec_axis(h.code));
    store_pops<L, ST>(a, h.n, f);
    return;
  }
  if (h.type == kSpecNode) spec_node_mirror<L>(f, h.code);
  else if (regwall<L, ST, OP, EQ, SH, FORCE>(a, b, h, i, f)) return;
  const size_t k = interior_index(a.g, h.n);
  const Macro<R> mc = collide<L, OP, EQ, SH, FORCE>(f, node_params<FORCE, R>(a, k));
  store_pops<L, ST>(a, h.n, f);
  if (a.rho) {
    reinterpret_cast<R*>(a.rho)[k] = mc.rho;
    reinterpret_cast<R*>(a.ux)[k] = mc.ux;
    reinterpret_cast<R*>(a.uy)[k] = mc.uy;
    reinterpret_cast<R*>(a.uz)[k] = mc.uz;
  }
}

// The state a RegWall node reports (compute_macroscopic, FluidSolver.hpp:1081-1188):
// the imposed velocity with the closure density, or the outflow's own.
template <class L, int ST, bool USH>
__global__ void __launch_bounds__(kBndThreads) bnd_macro(StepArgs a, BoundArgs b) {
  using R = typename StoreT<ST>::real;
  constexpr int Q = L::Q;
  const int i = b.begin + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= b.end) return;
  const BHead h = b.heads[i];
  if (h.type != kRegWall) return;
  const BNode& nd = b.nodes[i];
  R fw[Q];
  load_pops<L, ST>(a, h.n, fw);
  shift_pops<L, USH>(fw, R(1));
  const unsigned code = h.code;
  int nrm[3];
  normal_of_code(code, nrm);
  R uw[3];
  wall_velocity(b, h, i, uw);
  R rw;
  if (code == kNrmOutFree) {
    rw = R(b.out_rho);
    int onr[3];
    normal_of_code(nd.onrm, onr);
    R g[Q], m4[3];
    fetch_ref<L, ST, USH, false>(a, b, nd, 0, g);
    const R sm = moments<L>(g, m4);
    const R ir = (sm > R(0)) ? R(1) / sm : R(0);
    const R un = bc_normal_velocity<L>(fw, onr, rw);
    R utn = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) utn += m4[c] * ir * R(onr[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) uw[c] = m4[c] * ir + (un - utn) * R(onr[c]);
  } else if (code == kNrmOutEq) {
    rw = R(nd.u[3]);
    R g[Q], mu[3];
    fetch_ref<L, ST, USH, false>(a, b, nd, 0, g);
    const R sm = moments<L>(g, mu);
    const R ir = (sm > R(0)) ? R(1) / sm : R(0);
#pragma unroll
    for (int c = 0; c < 3; ++c) uw[c] = mu[c] * ir;
  } else if (code == kNrmOutXp) {
    rw = R(nd.u[3]);
    R ut[3];
    up_velocity<L, ST, USH, false>(a, b, nd, 0, ut);
    if (b.out_order >= 2) {
      R v2[3];
      up_velocity<L, ST, USH, false>(a, b, nd, 1, v2);
#pragma unroll
      for (int c = 0; c < 3; ++c) ut[c] = R(2) * ut[c] - v2[c];
    }
    const R un = bc_normal_velocity<L>(fw, nrm, rw);
    R utn = 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) utn += ut[c] * R(nrm[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) uw[c] = ut[c] + (un - utn) * R(nrm[c]);
  } else {
    rw = (code == kNrmCorner) ? reinterpret_cast<const R*>(b.wall_rho)[i] : bc_density<L>(fw, nrm, uw);
  }
  const Geo& g = a.g;
  int x, y, z;
  padded_coords(g, h.n, x, y, z);
  const size_t k = ((size_t)(z - g.hz) * g.ny + (y - g.hy)) * g.nx + (x - g.hx);
  reinterpret_cast<R*>(a.rho)[k] = rw;
  reinterpret_cast<R*>(a.ux)[k] = uw[0];
  reinterpret_cast<R*>(a.uy)[k] = uw[1];
  reinterpret_cast<R*>(a.uz)[k] = uw[2];
}

}  // namespace m3lb
