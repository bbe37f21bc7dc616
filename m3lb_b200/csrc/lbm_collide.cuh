// Collision operators of the M3LB lattice-Boltzmann step, in registers.
//
// Written once over an arithmetic type V: `f2` (two x-adjacent nodes with
// paired FP32 instructions), `float` or `double` (one node).  Populations are
// the stored variable: g = f - w with shifted storage, f with raw storage
// (src/memory/Storage.hpp:27-35).
//
// Operators and the reference code each one restates:
//   OP 0  none      pure streaming (the NullCollision mock,
//                   tests/test_streaming.cpp:28-38)
//   OP 1  BGK       src/collision/BGK.hpp:63-92
//   OP 2  TRT       src/collision/TRT.hpp:92-127
//   OP 3  raw MRT   src/collision/MomentCollision.hpp:234-314 (Central = false)
//   OP 4  central moments, same file (Central = true)
// Equilibria (BGK/TRT): EQ 0 second order, EQ 1 product form
// (src/equilibrium/Equilibrium.hpp:28-124).  Forcing: Guo with a uniform force
// (src/forcing/Forcing.hpp:26-82).
//
// The algebra is the reference's; the evaluation is rearranged for
// instruction count: opposite pairs share their even and odd parts, and the
// moment operators take only the order <= 2 moments from the forward
// transform, because every higher moment is overwritten by its equilibrium.
// Results therefore agree with the reference to rounding, not bit for bit;
// the streaming itself is bit-exact.
#pragma once
#include <type_traits>

#include "lbm_common.cuh"

namespace m3lb {

template <int N> using IC = std::integral_constant<int, N>;

// Compile-time loop: fn(IC<B>), fn(IC<B+STEP>), ... while < E.
template <int B, int E, int STEP = 1, class Fn>
__device__ __forceinline__ void static_for(Fn&& fn) {
  if constexpr (B < E) {
    fn(IC<B>{});
    static_for<B + STEP, E, STEP>(fn);
  }
}

template <class S, class FV = S>
struct CollideParams {
  S omega, omega2;
  FV fx, fy, fz;  // the body force: one value for the lattice, or one per node of a pair
};
// The force as the arithmetic type V: broadcast when it is one value.
template <class V, class FV>
__device__ __forceinline__ V fvec(FV x) {
  if constexpr (std::is_same_v<V, FV>) return x;
  else return bc<V>(x);
}

// Macroscopic state of one node (or node pair).
template <class V>
struct Macro {
  V dens;  // rho (raw storage) or rho - 1 (shifted storage)
  V rho;
  V ux, uy, uz;
};

template <class L, int I>
__host__ __device__ constexpr double weight() { return double(L::wn[I]) / double(L::WDEN); }

// c_I . (vx, vy, vz) for a compile-time direction (components in {-1,0,1}).
template <class L, int I, class V>
__device__ __forceinline__ V cdot(V vx, V vy, V vz) {
  constexpr int cx = L::cx[I], cy = L::cy[I], cz = L::cz[I];
  if constexpr (cx == 0 && cy == 0 && cz == 0) {
    return bc<V>(0);
  } else {
    V r = vx;
    bool have = false;
    if constexpr (cx != 0) { r = cx > 0 ? vx : neg(vx); have = true; }
    if constexpr (cy != 0) {
      if (have) r = cy > 0 ? add(r, vy) : sub(r, vy);
      else r = cy > 0 ? vy : neg(vy);
      have = true;
    }
    if constexpr (cz != 0) {
      if (have) r = cz > 0 ? add(r, vz) : sub(r, vz);
      else r = cz > 0 ? vz : neg(vz);
    }
    return r;
  }
}

// Accumulate sign * v into acc (first term initialises).
template <int SIGN, class V>
__device__ __forceinline__ void acc_signed(V& acc, bool& have, V v) {
  if constexpr (SIGN != 0) {
    if (have) acc = SIGN > 0 ? add(acc, v) : sub(acc, v);
    else acc = SIGN > 0 ? v : neg(v);
    have = true;
  }
}

// Density sum and momentum over opposite pairs (BGK.hpp:63-78, regrouped):
// with sp = f_i + f_opp and dm = f_i - f_opp, sum f = f_0 + sum sp and
// sum c f = sum c_i dm.
template <class L, class V>
__device__ __forceinline__ void pair_sums(const V* f, V& dens, V& mx, V& my, V& mz) {
  dens = f[0];
  bool hx = false, hy = false, hz = false;
  static_for<1, L::Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    const V sp = add(f[i], f[i + 1]);
    const V dm = sub(f[i], f[i + 1]);
    dens = add(dens, sp);
    acc_signed<L::cx[i]>(mx, hx, dm);
    acc_signed<L::cy[i]>(my, hy, dm);
    acc_signed<L::cz[i]>(mz, hz, dm);
  });
  if (!hz) mz = bc<V>(0);
}

// rho, u from (dens, momentum), with Guo's half-force velocity shift
// u += F / (2 rho) (Forcing.hpp:66-70).
template <bool SH, bool FORCE, class V, class S, class FV>
__device__ __forceinline__ Macro<V> finish_macro(V dens, V mx, V my, V mz,
                                                 const CollideParams<S, FV>& p) {
  Macro<V> m;
  m.dens = dens;
  m.rho = SH ? add(bc<V>(S(1)), dens) : dens;
  const V ir = rcp(m.rho);
  m.ux = mul(mx, ir);
  m.uy = mul(my, ir);
  m.uz = mul(mz, ir);
  if constexpr (FORCE) {
    const V h = mul(bc<V>(S(0.5)), ir);
    m.ux = fma(h, fvec<V>(p.fx), m.ux);
    m.uy = fma(h, fvec<V>(p.fy), m.uy);
    m.uz = fma(h, fvec<V>(p.fz), m.uz);
  }
  return m;
}

// ------------------------------------------------------------ equilibria
// Product-form factor per axis, chi(c, u) = 1 + delta(c, u):
//   delta(0) = -1.5 u^2, delta(+-1) = 3 u^2 +- 3 u   (Equilibrium.hpp:71-124),
// indexed by c + 1.
template <class V, class S>
__device__ __forceinline__ void chi_deltas(V u, V d[3]) {
  const V u2 = mul(u, u);
  const V t3u2 = mul(bc<V>(S(3)), u2);
  const V t3u = mul(bc<V>(S(3)), u);
  d[0] = sub(t3u2, t3u);
  d[1] = mul(bc<V>(S(-1.5)), u2);
  d[2] = add(t3u2, t3u);
}

// phi_i = prod_a (1 + delta_a) - 1, expanded so that no term of size one is
// formed (the same polynomial as the reference's chi products).
template <class L, int I, class V>
__device__ __forceinline__ V phi_product(const V* dx, const V* dy, const V* dz) {
  constexpr int ix = L::cx[I] + 1, iy = L::cy[I] + 1, iz = L::cz[I] + 1;
  const V a = dx[ix], b = dy[iy];
  const V pxy = fma(a, b, add(a, b));
  if constexpr (L::D == 3) {
    const V c = dz[iz];
    return fma(c, add(bc<V>(1), pxy), pxy);
  } else {
    return pxy;
  }
}

// ------------------------------------------------------------ BGK / TRT
// BGK: f += omega (feq - f) + (1 - omega/2) S          (BGK.hpp:81-92)
// TRT: even part relaxed at omega_p, odd part at omega_m (TRT.hpp:92-127)
// feq_i = w_i (D0 + rho phi_i), D0 = rho - 1 (shifted) or rho (raw).
// Second-order phi of a pair (c, -c): A +- B with A = 4.5 (c.u)^2 - 1.5 u.u,
// B = 3 c.u (Equilibrium.hpp:49-60).  Guo source of a pair: sym +- anti with
// sym = w (9 (c.u)(c.F) - 3 u.F), anti = 3 w c.F (Forcing.hpp:26-38).
template <class L, int OP, int EQ, bool SH, bool FORCE, class V, class S, class FV>
__device__ __forceinline__ void collide_bgk_trt(V* f, const Macro<V>& m,
                                                const CollideParams<S, FV>& p) {
  const V om = bc<V>(p.omega);
  const V D0 = SH ? m.dens : m.rho;
  const V uu = fma(m.uz, m.uz, fma(m.uy, m.uy, mul(m.ux, m.ux)));
  const V m15uu = mul(bc<V>(S(-1.5)), uu);
  V m3uF = bc<V>(0);
  if constexpr (FORCE)
    m3uF = mul(bc<V>(S(-3)),
               fma(m.uz, fvec<V>(p.fz), fma(m.uy, fvec<V>(p.fy), mul(m.ux, fvec<V>(p.fx)))));
  V dx[3], dy[3], dz[3];
  if constexpr (EQ == 1) {
    chi_deltas<V, S>(m.ux, dx);
    chi_deltas<V, S>(m.uy, dy);
    if constexpr (L::D == 3) chi_deltas<V, S>(m.uz, dz);
  }
  // Relaxation rates: BGK uses omega for both parts.
  const S wp = p.omega;
  const S wm = OP == 2 ? p.omega2 : p.omega;
  const S cp = S(1) - S(0.5) * wp;
  const S cm = S(1) - S(0.5) * wm;

  // rest population: opp(0) == 0, purely even
  {
    constexpr S w0 = S(weight<L, 0>());
    V ph;
    if constexpr (EQ == 1) ph = phi_product<L, 0>(dx, dy, dz);
    else ph = m15uu;
    const V feq = mul(bc<V>(w0), fma(m.rho, ph, D0));
    f[0] = fma(bc<V>(wp), sub(feq, f[0]), f[0]);
    if constexpr (FORCE) f[0] = fma(bc<V>(cp * w0), m3uF, f[0]);
  }
  static_for<1, L::Q, 2>([&](auto I) {
    constexpr int i = decltype(I)::value;
    constexpr int j = i + 1;
    constexpr S w = S(weight<L, i>());
    const V cu = cdot<L, i>(m.ux, m.uy, m.uz);
    // even / odd parts of the equilibrium of the pair (i, j)
    V ep, em;
    if constexpr (EQ == 0) {
      const V A = fma(mul(bc<V>(S(4.5)), cu), cu, m15uu);
      ep = mul(bc<V>(w), fma(m.rho, A, D0));
      em = mul(mul(bc<V>(S(3) * w), m.rho), cu);
    } else {
      const V ei = mul(bc<V>(w), fma(m.rho, phi_product<L, i>(dx, dy, dz), D0));
      const V ej = mul(bc<V>(w), fma(m.rho, phi_product<L, j>(dx, dy, dz), D0));
      ep = mul(bc<V>(S(0.5)), add(ei, ej));
      em = mul(bc<V>(S(0.5)), sub(ei, ej));
    }
    V ssym = bc<V>(0), santi = bc<V>(0);
    if constexpr (FORCE) {
      const V cF = cdot<L, i>(fvec<V>(p.fx), fvec<V>(p.fy), fvec<V>(p.fz));
      ssym = mul(bc<V>(w), fma(mul(bc<V>(S(9)), cu), cF, m3uF));
      santi = mul(bc<V>(S(3) * w), cF);
    }
    if constexpr (OP == 1) {
      // BGK: relax each member towards feq = ep +- em.
      const V fi = fma(om, sub(add(ep, em), f[i]), f[i]);
      const V fj = fma(om, sub(sub(ep, em), f[j]), f[j]);
      if constexpr (FORCE) {
        f[i] = fma(bc<V>(cp), add(ssym, santi), fi);
        f[j] = fma(bc<V>(cp), sub(ssym, santi), fj);
      } else {
        f[i] = fi;
        f[j] = fj;
      }
    } else {
      // TRT: half-sums relaxed separately, then recombined.
      const V hp = mul(bc<V>(S(0.5)), add(f[i], f[j]));
      const V hm = mul(bc<V>(S(0.5)), sub(f[i], f[j]));
      V sp = fma(bc<V>(wp), sub(ep, hp), hp);
      V sm = fma(bc<V>(wm), sub(em, hm), hm);
      if constexpr (FORCE) {
        sp = fma(bc<V>(cp), ssym, sp);
        sm = fma(bc<V>(cm), santi, sm);
      }
      f[i] = add(sp, sm);
      f[j] = sub(sp, sm);
    }
  });
}

// ------------------------------------------------------ moment operators
// Product basis {1, C, C^2 - cs2} per axis with C = c - u_b; u_b = u for
// central moments and 0 for raw MRT (ProductBasis.hpp:1-205,
// MomentCollision.hpp:1-48).  Moments are indexed (p*3 + q)*3 + r.
//
// Forward: only the ten moments of order <= 2 are formed, from monomial sums
// (1, c, c^2) per axis; orders >= 3 are replaced by their equilibrium anyway
// (MomentCollision.hpp:211-222).  The monomial sums give the density and the
// momentum as a by-product, so no separate macroscopic pass is needed.
template <class L, class V>
__device__ __forceinline__ void monomial_low(const V* f, V N[10]) {
  // N order: 000 100 010 001 200 020 002 110 101 011
  if constexpr (L::D == 3) {
    V Z[3][3][3];  // Z[r][a][b] = sum over cz of cz^r f(a, b, cz)
    static_for<0, 9>([&](auto AB) {
      constexpr int a = decltype(AB)::value / 3, b = decltype(AB)::value % 3;
      constexpr int im = dir_of<L>(a - 1, b - 1, -1), i0 = dir_of<L>(a - 1, b - 1, 0),
                    ip = dir_of<L>(a - 1, b - 1, 1);
      const V t = add(f[ip], f[im]);
      Z[0][a][b] = add(t, f[i0]);
      Z[1][a][b] = sub(f[ip], f[im]);
      Z[2][a][b] = t;
    });
    V Y0[3][3], Y1[3][2], Y2[3];  // Y_q[a][r]
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const V t = add(Z[0][a][2], Z[0][a][0]);
      Y0[a][0] = add(t, Z[0][a][1]);
      Y1[a][0] = sub(Z[0][a][2], Z[0][a][0]);
      Y2[a] = t;
      Y0[a][1] = add(add(Z[1][a][2], Z[1][a][0]), Z[1][a][1]);
      Y1[a][1] = sub(Z[1][a][2], Z[1][a][0]);
      Y0[a][2] = add(add(Z[2][a][2], Z[2][a][0]), Z[2][a][1]);
    }
    const V t = add(Y0[2][0], Y0[0][0]);
    N[0] = add(t, Y0[1][0]);                          // 000
    N[1] = sub(Y0[2][0], Y0[0][0]);                   // 100
    N[2] = add(add(Y1[2][0], Y1[0][0]), Y1[1][0]);    // 010
    N[3] = add(add(Y0[2][1], Y0[0][1]), Y0[1][1]);    // 001
    N[4] = t;                                         // 200
    N[5] = add(add(Y2[2], Y2[0]), Y2[1]);             // 020
    N[6] = add(add(Y0[2][2], Y0[0][2]), Y0[1][2]);    // 002
    N[7] = sub(Y1[2][0], Y1[0][0]);                   // 110
    N[8] = sub(Y0[2][1], Y0[0][1]);                   // 101
    N[9] = add(add(Y1[2][1], Y1[0][1]), Y1[1][1]);    // 011
  } else {
    V Y0[3], Y1[3], Y2[3];  // over cy for each x index a
    static_for<0, 3>([&](auto A) {
      constexpr int a = decltype(A)::value;
      constexpr int im = dir_of<L>(a - 1, -1, 0), i0 = dir_of<L>(a - 1, 0, 0),
                    ip = dir_of<L>(a - 1, 1, 0);
      const V t = add(f[ip], f[im]);
      Y0[a] = add(t, f[i0]);
      Y1[a] = sub(f[ip], f[im]);
      Y2[a] = t;
    });
    const V t = add(Y0[2], Y0[0]);
    N[0] = add(t, Y0[1]);
    N[1] = sub(Y0[2], Y0[0]);
    N[2] = add(add(Y1[2], Y1[0]), Y1[1]);
    N[3] = bc<V>(0);
    N[4] = t;
    N[5] = add(add(Y2[2], Y2[0]), Y2[1]);
    N[6] = bc<V>(0);
    N[7] = sub(Y1[2], Y1[0]);
    N[8] = bc<V>(0);
    N[9] = bc<V>(0);
  }
}

// One inverse 1D pass (ProductBasis.hpp:148-156): moments (m0, m1, m2) at
// basis velocity u -> values at c = -1, 0, +1.  uu2 = 2u, mq = cs2 - u^2.
template <class V, class S, bool ZERO_U>
__device__ __forceinline__ void inv1d(V& a, V& b, V& c, V u, V uu2, V mq) {
  const V m0 = a, m1 = b, m2 = c;
  V s1, s2;
  if constexpr (ZERO_U) {
    s1 = m1;
    s2 = fma(bc<V>(S(1) / S(3)), m0, m2);
  } else {
    s1 = fma(u, m0, m1);
    s2 = fma(mq, m0, fma(uu2, s1, m2));
  }
  const V q2 = mul(bc<V>(S(0.5)), s2);
  a = fma(bc<V>(S(-0.5)), s1, q2);
  b = sub(m0, s2);
  c = fma(bc<V>(S(0.5)), s1, q2);
}

// Equilibrium moment (p, q, r) as the product of per-axis factors E1[a][k].
template <int D, int P, int Qq, int Rr, class V>
__device__ __forceinline__ V eqm(const V (&E1)[3][3]) {
  V e = E1[0][P];
  if constexpr (Qq != 0) e = mul(e, E1[1][Qq]);
  if constexpr (D == 3 && Rr != 0) e = mul(e, E1[2][Rr]);
  return e;
}

template <class L, int OP, bool SH, bool FORCE, class V, class S, class FV>
__device__ __forceinline__ void collide_moments(V* f, Macro<V>& m, const CollideParams<S, FV>& p) {
  constexpr bool central = (OP == 4);
  constexpr int D = L::D;
  constexpr S cs2 = S(1) / S(3);
  V N[10];
  monomial_low<L>(f, N);
  m = finish_macro<SH, FORCE>(N[0], N[1], N[2], N[3], p);
  const V u[3] = {m.ux, m.uy, m.uz};
  const V rho = m.rho;

  // ---- order <= 2 moments in the product basis at u_b
  V K0, K1[3], K2d[3], K2s[3];  // K2s: 110 101 011
  // the -cs2 rho term enters each diagonal moment through one explicit FMA:
  // as a separate product followed by an add, the compiler could fuse the
  // two in the paired kernels only (lbm_common.cuh)
  const V mcs = bc<V>(-cs2);
  K0 = N[0];
  if constexpr (central) {
#pragma unroll
    for (int a = 0; a < 3; ++a) K1[a] = fma(neg(u[a]), N[0], N[1 + a]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
      K2d[a] = fma(mcs, N[0], fma(neg(u[a]), add(N[1 + a], K1[a]), N[4 + a]));
    K2s[0] = fma(neg(u[1]), K1[0], fma(neg(u[0]), N[2], N[7]));
    K2s[1] = fma(neg(u[2]), K1[0], fma(neg(u[0]), N[3], N[8]));
    K2s[2] = fma(neg(u[2]), K1[1], fma(neg(u[1]), N[3], N[9]));
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) K1[a] = N[1 + a];
#pragma unroll
    for (int a = 0; a < 3; ++a) K2d[a] = fma(mcs, N[0], N[4 + a]);
    K2s[0] = N[7];
    K2s[1] = N[8];
    K2s[2] = N[9];
  }

  // ---- equilibrium moments in the stored variable (MomentCollision.hpp:192-201)
  // central: k_eq = rho [N==0] - W, W = prod A(p, u_a), A = {1, -u, u^2}
  // raw:     k_eq = rho prod u_a^p - [N==0]  (shifted)   or  rho prod u_a^p (raw)
  V E1[3][3];  // per-axis factors, E[N] = E1[0][p] * E1[1][q] * E1[2][r] (+ offset)
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if constexpr (central) {
      // -W: fold the sign into the x factor
      E1[a][0] = bc<V>(a == 0 ? S(-1) : S(1));
      E1[a][1] = a == 0 ? u[a] : neg(u[a]);
      E1[a][2] = a == 0 ? neg(mul(u[a], u[a])) : mul(u[a], u[a]);
    } else {
      E1[a][0] = a == 0 ? rho : bc<V>(1);
      E1[a][1] = a == 0 ? mul(rho, u[a]) : u[a];
      E1[a][2] = a == 0 ? mul(E1[a][1], u[a]) : mul(u[a], u[a]);
    }
  }
  // second-order equilibria
  V e2d[3], e2s[3];
  if constexpr (central) {
    if constexpr (SH) {
      e2d[0] = eqm<D, 2, 0, 0>(E1); e2d[1] = eqm<D, 0, 2, 0>(E1); e2d[2] = eqm<D, 0, 0, 2>(E1);
      e2s[0] = eqm<D, 1, 1, 0>(E1); e2s[1] = eqm<D, 1, 0, 1>(E1); e2s[2] = eqm<D, 0, 1, 1>(E1);
    } else {
#pragma unroll
      for (int a = 0; a < 3; ++a) { e2d[a] = bc<V>(0); e2s[a] = bc<V>(0); }
    }
  } else {
    e2d[0] = eqm<D, 2, 0, 0>(E1); e2d[1] = eqm<D, 0, 2, 0>(E1); e2d[2] = eqm<D, 0, 0, 2>(E1);
    e2s[0] = eqm<D, 1, 1, 0>(E1); e2s[1] = eqm<D, 1, 0, 1>(E1); e2s[2] = eqm<D, 0, 1, 1>(E1);
  }

  // ---- relaxation (MomentCollision.hpp:263-288)
  const S om = p.omega;
  const S wb = p.omega2 < S(0) ? p.omega : p.omega2;
  const S w2 = S(1) - S(0.5) * om;
  const S invD = S(1) / S(D);
  const V F[3] = {fvec<V>(p.fx), fvec<V>(p.fy), fvec<V>(p.fz)};
  if constexpr (FORCE) {
#pragma unroll
    for (int a = 0; a < D; ++a) K1[a] = add(K1[a], F[a]);
  }
  {
    V tr = K2d[0], tre = e2d[0];
#pragma unroll
    for (int a = 1; a < D; ++a) { tr = add(tr, K2d[a]); tre = add(tre, e2d[a]); }
    V g[3], trg = bc<V>(0);
    constexpr bool force2 = FORCE && !central;  // 2 F_a du_a, zero for central
    if constexpr (force2) {
#pragma unroll
      for (int a = 0; a < D; ++a) g[a] = mul(mul(bc<V>(S(2)), F[a]), u[a]);
      trg = g[0];
#pragma unroll
      for (int a = 1; a < D; ++a) trg = add(trg, g[a]);
    }
    V trpost = fma(bc<V>(wb), tre, mul(bc<V>(S(1) - wb), tr));
    if constexpr (force2) trpost = fma(bc<V>(S(1) - S(0.5) * wb), trg, trpost);
    const V trD = mul(tr, bc<V>(invD)), treD = mul(tre, bc<V>(invD)),
            trpD = mul(trpost, bc<V>(invD));
    V trgD;
    if constexpr (force2) trgD = mul(trg, bc<V>(invD));
#pragma unroll
    for (int a = 0; a < D; ++a) {
      V k = fma(bc<V>(S(1) - om), sub(K2d[a], trD), trpD);
      k = fma(bc<V>(om), sub(e2d[a], treD), k);
      if constexpr (force2) k = fma(bc<V>(w2), sub(g[a], trgD), k);
      K2d[a] = k;
    }
    // shear: (1 - omega) k + omega e + w2 (F_b du_a + F_a du_b)
    constexpr int ns = D == 3 ? 3 : 1;
    constexpr int sa[3] = {0, 0, 1}, sb[3] = {1, 2, 2};
#pragma unroll
    for (int s = 0; s < ns; ++s) {
      V k = fma(bc<V>(om), e2s[s], mul(bc<V>(S(1) - om), K2s[s]));
      if constexpr (force2) {
        const V ge = fma(F[sa[s]], u[sb[s]], mul(F[sb[s]], u[sa[s]]));
        k = fma(bc<V>(w2), ge, k);
      }
      K2s[s] = k;
    }
  }

  // ---- assemble all moments; order >= 3 at equilibrium
  constexpr int NM = D == 3 ? 27 : 9;
  V K[NM];
  static_for<0, NM>([&](auto NN) {
    constexpr int n = decltype(NN)::value;
    constexpr int pp = D == 3 ? n / 9 : n / 3;
    constexpr int qq = D == 3 ? (n / 3) % 3 : n % 3;
    constexpr int rr = D == 3 ? n % 3 : 0;
    constexpr int ord = pp + qq + rr;
    if constexpr (ord == 0) K[n] = K0;
    else if constexpr (ord == 1) K[n] = K1[pp ? 0 : (qq ? 1 : 2)];
    else if constexpr (ord == 2 && (pp == 2 || qq == 2 || rr == 2))
      K[n] = K2d[pp == 2 ? 0 : (qq == 2 ? 1 : 2)];
    else if constexpr (ord == 2)
      K[n] = K2s[(pp && qq) ? 0 : (pp && rr ? 1 : 2)];
    else {
      if constexpr (central && !SH) K[n] = bc<V>(0);
      else K[n] = eqm<D, pp, qq, rr>(E1);
    }
  });

  // ---- inverse transform, x then y then z (ProductBasis.hpp:183-205)
  V ub[3], uu2[3], mq[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ub[a] = central ? u[a] : bc<V>(0);
    if constexpr (central) {
      uu2[a] = add(u[a], u[a]);
      mq[a] = fma(neg(u[a]), u[a], bc<V>(cs2));
    }
  }
  if constexpr (D == 3) {
#pragma unroll
    for (int qr = 0; qr < 9; ++qr)
      inv1d<V, S, !central>(K[qr], K[9 + qr], K[18 + qr], ub[0], uu2[0], mq[0]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int r = 0; r < 3; ++r)
        inv1d<V, S, !central>(K[a * 9 + r], K[a * 9 + 3 + r], K[a * 9 + 6 + r], ub[1], uu2[1],
                              mq[1]);
#pragma unroll
    for (int ab = 0; ab < 9; ++ab)
      inv1d<V, S, !central>(K[ab * 3], K[ab * 3 + 1], K[ab * 3 + 2], ub[2], uu2[2], mq[2]);
    static_for<0, 27>([&](auto NN) {
      constexpr int n = decltype(NN)::value;
      f[dir_of<L>(n / 9 - 1, (n / 3) % 3 - 1, n % 3 - 1)] = K[n];
    });
  } else {
#pragma unroll
    for (int q = 0; q < 3; ++q)
      inv1d<V, S, !central>(K[q], K[3 + q], K[6 + q], ub[0], uu2[0], mq[0]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
      inv1d<V, S, !central>(K[a * 3], K[a * 3 + 1], K[a * 3 + 2], ub[1], uu2[1], mq[1]);
    static_for<0, 9>([&](auto NN) {
      constexpr int n = decltype(NN)::value;
      f[dir_of<L>(n / 3 - 1, n % 3 - 1, 0)] = K[n];
    });
  }
}

// ---------------------------------------------------------------- dispatch
// Collide one node (pair) in place; returns the macroscopic state.
template <class L, int OP, int EQ, bool SH, bool FORCE, class V, class S, class FV>
__device__ __forceinline__ Macro<V> collide(V* f, const CollideParams<S, FV>& p) {
  Macro<V> m;
  if constexpr (OP == 0) {
    m.dens = bc<V>(1); m.rho = bc<V>(1);
    m.ux = m.uy = m.uz = bc<V>(0);
  } else if constexpr (OP == 1 || OP == 2) {
    V dens, mx, my, mz;
    pair_sums<L>(f, dens, mx, my, mz);
    m = finish_macro<SH, FORCE>(dens, mx, my, mz, p);
    collide_bgk_trt<L, OP, EQ, SH, FORCE>(f, m, p);
  } else {
    collide_moments<L, OP, SH, FORCE>(f, m, p);
  }
  return m;
}

// Macroscopic state only (compute_macroscopic, FluidSolver.hpp:1041-1179).
template <class L, int OP, bool SH, bool FORCE, class V, class S, class FV>
__device__ __forceinline__ Macro<V> macroscopic(const V* f, const CollideParams<S, FV>& p) {
  Macro<V> m;
  if constexpr (OP == 0) {
    m.dens = bc<V>(1); m.rho = bc<V>(1);
    m.ux = m.uy = m.uz = bc<V>(0);
  } else {
    V dens, mx, my, mz;
    pair_sums<L>(f, dens, mx, my, mz);
    m = finish_macro<SH, FORCE>(dens, mx, my, mz, p);
  }
  return m;
}

}  // namespace m3lb
