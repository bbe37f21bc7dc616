/*
 * Body of the CPU oracle, included once per arithmetic type by lbm_oracle.c
 * with R (the real type) and P (the symbol prefix) defined.  TEST
 * INFRASTRUCTURE: see lbm_oracle.h.
 *
 * Every routine restates one piece of the reference (paths relative to the
 * M3LB tree) in the same operation order, so that with floating-point
 * contraction off the double build reproduces the reference build bit for bit.
 */
#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define F(name) CAT(P, name)
#define S(name) CAT(CAT(P, s_), name)

typedef struct {
  int lattice, Q, D, op, eq, shifted, forcing, quant;
  int nx, ny, nz, hx, hy, hz, sx, sy, sz, per[3];
  long long n_padded, t;
  R omega, omega2, fx, fy, fz;
  R* f;          /* populations, node-major: f[n*Q + q] (host LayoutRight) */
  uint8_t* flags;
  uint8_t* spec_nrm;   /* SpecWall normal code per padded node */
  uint8_t* spec_faces; /* SpecNode face mask per padded node */
  /* regularised walls (FluidSolver.hpp:97-103, 272-552, 1266-1290), per
   * padded node; the state table is kept per node (u0 = as given) */
  uint8_t *bc_nrm, *bc_ext, *bc_onrm;
  uint32_t* bc_unk;
  long long* bc_don;
  R *bc_rho, *wall_u0, *wall_un;  /* u0: 4 per node (ux, uy, uz, rho) */
  R wall_scale, wall_un_scale, outflow_rho;
  int wall_un_on, has_corners, fd_corners, force_bc, out_order, has_walls;
  /* Boussinesq buoyancy (src/forcing/Forcing.hpp:93-127): per padded node
   * F = f_uniform + g rho0 beta (T - T0) */
  int buoyant;
  R* temp;
  R ufx, ufy, ufz, bgx, bgy, bgz, brho0, bbeta, bT0;
  R *rho, *ux, *uy, *uz; /* stored macroscopic fields (StoreMacro) */
} S(solver);

/* Storage rounding (narrow population storage emulated in R arithmetic). */
static inline R S(q)(const S(solver)* s, R v) {
  if (s->quant == 1) return (R)(_Float16)v;
  if (s->quant == 2) return (R)lbmo_bf16_round((float)v);
  if (s->quant == 3) return (R)lbmo_f16c_round((float)v);
  return v;
}

/* ---- Lattice constants: src/lattice/Lattices.hpp:166-185 ---- */
static inline R S(w)(const S(solver)* s, int i) {
  return s->Q == 9 ? (R)D2Q9_W[i] / (R)36 : (R)D3Q27_W[i] / (R)216;
}
static inline int S(c)(const S(solver)* s, int i, int a) {
  if (s->Q == 9) return a == 0 ? D2Q9_CX[i] : (a == 1 ? D2Q9_CY[i] : 0);
  return a == 0 ? D3Q27_CX[i] : (a == 1 ? D3Q27_CY[i] : D3Q27_CZ[i]);
}

/* ---- Domain: src/grid/Domain.hpp:47-123 ---- */
static int S(halo_for)(int n, int per) {           /* Domain.hpp:104-108 */
  if (n <= 1) return 0;
  if (per) return 0;
  return 1;
}
static inline int S(shift)(int v, int h, int n, int sz, int per) { /* Domain.hpp:113-123 */
  if (per) {
    if (v < h) return v + n;
    if (v >= h + n) return v - n;
    return v;
  }
  if (v < 0) return 0;
  if (v >= sz) return sz - 1;
  return v;
}
static inline long long S(idp)(const S(solver)* s, int x, int y, int z) {
  return ((long long)z * s->sy + y) * s->sx + x;
}
static inline void S(coords)(const S(solver)* s, long long n, int* x, int* y, int* z) {
  *x = (int)(n % s->sx);
  *y = (int)((n / s->sx) % s->sy);
  *z = (int)(n / ((long long)s->sx * s->sy));
}
static inline int S(is_interior)(const S(solver)* s, int x, int y, int z) {
  return x >= s->hx && x < s->hx + s->nx && y >= s->hy && y < s->hy + s->ny &&
         z >= s->hz && z < s->hz + s->nz;
}
/* Neighbour n + c_i for the odd directions (Domain.hpp:82-101); nb[i] valid for odd i. */
static void S(neighbours)(const S(solver)* s, long long n, long long nb[27]) {
  int x, y, z;
  S(coords)(s, n, &x, &y, &z);
  for (int i = 1; i < s->Q; i += 2)
    nb[i] = S(idp)(s, S(shift)(x + S(c)(s, i, 0), s->hx, s->nx, s->sx, s->per[0]),
                   S(shift)(y + S(c)(s, i, 1), s->hy, s->ny, s->sy, s->per[1]),
                   S(shift)(z + S(c)(s, i, 2), s->hz, s->nz, s->sz, s->per[2]));
}

/* ---- Esoteric Pull access: src/memory/EsotericPull.hpp:61-111 ---- */
#define A(node, q) s->f[(node) * s->Q + (q)]
static inline void S(load_all)(const S(solver)* s, int par, long long n, const long long* nb,
                               R* f) {
  f[0] = A(n, 0);                                          /* load_rest */
  for (int i = 1; i < s->Q; i += 2) {                      /* load_pair :88-91 */
    if (par == 0) { f[i] = A(n, i);     f[i + 1] = A(nb[i], i + 1); }
    else          { f[i] = A(n, i + 1); f[i + 1] = A(nb[i], i); }
  }
}
static inline void S(store_all)(S(solver)* s, int par, long long n, const long long* nb,
                                const R* f) {
  A(n, 0) = S(q)(s, f[0]);                                  /* store_rest */
  for (int i = 1; i < s->Q; i += 2) {                       /* store_pair :92-96 */
    if (par == 0) { A(nb[i], i + 1) = S(q)(s, f[i]); A(n, i) = S(q)(s, f[i + 1]); }
    else          { A(nb[i], i) = S(q)(s, f[i]);     A(n, i + 1) = S(q)(s, f[i + 1]); }
  }
}
/* Access::load (:69-77): the population of direction i about to arrive at n. */
static inline R S(load1)(const S(solver)* s, int par, long long n, const long long* nb, int i) {
  if (i == 0) return A(n, 0);
  if (par == 0) return (i & 1) ? A(n, i) : A(nb[i - 1], i);
  return (i & 1) ? A(n, i + 1) : A(nb[i - 1], i - 1);
}
/* Access::scatter (:104-111): exact inverse of load. */
static inline void S(scatter1)(S(solver)* s, int par, long long n, const long long* nb, int i,
                               R v) {
  v = S(q)(s, v);
  if (i == 0) { A(n, 0) = v; return; }
  if (par == 0) { if (i & 1) A(n, i) = v; else A(nb[i - 1], i) = v; }
  else          { if (i & 1) A(n, i + 1) = v; else A(nb[i - 1], i - 1) = v; }
}
#undef A
static inline void S(load_node)(const S(solver)* s, int par, long long n, R* g, int unshift) {
  long long nb[27];
  S(neighbours)(s, n, nb);
  S(load_all)(s, par, n, nb, g);
  if (unshift)
    for (int i = 0; i < s->Q; ++i) g[i] += S(w)(s, i);
}

/* ---- Specular walls: src/boundary/Specular.hpp ---- */
static inline int S(mir)(const S(solver)* s, int a, int i) {
  return s->Q == 9 ? D2Q9_MIR[a][i] : D3Q27_MIR[a][i];
}
static inline int S(mirror_axis)(uint8_t code) {            /* :124-128 */
  return (code == 1 || code == 2) ? 0 : ((code == 3 || code == 4) ? 1 : 2);
}
static inline int S(face_sign)(uint8_t faces, int a) {      /* :238-243 */
  if (faces & (1u << (2 * a))) return 1;
  if (faces & (1u << (2 * a + 1))) return -1;
  return 0;
}
/* mirror_unknowns_faces (:263-278): every direction pointing into the domain
 * across a masked face takes the value of its image, composed over the
 * masked axes it crosses. */
static void S(mirror_faces)(const S(solver)* s, R* f, uint8_t faces) {
  R h[27];
  for (int i = 0; i < s->Q; ++i) h[i] = f[i];
  for (int i = 0; i < s->Q; ++i) {
    int j = i, unknown = 0;
    for (int a = 0; a < 3; ++a) {
      const int sg = S(face_sign)(faces, a);
      if (sg != 0 && S(c)(s, i, a) * sg < 0) { j = S(mir)(s, a, j); unknown = 1; }
    }
    if (unknown) f[i] = h[j];
  }
}

/* ---- Equilibria: src/equilibrium/Equilibrium.hpp:28-124 ---- */
static inline R S(phi_e)(const S(solver)* s, int eqc, int i, R ux, R uy, R uz) {
  const R cx = (R)S(c)(s, i, 0), cy = (R)S(c)(s, i, 1), cz = (R)S(c)(s, i, 2);
  if (eqc == 0) {                                          /* SecondOrderPhi :49-60 */
    const R ics2 = (R)3 / (R)1;
    const R cu = cx * ux + cy * uy + cz * uz;
    const R uu = ux * ux + uy * uy + uz * uz;
    return ics2 * cu + (R)0.5 * ics2 * ics2 * cu * cu - (R)0.5 * ics2 * uu;
  }
  if (s->Q == 9) {                                           /* ProductFormPhi<D2Q9> :71-90 */
    const R cs2v = (R)1 / (R)3;
    const R ax = cx * cx - cs2v;
    const R ay = cy * cy - cs2v;
    const R o1 = (cx * ux + cy * uy) / cs2v;
    const R o2 = (ax * ux * ux + ay * uy * uy + (R)2 * cx * cy * ux * uy) /
                 ((R)2 * cs2v * cs2v);
    const R o3 = (ax * cy * ux * ux * uy + ay * cx * ux * uy * uy) /
                 ((R)2 * cs2v * cs2v * cs2v);
    const R o4 = (ax * ay * ux * ux * uy * uy) / ((R)4 * cs2v * cs2v * cs2v * cs2v);
    return o1 + o2 + o3 + o4;
  }
  /* ProductFormPhi<D3Q27> :110-124: chi = psi(c,u)/w1d(c) per axis */
  const int c3[3] = {S(c)(s, i, 0), S(c)(s, i, 1), S(c)(s, i, 2)};
  const R u3[3] = {ux, uy, uz};
  R chi[3];
  for (int a = 0; a < 3; ++a)
    chi[a] = (c3[a] == 0) ? (R)1 - (R)1.5 * u3[a] * u3[a]
                          : (R)1 + (R)3 * u3[a] * ((R)c3[a] + u3[a]);
  return chi[0] * chi[1] * chi[2] - (R)1;
}
static inline R S(phi)(const S(solver)* s, int i, R ux, R uy, R uz) {
  return S(phi_e)(s, s->eq, i, ux, uy, uz);
}
static inline R S(eq)(const S(solver)* s, int i, R rho, R ux, R uy, R uz) {
  return S(w)(s, i) * rho * ((R)1 + S(phi)(s, i, ux, uy, uz)); /* :34-37 */
}
static inline R S(eq_shifted)(const S(solver)* s, int i, R drho, R ux, R uy, R uz) {
  return S(w)(s, i) * (drho + ((R)1 + drho) * S(phi)(s, i, ux, uy, uz)); /* :40-43 */
}

/* ---- Guo source: src/forcing/Forcing.hpp:26-38 ---- */
static inline R S(guo_raw)(const S(solver)* s, int i, R ux, R uy, R uz) {
  const R ics2 = (R)3 / (R)1;
  const R cx = (R)S(c)(s, i, 0), cy = (R)S(c)(s, i, 1), cz = (R)S(c)(s, i, 2);
  const R cu = cx * ux + cy * uy + cz * uz;
  const R bx = (cx - ux) * ics2 + cu * ics2 * ics2 * cx;
  const R by = (cy - uy) * ics2 + cu * ics2 * ics2 * cy;
  const R bz = (cz - uz) * ics2 + cu * ics2 * ics2 * cz;
  return S(w)(s, i) * (bx * s->fx + by * s->fy + bz * s->fz);
}

/* ---- Macroscopic: src/collision/BGK.hpp:63-78 (TRT.hpp:69-84, MomentCollision.hpp:103-123) */
typedef struct { R dens, ux, uy, uz; } S(macro_t);
static inline R S(density)(const S(solver)* s, R dens) {       /* BGK.hpp:57-60 */
  if (s->op == 0) return dens;
  return s->shifted ? (R)1 + dens : dens;
}
static S(macro_t) S(macroscopic)(const S(solver)* s, const R* f) {
  S(macro_t) m;
  if (s->op == 0) { m.dens = (R)1; m.ux = m.uy = m.uz = (R)0; return m; } /* no-collision mock */
  R sm = 0, mx = 0, my = 0, mz = 0;
  for (int i = 0; i < s->Q; ++i) {
    sm += f[i];
    mx += f[i] * (R)S(c)(s, i, 0);
    my += f[i] * (R)S(c)(s, i, 1);
    mz += f[i] * (R)S(c)(s, i, 2);
  }
  m.dens = sm;
  const R rho = S(density)(s, sm);
  const R ir = (R)1 / rho;
  m.ux = mx * ir; m.uy = my * ir; m.uz = mz * ir;
  if (s->forcing) {                                            /* Forcing.hpp:66-70 */
    const R h = (R)0.5 / rho;
    m.ux += h * s->fx; m.uy += h * s->fy; m.uz += h * s->fz;
  }
  return m;
}

/* ---- BGK: src/collision/BGK.hpp:81-92 ---- */
static void S(collide_bgk)(const S(solver)* s, R* f, S(macro_t) m) {
  for (int i = 0; i < s->Q; ++i) {
    const R feq = s->shifted ? S(eq_shifted)(s, i, m.dens, m.ux, m.uy, m.uz)
                             : S(eq)(s, i, m.dens, m.ux, m.uy, m.uz);
    f[i] += s->omega * (feq - f[i]);
    if (s->forcing) f[i] += ((R)1 - (R)0.5 * s->omega) * S(guo_raw)(s, i, m.ux, m.uy, m.uz);
  }
}

/* ---- TRT: src/collision/TRT.hpp:92-127 ---- */
static void S(collide_trt)(const S(solver)* s, R* f, S(macro_t) m) {
  R e[27], sr[27];
  for (int i = 0; i < s->Q; ++i)
    e[i] = s->shifted ? S(eq_shifted)(s, i, m.dens, m.ux, m.uy, m.uz)
                      : S(eq)(s, i, m.dens, m.ux, m.uy, m.uz);
  if (s->forcing)
    for (int i = 0; i < s->Q; ++i) sr[i] = S(guo_raw)(s, i, m.ux, m.uy, m.uz);
  const R wp = s->omega, wm = s->omega2;
  const R cp = (R)1 - (R)0.5 * wp;
  const R cm = (R)1 - (R)0.5 * wm;
  f[0] += wp * (e[0] - f[0]);
  if (s->forcing) f[0] += cp * sr[0];
  for (int i = 1; i < s->Q; i += 2) {
    const int j = i + 1;
    const R fp = (R)0.5 * (f[i] + f[j]);
    const R fm = (R)0.5 * (f[i] - f[j]);
    const R ep = (R)0.5 * (e[i] + e[j]);
    const R em = (R)0.5 * (e[i] - e[j]);
    R dp = wp * (ep - fp);
    R dm = wm * (em - fm);
    if (s->forcing) {
      dp += cp * (R)0.5 * (sr[i] + sr[j]);
      dm += cm * (R)0.5 * (sr[i] - sr[j]);
    }
    f[i] += dp + dm;
    f[j] += dp - dm;
  }
}

/* ---- Product basis: src/collision/ProductBasis.hpp:118-205 ---- */
/* Population index for component indices a,b,c in {0,1,2} (velocity -1,0,+1). */
static inline int S(pi)(const S(solver)* s, int a, int b, int c) {
  if (s->Q == 9) return D2Q9_DIR[a][b];
  return D3Q27_DIR[a][b][c];
}
static inline void S(fwd1d)(R* a, R* b, R* c, R u) {          /* :138-146 */
  const R cs2v = (R)1 / (R)3;
  const R s0 = *a + *b + *c;
  const R s1 = *c - *a;
  const R s2 = *c + *a;
  *a = s0;
  *b = s1 - u * s0;
  *c = s2 - (R)2 * u * s1 + (u * u - cs2v) * s0;
}
static inline void S(inv1d)(R* a, R* b, R* c, R u) {          /* :148-156 */
  const R cs2v = (R)1 / (R)3;
  const R m0 = *a, m1 = *b, m2 = *c;
  const R s1 = m1 + u * m0;
  const R s2 = m2 + (R)2 * u * s1 - (u * u - cs2v) * m0;
  *a = (R)0.5 * (s2 - s1);
  *b = m0 - s2;
  *c = (R)0.5 * (s2 + s1);
}
#define MI3(p, q, r) (((p) * 3 + (q)) * 3 + (r))
#define MI2(p, q) ((p) * 3 + (q))
static void S(to_moments)(const S(solver)* s, const R* f, const R ub[3], R* k) { /* :159-181 */
  if (s->D == 2) {
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) k[a * 3 + b] = f[S(pi)(s, a, b, 1)];
    for (int a = 0; a < 3; ++a) S(fwd1d)(&k[a * 3 + 0], &k[a * 3 + 1], &k[a * 3 + 2], ub[1]);
    for (int q = 0; q < 3; ++q) S(fwd1d)(&k[0 * 3 + q], &k[1 * 3 + q], &k[2 * 3 + q], ub[0]);
  } else {
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) k[MI3(a, b, c)] = f[S(pi)(s, a, b, c)];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        S(fwd1d)(&k[MI3(a, b, 0)], &k[MI3(a, b, 1)], &k[MI3(a, b, 2)], ub[2]);
    for (int a = 0; a < 3; ++a)
      for (int r = 0; r < 3; ++r)
        S(fwd1d)(&k[MI3(a, 0, r)], &k[MI3(a, 1, r)], &k[MI3(a, 2, r)], ub[1]);
    for (int q = 0; q < 3; ++q)
      for (int r = 0; r < 3; ++r)
        S(fwd1d)(&k[MI3(0, q, r)], &k[MI3(1, q, r)], &k[MI3(2, q, r)], ub[0]);
  }
}
static void S(to_populations)(const S(solver)* s, R* k, const R ub[3], R* f) { /* :183-205 */
  if (s->D == 2) {
    for (int q = 0; q < 3; ++q) S(inv1d)(&k[0 * 3 + q], &k[1 * 3 + q], &k[2 * 3 + q], ub[0]);
    for (int a = 0; a < 3; ++a) S(inv1d)(&k[a * 3 + 0], &k[a * 3 + 1], &k[a * 3 + 2], ub[1]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) f[S(pi)(s, a, b, 1)] = k[a * 3 + b];
  } else {
    for (int q = 0; q < 3; ++q)
      for (int r = 0; r < 3; ++r)
        S(inv1d)(&k[MI3(0, q, r)], &k[MI3(1, q, r)], &k[MI3(2, q, r)], ub[0]);
    for (int a = 0; a < 3; ++a)
      for (int r = 0; r < 3; ++r)
        S(inv1d)(&k[MI3(a, 0, r)], &k[MI3(a, 1, r)], &k[MI3(a, 2, r)], ub[1]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        S(inv1d)(&k[MI3(a, b, 0)], &k[MI3(a, b, 1)], &k[MI3(a, b, 2)], ub[2]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int c = 0; c < 3; ++c) f[S(pi)(s, a, b, c)] = k[MI3(a, b, c)];
  }
}

/* ---- Moment collision: src/collision/MomentCollision.hpp:192-330 ---- */
/* Moment slot n -> exponents (p, q, r): ProductBasis.hpp:97-107. */
static inline void S(pqr)(const S(solver)* s, int n, int* p, int* q, int* r) {
  if (s->D == 2) { *p = n / 3; *q = n % 3; *r = 0; }
  else { *p = n / 9; *q = (n / 3) % 3; *r = n % 3; }
}
static inline R S(eq_moment)(const S(solver)* s, int n, R rho, R Qf[3][3], R Aw[3][3]) {
  int p, q, r;                                               /* eq_moment<N> :192-201 */
  S(pqr)(s, n, &p, &q, &r);
  R e = rho * Qf[0][p] * Qf[1][q];
  R w = Aw[0][p] * Aw[1][q];
  if (s->D == 3) { e *= Qf[2][r]; w *= Aw[2][r]; }
  return s->shifted ? e - w : e;
}
static void S(collide_moment)(const S(solver)* s, R* f, S(macro_t) m) { /* :234-314 */
  const int D = s->D, NM = s->Q, central = (s->op == 4);
  const R rho = S(density)(s, m.dens);
  const R u[3] = {m.ux, m.uy, m.uz};
  R ub[3], du[3];
  for (int a = 0; a < 3; ++a) {
    ub[a] = central ? u[a] : (R)0;
    du[a] = u[a] - ub[a];
  }
  R Qf[3][3], Aw[3][3];
  for (int a = 0; a < 3; ++a) {                              /* ProductBasis::eq_1d */
    Qf[a][0] = (R)1; Qf[a][1] = du[a]; Qf[a][2] = du[a] * du[a];
    Aw[a][0] = (R)1; Aw[a][1] = -ub[a]; Aw[a][2] = ub[a] * ub[a];
  }
  R k[27];
  S(to_moments)(s, f, ub, k);
  const R Fv[3] = {s->forcing ? s->fx : (R)0, s->forcing ? s->fy : (R)0,
                   s->forcing ? s->fz : (R)0};
  const R w2 = (R)1 - (R)0.5 * s->omega;
  const R wb = s->omega2 < (R)0 ? s->omega : s->omega2;      /* bulk() :89-91 */
  /* slots located through the basis (i1/i2d/i2s :340-372) */
  int i1[3], i2d[3];
  if (D == 2) { i1[0] = MI2(1, 0); i1[1] = MI2(0, 1); i2d[0] = MI2(2, 0); i2d[1] = MI2(0, 2); }
  else {
    i1[0] = MI3(1, 0, 0); i1[1] = MI3(0, 1, 0); i1[2] = MI3(0, 0, 1);
    i2d[0] = MI3(2, 0, 0); i2d[1] = MI3(0, 2, 0); i2d[2] = MI3(0, 0, 2);
  }
  if (s->forcing)
    for (int a = 0; a < D; ++a) k[i1[a]] += Fv[a];
  {
    R d[3], e[3], g[3];
    R tr = 0, tre = 0, trg = 0;
    for (int a = 0; a < D; ++a) {
      d[a] = k[i2d[a]];
      e[a] = S(eq_moment)(s, i2d[a], rho, Qf, Aw);
      g[a] = s->forcing ? (R)2 * Fv[a] * du[a] : (R)0;
      tr += d[a]; tre += e[a]; trg += g[a];
    }
    const R invD = (R)1 / (R)D;
    const R tr_post = ((R)1 - wb) * tr + wb * tre + ((R)1 - (R)0.5 * wb) * trg;
    for (int a = 0; a < D; ++a)
      k[i2d[a]] = ((R)1 - s->omega) * (d[a] - tr * invD) + s->omega * (e[a] - tre * invD) +
                  w2 * (g[a] - trg * invD) + tr_post * invD;
    for (int a = 0; a < D; ++a)
      for (int b = a + 1; b < D; ++b) {
        const int id = (D == 2) ? MI2(1, 1)
                                : MI3((a == 0 || b == 0), (a == 1 || b == 1), (a == 2 || b == 2));
        const R ge = s->forcing ? (Fv[b] * du[a] + Fv[a] * du[b]) : (R)0;
        k[id] = ((R)1 - s->omega) * k[id] + s->omega * S(eq_moment)(s, id, rho, Qf, Aw) + w2 * ge;
      }
  }
  for (int n = 0; n < NM; ++n) {                             /* relax_high :211-222 */
    int p, q, r;
    S(pqr)(s, n, &p, &q, &r);
    if (p + q + r >= 3) k[n] = S(eq_moment)(s, n, rho, Qf, Aw);
  }
  S(to_populations)(s, k, ub, f);
}

/* ---- seed_value: BGK.hpp:95-99, TRT.hpp:129-133, MomentCollision.hpp:320-330 ---- */
static R S(seed_value)(const S(solver)* s, int i, R rho, R ux, R uy, R uz) {
  if (s->op == 0) return rho;                                 /* no-collision mock */
  if (s->op == 1 || s->op == 2)
    return s->shifted ? S(eq_shifted)(s, i, rho - (R)1, ux, uy, uz) : S(eq)(s, i, rho, ux, uy, uz);
  const R ub[3] = {0, 0, 0};
  const R du[3] = {ux, uy, uz};
  R Qf[3][3], Aw[3][3];
  for (int a = 0; a < 3; ++a) {
    Qf[a][0] = (R)1; Qf[a][1] = du[a]; Qf[a][2] = du[a] * du[a];
    Aw[a][0] = (R)1; Aw[a][1] = -ub[a]; Aw[a][2] = ub[a] * ub[a];
  }
  R k[27], f[27];
  for (int n = 0; n < s->Q; ++n) k[n] = S(eq_moment)(s, n, rho, Qf, Aw);
  S(to_populations)(s, k, ub, f);
  return f[i];
}

/* ---- Regularised walls: src/boundary/Regularized.hpp ---- */
static void S(normal_of)(uint8_t code, int n[3]) {          /* :153-166 */
  n[0] = n[1] = n[2] = 0;
  if (code >= 1 && code <= 6) n[(code - 1) / 2] = (code & 1) ? 1 : -1;
  else if (code == NRM_OUTXP) n[0] = 1;
}
/* The equilibrium the wall rebuilds against (EquilibriumOf, :47-57): the
 * operator's own for BGK/TRT, the product form for the moment operators,
 * second order for the no-collision mock. */
static inline int S(bc_eq)(const S(solver)* s) { return s->op >= 3 ? 1 : (s->op == 0 ? 0 : s->eq); }
static inline R S(bc_feq)(const S(solver)* s, int i, R rho, R ux, R uy, R uz) {
  return S(w)(s, i) * rho * ((R)1 + S(phi_e)(s, S(bc_eq)(s), i, ux, uy, uz));
}
static inline int S(unshift)(const S(solver)* s) { return s->shifted && s->op != 0; }
static R S(bc_density)(const S(solver)* s, const R* f, const int nrm[3], const R* u) { /* :178-190 */
  R out = 0, tang = 0;
  for (int i = 0; i < s->Q; ++i) {
    const int cn = S(c)(s, i, 0) * nrm[0] + S(c)(s, i, 1) * nrm[1] + S(c)(s, i, 2) * nrm[2];
    if (cn > 0) out += f[i];
    else if (cn == 0) tang += f[i];
  }
  const R uperp = u[0] * (R)nrm[0] + u[1] * (R)nrm[1] + u[2] * (R)nrm[2];
  return ((R)2 * out + tang) / ((R)1 + uperp);
}
static R S(bc_normal_velocity)(const S(solver)* s, const R* f, const int nrm[3], R rho) { /* :196-206 */
  R out = 0, tang = 0;
  for (int i = 0; i < s->Q; ++i) {
    const int cn = S(c)(s, i, 0) * nrm[0] + S(c)(s, i, 1) * nrm[1] + S(c)(s, i, 2) * nrm[2];
    if (cn > 0) out += f[i];
    else if (cn == 0) tang += f[i];
  }
  return ((R)2 * out + tang) / rho - (R)1;
}
/* Q_i : Pi with the off-diagonal terms twice (:226-231, 314-318). */
static inline R S(q_pi)(const S(solver)* s, int i, const R* Pi) {
  const R cs2v = (R)1 / (R)3;
  const R cx = (R)S(c)(s, i, 0), cy = (R)S(c)(s, i, 1), cz = (R)S(c)(s, i, 2);
  const int d3 = s->D == 3;
  return (cx * cx - cs2v) * Pi[0] + (cy * cy - cs2v) * Pi[1] +
         (d3 ? (cz * cz - cs2v) * Pi[2] : (R)0) +
         (R)2 * (cx * cy * Pi[3] + (d3 ? (cx * cz * Pi[4] + cy * cz * Pi[5]) : (R)0));
}
static void S(bc_apply_with_stress)(const S(solver)* s, R* f, R rho, const R* u, const R* Pi) { /* :219-236 */
  const R cs2v = (R)1 / (R)3, cs4v = cs2v * cs2v;
  for (int i = 0; i < s->Q; ++i)
    f[i] = S(bc_feq)(s, i, rho, u[0], u[1], u[2]) + S(w)(s, i) / ((R)2 * cs4v) * S(q_pi)(s, i, Pi);
}
static void S(bc_stress_from_gradient)(R rho, R omega, R g[3][3], R* Pi) { /* :240-250 */
  const R cs2v = (R)1 / (R)3;
  const R k = -(R)2 * cs2v * rho / omega;
  Pi[0] = k * g[0][0];
  Pi[1] = k * g[1][1];
  Pi[2] = k * g[2][2];
  Pi[3] = k * (R)0.5 * (g[0][1] + g[1][0]);
  Pi[4] = k * (R)0.5 * (g[0][2] + g[2][0]);
  Pi[5] = k * (R)0.5 * (g[1][2] + g[2][1]);
}
static inline int S(opp)(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
/* Eqs. (44)-(45) with the forced corrections (:262-328). */
static void S(bc_apply)(const S(solver)* s, R* f, R rho, const R* u, uint32_t unknown, const R* Fv) {
  const R cs2v = (R)1 / (R)3, cs4v = cs2v * cs2v;
  R feq[27];
  for (int i = 0; i < s->Q; ++i) feq[i] = S(bc_feq)(s, i, rho, u[0], u[1], u[2]);
  const R hodd = (R)0.5 / cs2v;
  for (int i = 0; i < s->Q; ++i) {
    if (!(unknown & (1u << i))) continue;
    const R cF = Fv ? ((R)S(c)(s, i, 0) * Fv[0] + (R)S(c)(s, i, 1) * Fv[1] +
                       (R)S(c)(s, i, 2) * Fv[2]) : (R)0;
    const R odd = S(w)(s, i) * hodd * cF;
    const int o = S(opp)(i);
    f[i] = (unknown & (1u << o)) ? feq[i] - odd : feq[i] + (f[o] - feq[o]) - (R)2 * odd;
  }
  R Pi[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < s->Q; ++i) {
    const R d = f[i] - feq[i];
    const R cx = (R)S(c)(s, i, 0), cy = (R)S(c)(s, i, 1), cz = (R)S(c)(s, i, 2);
    Pi[0] += d * cx * cx; Pi[1] += d * cy * cy; Pi[2] += d * cz * cz;
    Pi[3] += d * cx * cy; Pi[4] += d * cx * cz; Pi[5] += d * cy * cz;
  }
  for (int i = 0; i < s->Q; ++i) {
    const R cx = (R)S(c)(s, i, 0), cy = (R)S(c)(s, i, 1), cz = (R)S(c)(s, i, 2);
    const R cF = Fv ? (cx * Fv[0] + cy * Fv[1] + cz * Fv[2]) : (R)0;
    f[i] = feq[i] - S(w)(s, i) * hodd * cF + S(w)(s, i) / ((R)2 * cs4v) * S(q_pi)(s, i, Pi);
  }
}
/* Interior coordinates -> padded index, unwrapped (Domain::id). */
static inline long long S(idi)(const S(solver)* s, long long x, long long y, long long z) {
  return ((z + s->hz) * s->sy + (y + s->hy)) * s->sx + (x + s->hx);
}
/* Wall velocity of a node: the per-node field when set, else its state. */
static inline void S(wall_vel)(const S(solver)* s, long long n, R* uw) {
  for (int a = 0; a < 3; ++a)
    uw[a] = s->wall_un_on ? s->wall_un_scale * s->wall_un[n * 3 + a]
                          : s->wall_u0[n * 4 + a] * s->wall_scale;
}
static inline void S(load_node)(const S(solver)* s, int par, long long n, R* g, int unshift);
/* Velocity at the k-th upstream node of an outflow face (:896-912). */
static void S(up_vel)(const S(solver)* s, int par, long long n, int k, R* v) {
  int px, py, pz;
  S(coords)(s, n, &px, &py, &pz);
  const long long m = S(idi)(s, px - s->hx - k, py - s->hy, pz - s->hz);
  R g[27];
  S(load_node)(s, par, m, g, S(unshift)(s));
  R sm = 0;
  v[0] = v[1] = v[2] = 0;
  for (int i = 0; i < s->Q; ++i) {
    sm += g[i];
    for (int a = 0; a < 3; ++a) v[a] += g[i] * (R)S(c)(s, i, a);
  }
  const R ir = (R)1 / sm;
  for (int a = 0; a < 3; ++a) v[a] *= ir;
}

/* ---- FluidSolver: src/solver/FluidSolver.hpp ---- */
void* F(create)(int lattice, int op, int eq, int shifted, int forcing, int quant, int nx, int ny,
                int nz, int px, int py, int pz, double omega, double omega2, double fx, double fy,
                double fz) {
  if ((lattice != 9 && lattice != 27) || op < 0 || op > 4) return 0;
  S(solver)* s = (S(solver)*)calloc(1, sizeof(S(solver)));
  s->lattice = lattice; s->Q = lattice; s->D = lattice == 9 ? 2 : 3;
  s->op = op; s->eq = eq; s->shifted = shifted; s->forcing = forcing; s->quant = quant;
  s->nx = nx; s->ny = ny; s->nz = nz;
  s->per[0] = px != 0; s->per[1] = py != 0; s->per[2] = pz != 0;
  s->hx = S(halo_for)(nx, s->per[0]); s->hy = S(halo_for)(ny, s->per[1]);
  s->hz = S(halo_for)(nz, s->per[2]);
  s->sx = nx + 2 * s->hx; s->sy = ny + 2 * s->hy; s->sz = nz + 2 * s->hz;
  s->n_padded = (long long)s->sx * s->sy * s->sz;
  s->omega = (R)omega; s->omega2 = (R)omega2;
  s->fx = (R)fx; s->fy = (R)fy; s->fz = (R)fz;
  s->ufx = s->fx; s->ufy = s->fy; s->ufz = s->fz;
  s->temp = (R*)calloc((size_t)s->n_padded, sizeof(R));
  s->f = (R*)calloc((size_t)s->n_padded * s->Q, sizeof(R));
  s->flags = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->spec_nrm = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->spec_faces = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->bc_nrm = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->bc_ext = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->bc_onrm = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->bc_unk = (uint32_t*)calloc((size_t)s->n_padded, sizeof(uint32_t));
  s->bc_don = (long long*)calloc((size_t)s->n_padded, sizeof(long long));
  s->bc_rho = (R*)calloc((size_t)s->n_padded, sizeof(R));
  s->wall_u0 = (R*)calloc((size_t)s->n_padded * 4, sizeof(R));
  s->wall_un = (R*)calloc((size_t)s->n_padded * 3, sizeof(R));
  s->wall_scale = (R)1; s->wall_un_scale = (R)1; s->outflow_rho = (R)1;
  s->fd_corners = op != 0;   /* has_shear_omega: every operator but the no-collision mock */
  s->force_bc = 1; s->out_order = 1;
  s->rho = (R*)calloc((size_t)s->n_padded, sizeof(R));
  s->ux = (R*)calloc((size_t)s->n_padded, sizeof(R));
  s->uy = (R*)calloc((size_t)s->n_padded, sizeof(R));
  s->uz = (R*)calloc((size_t)s->n_padded, sizeof(R));
  for (long long n = 0; n < s->n_padded; ++n) {              /* ctor :57-63 */
    int x, y, z;
    S(coords)(s, n, &x, &y, &z);
    s->flags[n] = S(is_interior)(s, x, y, z) ? 0 : 2;
  }
  return s;
}
void F(destroy)(void* h) {
  S(solver)* s = (S(solver)*)h;
  if (!s) return;
  free(s->f); free(s->flags); free(s->spec_nrm); free(s->spec_faces);
  free(s->bc_nrm); free(s->bc_ext); free(s->bc_onrm); free(s->bc_unk); free(s->bc_don);
  free(s->bc_rho); free(s->wall_u0); free(s->wall_un); free(s->temp); free(s->rho); free(s->ux); free(s->uy); free(s->uz);
  free(s);
}
void F(set_geometry)(void* h, const uint8_t* fl) {           /* :74-82 */
  S(solver)* s = (S(solver)*)h;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x)
        s->flags[S(idp)(s, x + s->hx, y + s->hy, z + s->hz)] =
            fl[((size_t)z * s->ny + y) * s->nx + x];
}
/* set_specular_walls (:193-218): interior normal codes, 0 = leave the node. */
int F(set_specular_walls)(void* h, const uint8_t* codes) {
  S(solver)* s = (S(solver)*)h;
  const size_t nint = (size_t)s->nx * s->ny * s->nz;
  for (size_t k = 0; k < nint; ++k)
    if (codes[k] > 6) return -1;
  memset(s->spec_nrm, 0, (size_t)s->n_padded);
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const uint8_t c = codes[((size_t)z * s->ny + y) * s->nx + x];
        if (c == 0) continue;
        const long long n = S(idp)(s, x + s->hx, y + s->hy, z + s->hz);
        s->spec_nrm[n] = c;
        s->flags[n] = 4;
      }
  return 0;
}
/* set_specular_nodes (:236-268): interior face masks, 0 = leave the node. */
int F(set_specular_nodes)(void* h, const uint8_t* masks) {
  S(solver)* s = (S(solver)*)h;
  const size_t nint = (size_t)s->nx * s->ny * s->nz;
  for (size_t k = 0; k < nint; ++k) {
    const unsigned m = masks[k];
    if (m > 0x3F) return -1;
    for (int a = 0; a < 3; ++a)
      if ((m & (1u << (2 * a))) && (m & (1u << (2 * a + 1)))) return -1;
  }
  memset(s->spec_faces, 0, (size_t)s->n_padded);
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const uint8_t m = masks[((size_t)z * s->ny + y) * s->nx + x];
        if (m == 0) continue;
        const long long n = S(idp)(s, x + s->hx, y + s->hy, z + s->hz);
        s->spec_faces[n] = m;
        s->flags[n] = 5;
      }
  return 0;
}
/* set_regularized_walls (:372-552): normal code per interior node (0 none)
 * and, per node, the state (ux, uy, uz, rho) or NULL for (0, 0, 0, 1).
 * Returns -1 without changes for a code above NrmOutEq, or an NrmOutXp /
 * NrmOutEq node whose upstream stencil leaves the interior (x < 1, or x < 2
 * at outflow order 2). */
int F(set_regularized_walls)(void* h, const uint8_t* codes, const double* spec) {
  S(solver)* s = (S(solver)*)h;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const uint8_t c = codes[((size_t)z * s->ny + y) * s->nx + x];
        if (c > NRM_OUTEQ) return -1;
        if ((c == NRM_OUTXP || c == NRM_OUTEQ) && x < (c == NRM_OUTXP ? s->out_order : 1))
          return -1;
      }
  memset(s->bc_nrm, 0, (size_t)s->n_padded);
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const size_t k = ((size_t)z * s->ny + y) * s->nx + x;
        if (!codes[k]) continue;
        const long long n = S(idi)(s, x, y, z);
        s->bc_nrm[n] = codes[k];
        for (int a = 0; a < 4; ++a) s->wall_u0[n * 4 + a] = spec ? (R)spec[k * 4 + a] : (R)(a == 3);
        s->flags[n] = 3;
      }
  /* corners: an axis direction whose next two nodes are straight walls */
  static const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
  memset(s->bc_ext, 0, (size_t)s->n_padded);
  s->has_corners = 0;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = S(idi)(s, x, y, z);
        if (s->bc_nrm[n] != NRM_CORNER) continue;
        s->has_corners = 1;
        for (int k = 0; k < (s->nz > 1 ? 6 : 4); ++k) {
          const int x1 = x + d6[k][0], y1 = y + d6[k][1], z1 = z + d6[k][2];
          const int x2 = x + 2 * d6[k][0], y2 = y + 2 * d6[k][1], z2 = z + 2 * d6[k][2];
          if (x1 < 0 || y1 < 0 || z1 < 0 || x2 < 0 || y2 < 0 || z2 < 0) continue;
          if (x1 >= s->nx || y1 >= s->ny || z1 >= s->nz) continue;
          if (x2 >= s->nx || y2 >= s->ny || z2 >= s->nz) continue;
          const uint8_t a = s->bc_nrm[S(idi)(s, x1, y1, z1)], b = s->bc_nrm[S(idi)(s, x2, y2, z2)];
          if (a != 0 && a != NRM_CORNER && b != 0 && b != NRM_CORNER) {
            s->bc_ext[n] = (uint8_t)(k + 1);
            break;
          }
        }
      }
  /* unknown directions: the source node is outside the domain, Excluded or Solid */
  memset(s->bc_unk, 0, (size_t)s->n_padded * sizeof(uint32_t));
  const int nn[3] = {s->nx, s->ny, s->nz};
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = S(idi)(s, x, y, z);
        if (!s->bc_nrm[n]) continue;
        uint32_t m = 0;
        for (int i = 0; i < s->Q; ++i) {
          int src[3] = {x - S(c)(s, i, 0), y - S(c)(s, i, 1), z - S(c)(s, i, 2)};
          int outside = 0;
          for (int a = 0; a < 3; ++a) {
            if (s->per[a]) src[a] = (src[a] + nn[a]) % nn[a];
            else if (src[a] < 0 || src[a] >= nn[a]) outside = 1;
          }
          if (!outside) {
            const uint8_t sf = s->flags[S(idi)(s, src[0], src[1], src[2])];
            if (sf == 2 || sf == 1) outside = 1;
          }
          if (outside) m |= 1u << i;
        }
        s->bc_unk[n] = m;
      }
  /* outflow donors: the fluid neighbour opposite the axis step that leaves */
  static const int dd[6][3] = {{-1,0,0},{1,0,0},{0,-1,0},{0,1,0},{0,0,-1},{0,0,1}};
  static const uint8_t dcode[6] = {2, 1, 4, 3, 6, 5};
  for (long long n = 0; n < s->n_padded; ++n) { s->bc_don[n] = n; s->bc_onrm[n] = 0; }
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = S(idi)(s, x, y, z);
        if (s->bc_nrm[n] != NRM_OUTFREE) continue;
        for (int k = 0; k < 6; ++k) {
          const int qx = x + dd[k][0], qy = y + dd[k][1], qz = z + dd[k][2];
          const int leaves = (qx < 0 || qx >= s->nx || qy < 0 || qy >= s->ny || qz < 0 ||
                              qz >= s->nz) || s->flags[S(idi)(s, qx, qy, qz)] == 1;
          if (!leaves) continue;
          const int o = k ^ 1;
          const int rx = x + dd[o][0], ry = y + dd[o][1], rz = z + dd[o][2];
          if (rx < 0 || rx >= s->nx || ry < 0 || ry >= s->ny || rz < 0 || rz >= s->nz) continue;
          const long long m = S(idi)(s, rx, ry, rz);
          if (s->flags[m] != 0) continue;
          s->bc_don[n] = m;
          s->bc_onrm[n] = dcode[k];
          break;
        }
      }
  s->wall_scale = (R)1;
  s->has_walls = 1;
  return 0;
}
void F(set_wall_velocity_scale)(void* h, double sc) { ((S(solver)*)h)->wall_scale = (R)sc; } /* :294-303 */
void F(set_wall_density)(void* h, double r) {                                  /* :328-333 */
  S(solver)* s = (S(solver)*)h;
  for (long long n = 0; n < s->n_padded; ++n) s->wall_u0[n * 4 + 3] = (R)r;
}
void F(set_wall_velocity_field)(void* h, const double* u3) {                     /* :353-368 */
  S(solver)* s = (S(solver)*)h;
  memset(s->wall_un, 0, (size_t)s->n_padded * 3 * sizeof(R));
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const size_t k = ((size_t)z * s->ny + y) * s->nx + x;
        const long long n = S(idi)(s, x, y, z);
        for (int a = 0; a < 3; ++a) s->wall_un[n * 3 + a] = (R)u3[k * 3 + a];
      }
  s->wall_un_on = 1;
  s->wall_un_scale = (R)1;
}
void F(set_wall_velocity_field_scale)(void* h, double sc) { ((S(solver)*)h)->wall_un_scale = (R)sc; }
void F(set_fd_corners)(void* h, int on) { ((S(solver)*)h)->fd_corners = on != 0; }
void F(set_force_correction)(void* h, int on) { ((S(solver)*)h)->force_bc = on != 0; }
int F(set_outflow_order)(void* h, int k) {                                       /* :1324 */
  S(solver)* s = (S(solver)*)h;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < (k >= 2 ? 2 : 1) && x < s->nx; ++x)
        if (s->flags[S(idi)(s, x, y, z)] == 3 && s->bc_nrm[S(idi)(s, x, y, z)] == NRM_OUTXP) return -1;
  s->out_order = k;
  return 0;
}
void F(set_outflow_density)(void* h, double r) { ((S(solver)*)h)->outflow_rho = (R)r; }

/* Boussinesq forcing (BoussinesqGuo, Forcing.hpp:93-127): T per interior
 * node; NULL returns to the uniform force. */
void F(set_buoyancy)(void* h, const double* T, double gx, double gy, double gz, double rho0,
                     double beta, double T0) {
  S(solver)* s = (S(solver)*)h;
  s->buoyant = T != 0;
  s->bgx = (R)gx; s->bgy = (R)gy; s->bgz = (R)gz;
  s->brho0 = (R)rho0; s->bbeta = (R)beta; s->bT0 = (R)T0;
  if (T)
    for (int z = 0; z < s->nz; ++z)
      for (int y = 0; y < s->ny; ++y)
        for (int x = 0; x < s->nx; ++x)
          s->temp[S(idi)(s, x, y, z)] = (R)T[((size_t)z * s->ny + y) * s->nx + x];
  s->fx = s->ufx; s->fy = s->ufy; s->fz = s->ufz;
}
/* BoussinesqGuo::at(n): the force at node n (sets fx, fy, fz). */
static inline void S(force_at)(S(solver)* s, long long n) {
  if (!s->buoyant) return;
  const R b = s->brho0 * s->bbeta * (s->temp[n] - s->bT0);
  s->fx = s->ufx + s->bgx * b;
  s->fy = s->ufy + s->bgy * b;
  s->fz = s->ufz + s->bgz * b;
}

/* corner_density<P> (:664-712): closure density of every straight wall node,
 * then the corners extrapolated from two of them, at the parity the sweep
 * is about to read. */
static void S(corner_density)(S(solver)* s, int par) {
  static const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
  for (long long n = 0; n < s->n_padded; ++n) {
    if (s->flags[n] != 3) continue;
    const uint8_t code = s->bc_nrm[n];
    if (code == NRM_CORNER || code == 0) continue;
    R f[27], uw[3];
    int nrm[3];
    S(load_node)(s, par, n, f, S(unshift)(s));
    S(normal_of)(code, nrm);
    S(wall_vel)(s, n, uw);
    s->bc_rho[n] = (code == NRM_OUTXP || code == NRM_OUTEQ) ? s->wall_u0[n * 4 + 3]
                 : (code == NRM_OUTFREE) ? s->outflow_rho : S(bc_density)(s, f, nrm, uw);
  }
  for (long long n = 0; n < s->n_padded; ++n) {
    if (s->flags[n] != 3 || s->bc_nrm[n] != NRM_CORNER) continue;
    const int k = s->bc_ext[n];
    if (k == 0) { s->bc_rho[n] = (R)1; continue; }
    int px, py, pz;
    S(coords)(s, n, &px, &py, &pz);
    const int x = px - s->hx, y = py - s->hy, z = pz - s->hz;
    const int* e = d6[k - 1];
    const long long n1 = S(idi)(s, x + e[0], y + e[1], z + e[2]);
    const long long n2 = S(idi)(s, x + 2 * e[0], y + 2 * e[1], z + 2 * e[2]);
    s->bc_rho[n] = (R)2 * s->bc_rho[n1] - s->bc_rho[n2];
  }
}

/* Velocity of a node for the corner stencil (:965-986): a wall node's
 * imposed state velocity, else the moments of its populations. */
static void S(vel_at)(const S(solver)* s, int par, long long m, R* out) {
  if (s->flags[m] == 3) {
    for (int a = 0; a < 3; ++a) out[a] = s->wall_u0[m * 4 + a] * s->wall_scale;
    return;
  }
  long long nb[27];
  R g2[27];
  S(neighbours)(s, m, nb);
  S(load_all)(s, par, m, nb, g2);
  R sm = 0, mx = 0, my = 0, mz = 0;
  for (int i = 0; i < s->Q; ++i) {
    R v = g2[i];
    if (S(unshift)(s)) v += S(w)(s, i);
    sm += v;
    mx += v * (R)S(c)(s, i, 0);
    my += v * (R)S(c)(s, i, 1);
    mz += v * (R)S(c)(s, i, 2);
  }
  const R ir = (R)1 / sm;
  out[0] = mx * ir; out[1] = my * ir; out[2] = mz * ir;
}

/* The RegWall branch of run_step (:792-1021).  Returns 1 when the node is
 * finished (outflow codes that overwrite the node), 0 when it goes on to
 * collide like a fluid node. */
static int S(regwall)(S(solver)* s, int par, long long n, const long long* nb, R* f) {
  const int Q = s->Q;
  const int unsh = S(unshift)(s);
  if (unsh)
    for (int i = 0; i < Q; ++i) f[i] += S(w)(s, i);
  const uint8_t code = s->bc_nrm[n];
  int nrm[3];
  S(normal_of)(code, nrm);
  R uw[3];
  S(wall_vel)(s, n, uw);
  /* has_forcing<Collision> (Regularized.hpp:81-86) looks for a ForcingPolicy
   * member type, which of these operators only BGK declares (BGK.hpp:37):
   * the wall sees the force under BGK alone. */
  R Fv[3] = {0, 0, 0};
  if (s->forcing && s->op == 1) { Fv[0] = s->fx; Fv[1] = s->fy; Fv[2] = s->fz; }
  R ur[3] = {uw[0], uw[1], uw[2]};
  R rw;
  if (code == NRM_OUTFREE) {
    R g[27];
    S(load_node)(s, par, s->bc_don[n], g, unsh);
    R sm = 0;
    for (int i = 0; i < Q; ++i) sm += g[i];
    if (sm > (R)0) {
      const R sc = s->outflow_rho / sm;
      for (int i = 0; i < Q; ++i) f[i] = g[i] * sc;
    }
    if (unsh)
      for (int i = 0; i < Q; ++i) f[i] -= S(w)(s, i);
    S(store_all)(s, par, n, nb, f);
    return 1;
  } else if (code == NRM_OUTEQ) {
    const R rw2 = s->wall_u0[n * 4 + 3];
    int px, py, pz;
    S(coords)(s, n, &px, &py, &pz);
    R g[27];
    S(load_node)(s, par, S(idi)(s, px - s->hx - 1, py - s->hy, pz - s->hz), g, unsh);
    R sm = 0, mu[3] = {0, 0, 0};
    for (int i = 0; i < Q; ++i) {
      sm += g[i];
      for (int a = 0; a < 3; ++a) mu[a] += g[i] * (R)S(c)(s, i, a);
    }
    const R ir = (sm > (R)0) ? (R)1 / sm : (R)0;
    for (int a = 0; a < 3; ++a) mu[a] *= ir;
    for (int i = 0; i < Q; ++i) f[i] = S(bc_feq)(s, i, rw2, mu[0], mu[1], mu[2]);
    if (unsh)
      for (int i = 0; i < Q; ++i) f[i] -= S(w)(s, i);
    S(store_all)(s, par, n, nb, f);
    return 1;
  } else if (code == NRM_OUTXP) {
    rw = s->wall_u0[n * 4 + 3];
    R ut[3];
    S(up_vel)(s, par, n, 1, ut);
    if (s->out_order >= 2) {
      R v2[3];
      S(up_vel)(s, par, n, 2, v2);
      for (int a = 0; a < 3; ++a) ut[a] = (R)2 * ut[a] - v2[a];
    }
    const R un = S(bc_normal_velocity)(s, f, nrm, rw);
    R utn = 0;
    for (int a = 0; a < 3; ++a) utn += ut[a] * (R)nrm[a];
    for (int a = 0; a < 3; ++a) ur[a] = ut[a] + (un - utn) * (R)nrm[a];
  } else {
    rw = (code == NRM_CORNER) ? s->bc_rho[n] : S(bc_density)(s, f, nrm, ur);
  }
  if (s->fd_corners && s->op != 0 && code == NRM_CORNER) {
    int px, py, pz;
    S(coords)(s, n, &px, &py, &pz);
    const int ic[3] = {px - s->hx, py - s->hy, pz - s->hz};
    const int nn[3] = {s->nx, s->ny, s->nz};
    R grad[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < s->D; ++a) {
      if (nn[a] < 3) continue;
      int dir = 0;
      if (!s->per[a]) {
        if (ic[a] == 0) dir = 1;
        else if (ic[a] == nn[a] - 1) dir = -1;
      }
      R u1[3], u2[3];
      int c1[3] = {ic[0], ic[1], ic[2]}, c2[3] = {ic[0], ic[1], ic[2]};
      if (dir != 0) {
        c1[a] += dir; c2[a] += 2 * dir;
        S(vel_at)(s, par, S(idi)(s, c1[0], c1[1], c1[2]), u1);
        S(vel_at)(s, par, S(idi)(s, c2[0], c2[1], c2[2]), u2);
        for (int b = 0; b < s->D; ++b)
          grad[a][b] = (R)dir * ((R)(-1.5) * uw[b] + (R)2 * u1[b] - (R)0.5 * u2[b]);
      } else {
        c1[a] = (ic[a] + 1) % nn[a];
        c2[a] = (ic[a] - 1 + nn[a]) % nn[a];
        S(vel_at)(s, par, S(idi)(s, c1[0], c1[1], c1[2]), u1);
        S(vel_at)(s, par, S(idi)(s, c2[0], c2[1], c2[2]), u2);
        for (int b = 0; b < s->D; ++b) grad[a][b] = (R)0.5 * (u1[b] - u2[b]);
      }
    }
    R Pi[6];
    S(bc_stress_from_gradient)(rw, s->omega, grad, Pi);
    S(bc_apply_with_stress)(s, f, rw, ur, Pi);
  } else {
    S(bc_apply)(s, f, rw, ur, s->bc_unk[n], s->force_bc ? Fv : 0);
  }
  if (unsh)
    for (int i = 0; i < Q; ++i) f[i] -= S(w)(s, i);
  return 0;
}

/* seed_populations -> scatter<P> (:634-637, 1231-1241), sequential node order. */
static void S(scatter_fn)(S(solver)* s, const double* rho, const double* ux, const double* uy,
                          const double* uz, R rho0, R ux0, R uy0, R uz0, int field) {
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    S(neighbours)(s, n, nb);
    const int fluid = s->flags[n] == 0 || s->flags[n] == 3 || s->flags[n] == 5; /* :557, 575 */
    R r = rho0, a = ux0, b = uy0, c = uz0;
    if (field) {                                             /* initialize_field :568-579 */
      r = (R)1; a = b = c = (R)0;
      if (fluid) {
        int x, y, z;
        S(coords)(s, n, &x, &y, &z);
        const size_t k = ((size_t)(z - s->hz) * s->ny + (y - s->hy)) * s->nx + (x - s->hx);
        r = (R)rho[k]; a = (R)ux[k]; b = (R)uy[k]; c = (R)uz[k];
      }
    } else if (!fluid) {                                     /* initialize :553-561 */
      a = b = c = (R)0;
    }
    for (int i = 0; i < s->Q; ++i) S(scatter1)(s, par, n, nb, i, S(seed_value)(s, i, r, a, b, c));
  }
}
void F(initialize)(void* h, double rho, double ux, double uy, double uz) {
  S(solver)* s = (S(solver)*)h;
  s->t = 0;
  S(scatter_fn)(s, 0, 0, 0, 0, (R)rho, (R)ux, (R)uy, (R)uz, 0);
}
void F(initialize_field)(void* h, const double* rho, const double* ux, const double* uy,
                         const double* uz) {
  S(solver)* s = (S(solver)*)h;
  s->t = 0;
  S(scatter_fn)(s, rho, ux, uy, uz, 0, 0, 0, 0, 1);
}
/* step -> run_step<P, StoreMacro> (:582-591, 712-1038): fluid, SpecWall
 * (:745-757) and SpecNode (:791) branches. */
void F(step)(void* h, int nsteps, int store_macro) {
  S(solver)* s = (S(solver)*)h;
  for (int t = 0; t < nsteps; ++t) {
    const int par = (int)(s->t % 2);
    if (s->has_walls && s->has_corners) S(corner_density)(s, par);
    /* Regularised walls may read neighbour nodes inside the in-place sweep,
     * so with walls the sweep runs in index order, as the reference's
     * one-thread build runs it. */
#pragma omp parallel for schedule(static) if (!s->has_walls && !s->buoyant)
    for (long long n = 0; n < s->n_padded; ++n) {
      const uint8_t fl = s->flags[n];
      if (fl != 0 && fl != 3 && fl != 4 && fl != 5) continue; /* Excluded / Solid skipped */
      S(force_at)(s, n);
      long long nb[27];
      R f[27];
      S(neighbours)(s, n, nb);
      S(load_all)(s, par, n, nb, f);
      if (fl == 3 && S(regwall)(s, par, n, nb, f)) continue;
      if (fl == 4) {                                         /* ghost mirror, no collision */
        const int ax = S(mirror_axis)(s->spec_nrm[n]);
        R g[27];
        for (int i = 0; i < s->Q; ++i) g[i] = f[S(mir)(s, ax, i)];
        S(store_all)(s, par, n, nb, g);
        continue;
      }
      if (fl == 5) S(mirror_faces)(s, f, s->spec_faces[n]);
      const S(macro_t) m = S(macroscopic)(s, f);
      if (s->op == 1) S(collide_bgk)(s, f, m);
      else if (s->op == 2) S(collide_trt)(s, f, m);
      else if (s->op >= 3) S(collide_moment)(s, f, m);
      S(store_all)(s, par, n, nb, f);
      if (store_macro) {
        s->rho[n] = S(density)(s, m.dens);
        s->ux[n] = m.ux; s->uy[n] = m.uy; s->uz[n] = m.uz;
      }
    }
    ++s->t;
  }
}
static void S(copy_interior)(const S(solver)* s, double* rho, double* ux, double* uy, double* uz) {
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = S(idp)(s, x + s->hx, y + s->hy, z + s->hz);
        const size_t k = ((size_t)z * s->ny + y) * s->nx + x;
        rho[k] = (double)s->rho[n]; ux[k] = (double)s->ux[n];
        uy[k] = (double)s->uy[n]; uz[k] = (double)s->uz[n];
      }
}
/* compute_macroscopic -> macro_kernel<P> (:597-599, 1041-1179), fluid branch. */
void F(macro)(void* h, double* rho, double* ux, double* uy, double* uz) {
  S(solver)* s = (S(solver)*)h;
  const int par = (int)(s->t % 2);
  for (long long n = 0; n < s->n_padded; ++n) {
    const uint8_t fl = s->flags[n];
    if (fl != 0 && fl != 3 && fl != 5) { s->rho[n] = s->ux[n] = s->uy[n] = s->uz[n] = (R)0; continue; }
    S(force_at)(s, n);
    long long nb[27];
    R f[27];
    S(neighbours)(s, n, nb);
    S(load_all)(s, par, n, nb, f);
    if (fl == 3) {                                           /* :1085-1188, reported state */
      if (S(unshift)(s))
        for (int i = 0; i < s->Q; ++i) f[i] += S(w)(s, i);
      const uint8_t code = s->bc_nrm[n];
      int nrm[3];
      S(normal_of)(code, nrm);
      R uw[3];
      S(wall_vel)(s, n, uw);
      R rw;
      if (code == NRM_OUTFREE) {
        rw = s->outflow_rho;
        int onr[3];
        S(normal_of)(s->bc_onrm[n], onr);
        R g[27];
        S(load_node)(s, par, s->bc_don[n], g, S(unshift)(s));
        R sm = 0, m4[3] = {0, 0, 0};
        for (int i = 0; i < s->Q; ++i) {
          sm += g[i];
          for (int a = 0; a < 3; ++a) m4[a] += g[i] * (R)S(c)(s, i, a);
        }
        const R ir = (sm > (R)0) ? (R)1 / sm : (R)0;
        const R un = S(bc_normal_velocity)(s, f, onr, rw);
        R utn = 0;
        for (int a = 0; a < 3; ++a) utn += m4[a] * ir * (R)onr[a];
        for (int a = 0; a < 3; ++a) uw[a] = m4[a] * ir + (un - utn) * (R)onr[a];
      } else if (code == NRM_OUTEQ) {
        rw = s->wall_u0[n * 4 + 3];
        int px, py, pz;
        S(coords)(s, n, &px, &py, &pz);
        R g[27];
        S(load_node)(s, par, S(idi)(s, px - s->hx - 1, py - s->hy, pz - s->hz), g, S(unshift)(s));
        R sm = 0, mu[3] = {0, 0, 0};
        for (int i = 0; i < s->Q; ++i) {
          sm += g[i];
          for (int a = 0; a < 3; ++a) mu[a] += g[i] * (R)S(c)(s, i, a);
        }
        const R ir = (sm > (R)0) ? (R)1 / sm : (R)0;
        for (int a = 0; a < 3; ++a) uw[a] = mu[a] * ir;
      } else if (code == NRM_OUTXP) {
        rw = s->wall_u0[n * 4 + 3];
        R ut[3];
        S(up_vel)(s, par, n, 1, ut);
        if (s->out_order >= 2) {
          R v2[3];
          S(up_vel)(s, par, n, 2, v2);
          for (int a = 0; a < 3; ++a) ut[a] = (R)2 * ut[a] - v2[a];
        }
        const R un = S(bc_normal_velocity)(s, f, nrm, rw);
        R utn = 0;
        for (int a = 0; a < 3; ++a) utn += ut[a] * (R)nrm[a];
        for (int a = 0; a < 3; ++a) uw[a] = ut[a] + (un - utn) * (R)nrm[a];
      } else {
        rw = (code == NRM_CORNER) ? s->bc_rho[n] : S(bc_density)(s, f, nrm, uw);
      }
      s->rho[n] = rw;
      s->ux[n] = uw[0]; s->uy[n] = uw[1]; s->uz[n] = uw[2];
      continue;
    }
    if (fl == 5) {                                           /* :1061-1080, raw moments */
      S(mirror_faces)(s, f, s->spec_faces[n]);
      if (s->shifted && s->op != 0)                          /* no-collision runs raw */
        for (int i = 0; i < s->Q; ++i) f[i] += S(w)(s, i);
      R sm = 0, mx = 0, my = 0, mz = 0;
      for (int i = 0; i < s->Q; ++i) {
        sm += f[i];
        mx += f[i] * (R)S(c)(s, i, 0);
        my += f[i] * (R)S(c)(s, i, 1);
        mz += f[i] * (R)S(c)(s, i, 2);
      }
      const R ir = (R)1 / sm;
      s->rho[n] = sm; s->ux[n] = mx * ir; s->uy[n] = my * ir; s->uz[n] = mz * ir;
      continue;
    }
    const S(macro_t) m = S(macroscopic)(s, f);
    s->rho[n] = S(density)(s, m.dens);
    s->ux[n] = m.ux; s->uy[n] = m.uy; s->uz[n] = m.uz;
  }
  S(copy_interior)(s, rho, ux, uy, uz);
}
void F(stored_macro)(void* h, double* rho, double* ux, double* uy, double* uz) {
  S(copy_interior)((S(solver)*)h, rho, ux, uy, uz);
}
/* total_mass / total_momentum -> reduce<P>(axis) (:601-606, 1205-1229). */
static double S(reduce)(S(solver)* s, int axis) {
  const int par = (int)(s->t % 2);
  R sum = 0;
  for (long long n = 0; n < s->n_padded; ++n) {
    if (s->flags[n] != 0 && s->flags[n] != 3 && s->flags[n] != 5) continue;
    S(force_at)(s, n);
    long long nb[27];
    R f[27];
    S(neighbours)(s, n, nb);
    for (int i = 0; i < s->Q; ++i) f[i] = S(load1)(s, par, n, nb, i);
    if (s->flags[n] == 5) S(mirror_faces)(s, f, s->spec_faces[n]);   /* :1221-1222 */
    const S(macro_t) m = S(macroscopic)(s, f);
    const R r = S(density)(s, m.dens);
    sum += (axis < 0) ? r : r * (axis == 0 ? m.ux : (axis == 1 ? m.uy : m.uz));
  }
  return (double)sum;
}
double F(total_mass)(void* h) { return S(reduce)((S(solver)*)h, -1); }
double F(total_momentum)(void* h, int a) { return S(reduce)((S(solver)*)h, a); }
/* gather_populations -> gather<P> (:620-624, 1243-1253). */
void F(gather)(void* h, double* out) {
  S(solver)* s = (S(solver)*)h;
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    S(neighbours)(s, n, nb);
    for (int i = 0; i < s->Q; ++i) out[n * s->Q + i] = (double)S(load1)(s, par, n, nb, i);
  }
}
void F(seed)(void* h, const double* in) {
  S(solver)* s = (S(solver)*)h;
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    S(neighbours)(s, n, nb);
    for (int i = 0; i < s->Q; ++i) S(scatter1)(s, par, n, nb, i, (R)in[n * s->Q + i]);
  }
}
/* Sum of every stored slot (EsotericPull::storage, EsotericPull.hpp:119-123). */
double F(slot_sum)(void* h) {
  S(solver)* s = (S(solver)*)h;
  double acc = 0;
  for (long long k = 0; k < s->n_padded * s->Q; ++k) acc += (double)s->f[k];
  return acc;
}
long long F(n_padded)(void* h) { return ((S(solver)*)h)->n_padded; }
long long F(timestep)(void* h) { return ((S(solver)*)h)->t; }

#undef MI3
#undef MI2
#undef F
#undef S
#undef CAT
#undef CAT_
