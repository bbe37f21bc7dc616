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
  R *rho, *ux, *uy, *uz; /* stored macroscopic fields (StoreMacro) */
} S(solver);

/* Storage rounding (narrow population storage emulated in R arithmetic). */
static inline R S(q)(const S(solver)* s, R v) {
  if (s->quant == 1) return (R)(_Float16)v;
  if (s->quant == 2) return (R)lbmo_bf16_round((float)v);
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
static inline R S(phi)(const S(solver)* s, int i, R ux, R uy, R uz) {
  const R cx = (R)S(c)(s, i, 0), cy = (R)S(c)(s, i, 1), cz = (R)S(c)(s, i, 2);
  if (s->eq == 0) {                                          /* SecondOrderPhi :49-60 */
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
  s->f = (R*)calloc((size_t)s->n_padded * s->Q, sizeof(R));
  s->flags = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->spec_nrm = (uint8_t*)calloc((size_t)s->n_padded, 1);
  s->spec_faces = (uint8_t*)calloc((size_t)s->n_padded, 1);
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
  free(s->f); free(s->flags); free(s->spec_nrm); free(s->spec_faces); free(s->rho); free(s->ux); free(s->uy); free(s->uz);
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
/* seed_populations -> scatter<P> (:634-637, 1231-1241), sequential node order. */
static void S(scatter_fn)(S(solver)* s, const double* rho, const double* ux, const double* uy,
                          const double* uz, R rho0, R ux0, R uy0, R uz0, int field) {
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    S(neighbours)(s, n, nb);
    const int fluid = s->flags[n] == 0 || s->flags[n] == 5;  /* SpecNode seeds as fluid */
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
#pragma omp parallel for schedule(static)
    for (long long n = 0; n < s->n_padded; ++n) {
      const uint8_t fl = s->flags[n];
      if (fl != 0 && fl != 4 && fl != 5) continue;           /* Excluded / Solid skipped */
      long long nb[27];
      R f[27];
      S(neighbours)(s, n, nb);
      S(load_all)(s, par, n, nb, f);
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
    if (fl != 0 && fl != 5) { s->rho[n] = s->ux[n] = s->uy[n] = s->uz[n] = (R)0; continue; }
    long long nb[27];
    R f[27];
    S(neighbours)(s, n, nb);
    S(load_all)(s, par, n, nb, f);
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
    if (s->flags[n] != 0 && s->flags[n] != 5) continue;
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
