/*
 * Body of the CPU oracle for the scalar (advection-diffusion) lattice,
 * included once per arithmetic type by lbm_oracle.c with R and P defined.
 * TEST INFRASTRUCTURE: see lbm_oracle.h.
 *
 * Restates src/solver/ScalarSolver.hpp (D2Q5 / D3Q7 on Esoteric Pull) with
 * the operators of src/collision/ScalarBGK.hpp, ScalarTRT.hpp and
 * ScalarRegularised.hpp, the on-node moment wall of
 * src/boundary/MomentDirichlet.hpp and the scalar mirror of
 * src/boundary/Specular.hpp, in the reference's operation order.
 */
#define SC_(a, b) a##b
#define SC(a, b) SC_(a, b)
#define SF(name) SC(P, SC(s, name))
#define SS(name) SC(SC(P, ss_), name)

typedef struct {
  int lattice, Q, D, op;
  int nx, ny, nz, hx, hy, hz, sx, sy, sz, per[3];
  long long n_padded, t;
  R omega, T_ref, Lambda;
  R* g;             /* populations, node-major g[n*Q + q] */
  uint8_t* flags;   /* ScalarCell per padded node */
  uint8_t* spec;    /* face mask per padded node */
  uint32_t* unk;    /* moment-wall unknown directions */
  long long* don;   /* outflow donor */
  R *wall, *field, *omega_of, *ux, *uy, *uz;
  int has_outflow, have_u, have_omega;
} SS(solver);

/* ---- D2Q5 / D3Q7: src/lattice/Lattices.hpp:51-70, 100-121 ---- */
/* (and the fluid lattices D2Q9 / D3Q27, which ScalarBGK also runs on) */
static inline int SS(c)(const SS(solver)* s, int i, int a) {
  switch (s->Q) {
    case 5: return a == 2 ? 0 : D2Q5_C[a][i];
    case 7: return D3Q7_C[a][i];
    case 9: return a == 0 ? D2Q9_CX[i] : (a == 1 ? D2Q9_CY[i] : 0);
    default: return a == 0 ? D3Q27_CX[i] : (a == 1 ? D3Q27_CY[i] : D3Q27_CZ[i]);
  }
}
static inline R SS(w)(const SS(solver)* s, int i) {
  switch (s->Q) {
    case 5: return (R)D2Q5_W[i] / (R)6;
    case 7: return (R)D3Q7_W[i] / (R)8;
    case 9: return (R)D2Q9_W[i] / (R)36;
    default: return (R)D3Q27_W[i] / (R)216;
  }
}
static inline R SS(cs2)(const SS(solver)* s) { return s->Q == 7 ? (R)1 / (R)4 : (R)1 / (R)3; }
static inline R SS(ics2)(const SS(solver)* s) { return s->Q == 7 ? (R)4 / (R)1 : (R)3 / (R)1; }
static inline int SS(mir)(const SS(solver)* s, int a, int i) {
  switch (s->Q) {
    case 5: return D2Q5_MIR[a][i];
    case 7: return D3Q7_MIR[a][i];
    case 9: return D2Q9_MIR[a][i];
    default: return D3Q27_MIR[a][i];
  }
}

static inline long long SS(idp)(const SS(solver)* s, int x, int y, int z) {
  return ((long long)z * s->sy + y) * s->sx + x;
}
static inline long long SS(idi)(const SS(solver)* s, int x, int y, int z) {
  return SS(idp)(s, x + s->hx, y + s->hy, z + s->hz);
}
static inline void SS(coords)(const SS(solver)* s, long long n, int* x, int* y, int* z) {
  *x = (int)(n % s->sx);
  *y = (int)((n / s->sx) % s->sy);
  *z = (int)(n / ((long long)s->sx * s->sy));
}
static inline int SS(shift)(int v, int h, int n, int sz, int per) {
  if (per) {
    if (v < h) return v + n;
    if (v >= h + n) return v - n;
    return v;
  }
  if (v < 0) return 0;
  if (v >= sz) return sz - 1;
  return v;
}
static void SS(neighbours)(const SS(solver)* s, long long n, long long nb[27]) {
  int x, y, z;
  SS(coords)(s, n, &x, &y, &z);
  for (int i = 1; i < s->Q; i += 2)
    nb[i] = SS(idp)(s, SS(shift)(x + SS(c)(s, i, 0), s->hx, s->nx, s->sx, s->per[0]),
                    SS(shift)(y + SS(c)(s, i, 1), s->hy, s->ny, s->sy, s->per[1]),
                    SS(shift)(z + SS(c)(s, i, 2), s->hz, s->nz, s->sz, s->per[2]));
}
#define SA(node, q) s->g[(node) * s->Q + (q)]
static void SS(load_all)(const SS(solver)* s, int par, long long n, const long long* nb, R* g) {
  g[0] = SA(n, 0);
  for (int i = 1; i < s->Q; i += 2) {
    if (par == 0) { g[i] = SA(n, i);     g[i + 1] = SA(nb[i], i + 1); }
    else          { g[i] = SA(n, i + 1); g[i + 1] = SA(nb[i], i); }
  }
}
static void SS(store_all)(SS(solver)* s, int par, long long n, const long long* nb, const R* g) {
  SA(n, 0) = g[0];
  for (int i = 1; i < s->Q; i += 2) {
    if (par == 0) { SA(nb[i], i + 1) = g[i]; SA(n, i) = g[i + 1]; }
    else          { SA(nb[i], i) = g[i];     SA(n, i + 1) = g[i + 1]; }
  }
}
static inline R* SS(slot)(SS(solver)* s, int par, long long n, const long long* nb, int i) {
  if (i == 0) return &SA(n, 0);
  if (par == 0) return (i & 1) ? &SA(n, i) : &SA(nb[i - 1], i);
  return (i & 1) ? &SA(n, i + 1) : &SA(nb[i - 1], i - 1);
}
#undef SA

/* ---- operators: ScalarBGK.hpp:38-70, ScalarTRT.hpp:30-60, ScalarRegularised.hpp:33-50 ---- */
static inline R SS(deviation)(const SS(solver)* s, const R* h) {
  R t = 0;
  for (int i = 0; i < s->Q; ++i) t += h[i];
  return t;
}
static inline R SS(eq)(const SS(solver)* s, int i, R dT, R ux, R uy, R uz) {
  const R ics2 = SS(ics2)(s);
  const R cu = (R)SS(c)(s, i, 0) * ux + (R)SS(c)(s, i, 1) * uy + (R)SS(c)(s, i, 2) * uz;
  return SS(w)(s, i) * (dT + (s->T_ref + dT) * ics2 * cu);
}
static inline R SS(omega_at)(const SS(solver)* s, long long n) {
  return s->have_omega ? s->omega_of[n] : s->omega;
}
static void SS(collide)(const SS(solver)* s, R* h, R dT, R ux, R uy, R uz, R w) {
  if (s->op == 1) {
    for (int i = 0; i < s->Q; ++i) h[i] += w * (SS(eq)(s, i, dT, ux, uy, uz) - h[i]);
    return;
  }
  const R cs2v = SS(cs2)(s);
  const R T = s->T_ref + dT;
  const R u[3] = {ux, uy, uz};
  const R d = cs2v * dT;
  if (s->op == 2) {
    const R tm = (R)1 / w - (R)0.5;
    const R wp = tm > (R)0 ? (R)1 / (s->Lambda / tm + (R)0.5) : (R)0;
    R msum = 0;
    for (int a = 0; a < s->D; ++a) {
      const R j = h[2 * a + 1] - h[2 * a + 2];
      const R m = h[2 * a + 1] + h[2 * a + 2];
      const R p = j + w * (T * u[a] - j);
      const R g = m + wp * (d - m);
      h[2 * a + 1] = (R)0.5 * (g + p);
      h[2 * a + 2] = (R)0.5 * (g - p);
      msum += g;
    }
    h[0] = dT - msum;
    return;
  }
  for (int a = 0; a < s->D; ++a) {
    const R j = h[2 * a + 1] - h[2 * a + 2];
    const R p = j + w * (T * u[a] - j);
    h[2 * a + 1] = (R)0.5 * (d + p);
    h[2 * a + 2] = (R)0.5 * (d - p);
  }
  h[0] = dT - (R)s->D * d;
}
/* impose_moment (MomentDirichlet.hpp): the unknowns share the deficit by weight. */
static void SS(impose_moment)(const SS(solver)* s, R* g, R target, uint32_t unknown) {
  R known = 0, wsum = 0;
  for (int i = 0; i < s->Q; ++i) {
    if (unknown & (1u << i)) wsum += SS(w)(s, i);
    else known += g[i];
  }
  if (!(wsum > (R)0)) return;
  const R deficit = target - known;
  for (int i = 0; i < s->Q; ++i)
    if (unknown & (1u << i)) g[i] = deficit * SS(w)(s, i) / wsum;
}
static void SS(mirror_faces)(const SS(solver)* s, R* f, uint8_t faces) {
  R h[27];
  for (int i = 0; i < s->Q; ++i) h[i] = f[i];
  for (int i = 0; i < s->Q; ++i) {
    int j = i, unknown = 0;
    for (int a = 0; a < 3; ++a) {
      const int sg = (faces & (1u << (2 * a))) ? 1 : ((faces & (1u << (2 * a + 1))) ? -1 : 0);
      if (sg != 0 && SS(c)(s, i, a) * sg < 0) { j = SS(mir)(s, a, j); unknown = 1; }
    }
    if (unknown) f[i] = h[j];
  }
}

/* ---- ScalarSolver (src/solver/ScalarSolver.hpp) ---- */
void* SF(create)(int lattice, int op, int nx, int ny, int nz, int px, int py, int pz, double omega,
                 double T_ref, double Lambda) {
  if ((lattice != 5 && lattice != 7 && lattice != 9 && lattice != 27) || op < 1 || op > 3) return 0;
  if ((lattice == 5 || lattice == 9) && nz != 1) return 0;
  if ((lattice == 9 || lattice == 27) && op != 1) return 0;   /* TRT / regularised: axis-pair lattices */
  SS(solver)* s = (SS(solver)*)calloc(1, sizeof(SS(solver)));
  s->lattice = lattice; s->Q = lattice; s->D = (lattice == 5 || lattice == 9) ? 2 : 3; s->op = op;
  s->nx = nx; s->ny = ny; s->nz = nz;
  s->per[0] = px != 0; s->per[1] = py != 0; s->per[2] = pz != 0;
  s->hx = (nx <= 1 || s->per[0]) ? 0 : 1;
  s->hy = (ny <= 1 || s->per[1]) ? 0 : 1;
  s->hz = (nz <= 1 || s->per[2]) ? 0 : 1;
  s->sx = nx + 2 * s->hx; s->sy = ny + 2 * s->hy; s->sz = nz + 2 * s->hz;
  s->n_padded = (long long)s->sx * s->sy * s->sz;
  s->omega = (R)omega; s->T_ref = (R)T_ref; s->Lambda = (R)Lambda;
  const size_t np = (size_t)s->n_padded;
  s->g = (R*)calloc(np * s->Q, sizeof(R));
  s->flags = (uint8_t*)calloc(np, 1);
  s->spec = (uint8_t*)calloc(np, 1);
  s->unk = (uint32_t*)calloc(np, sizeof(uint32_t));
  s->don = (long long*)calloc(np, sizeof(long long));
  s->wall = (R*)calloc(np, sizeof(R));
  s->field = (R*)calloc(np, sizeof(R));
  s->omega_of = (R*)calloc(np, sizeof(R));
  s->ux = (R*)calloc(np, sizeof(R));
  s->uy = (R*)calloc(np, sizeof(R));
  s->uz = (R*)calloc(np, sizeof(R));
  for (long long n = 0; n < s->n_padded; ++n) {               /* ctor :81-86 */
    int x, y, z;
    SS(coords)(s, n, &x, &y, &z);
    const int in = x >= s->hx && x < s->hx + nx && y >= s->hy && y < s->hy + ny &&
                   z >= s->hz && z < s->hz + nz;
    s->flags[n] = in ? SB_BULK : SB_EXCLUDED;
    s->don[n] = n;
  }
  return s;
}
void SF(destroy)(void* h) {
  SS(solver)* s = (SS(solver)*)h;
  if (!s) return;
  free(s->g); free(s->flags); free(s->spec); free(s->unk); free(s->don); free(s->wall);
  free(s->field); free(s->omega_of); free(s->ux); free(s->uy); free(s->uz);
  free(s);
}
void SF(set_geometry)(void* h, const uint8_t* cells) {             /* :92-99 */
  SS(solver)* s = (SS(solver)*)h;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x)
        s->flags[SS(idi)(s, x, y, z)] = cells[((size_t)z * s->ny + y) * s->nx + x];
}
void SF(set_wall_values)(void* h, const double* tw) {              /* :101-108 */
  SS(solver)* s = (SS(solver)*)h;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x)
        s->wall[SS(idi)(s, x, y, z)] = (R)tw[((size_t)z * s->ny + y) * s->nx + x];
}
int SF(set_specular_walls)(void* h, const uint8_t* codes) {        /* :113-132 */
  SS(solver)* s = (SS(solver)*)h;
  const size_t ni = (size_t)s->nx * s->ny * s->nz;
  for (size_t k = 0; k < ni; ++k)
    if (codes[k] > 6) return -1;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const uint8_t c = codes[((size_t)z * s->ny + y) * s->nx + x];
        if (!c) continue;
        s->spec[SS(idi)(s, x, y, z)] = (uint8_t)(1u << (c - 1));   /* faces_of_normal */
      }
  return 0;
}
int SF(set_specular_nodes)(void* h, const uint8_t* masks) {        /* :140-164 */
  SS(solver)* s = (SS(solver)*)h;
  const size_t ni = (size_t)s->nx * s->ny * s->nz;
  for (size_t k = 0; k < ni; ++k) {
    const unsigned m = masks[k];
    if (m > 0x3F) return -1;
    for (int a = 0; a < 3; ++a)
      if ((m & (1u << (2 * a))) && (m & (1u << (2 * a + 1)))) return -1;
  }
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const uint8_t m = masks[((size_t)z * s->ny + y) * s->nx + x];
        if (m) s->spec[SS(idi)(s, x, y, z)] = m;
      }
  return 0;
}
/* omega_of (ScalarBGK.hpp: per-node rate), interior array; NULL clears it. */
void SF(set_omega_field)(void* h, const double* om) {
  SS(solver)* s = (SS(solver)*)h;
  s->have_omega = om != 0;
  if (!om) return;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x)
        s->omega_of[SS(idi)(s, x, y, z)] = (R)om[((size_t)z * s->ny + y) * s->nx + x];
}
/* set_velocity (:166-168): the advecting velocity per interior node; NULL clears it. */
void SF(set_velocity)(void* h, const double* ux, const double* uy, const double* uz) {
  SS(solver)* s = (SS(solver)*)h;
  s->have_u = ux != 0;
  if (!ux) return;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const size_t k = ((size_t)z * s->ny + y) * s->nx + x;
        const long long n = SS(idi)(s, x, y, z);
        s->ux[n] = (R)ux[k]; s->uy[n] = (R)uy[k]; s->uz[n] = (R)uz[k];
      }
}
/* finalize_geometry + build_donors (:223-296). */
void SF(finalize_geometry)(void* h) {
  SS(solver)* s = (SS(solver)*)h;
  const int nn[3] = {s->nx, s->ny, s->nz};
  memset(s->unk, 0, (size_t)s->n_padded * sizeof(uint32_t));
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = SS(idi)(s, x, y, z);
        if (s->flags[n] != SB_MOMENT) continue;
        uint32_t m = 0;
        for (int i = 0; i < s->Q; ++i) {
          int src[3] = {x - SS(c)(s, i, 0), y - SS(c)(s, i, 1), z - SS(c)(s, i, 2)};
          int outside = 0;
          for (int a = 0; a < 3; ++a) {
            if (s->per[a]) src[a] = (src[a] + nn[a]) % nn[a];
            else if (src[a] < 0 || src[a] >= nn[a]) outside = 1;
          }
          if (!outside && s->flags[SS(idi)(s, src[0], src[1], src[2])] == SB_EXCLUDED) outside = 1;
          if (outside) m |= 1u << i;
        }
        s->unk[n] = m;
      }
  /* donors */
  static const int d6[6][3] = {{-1,0,0},{1,0,0},{0,-1,0},{0,1,0},{0,0,-1},{0,0,1}};
  for (long long n = 0; n < s->n_padded; ++n) s->don[n] = n;
  int nout = 0;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = SS(idi)(s, x, y, z);
        if (s->flags[n] != SB_OUTFLOW) continue;
        ++nout;
        int ix = 0, iy = 0, iz = 0;
        for (int k = 0; k < 6; ++k) {
          int q[3] = {x + d6[k][0], y + d6[k][1], z + d6[k][2]};
          int outside = 0;
          for (int a = 0; a < 3; ++a) {
            if (s->per[a]) { if (q[a] < 0) q[a] += nn[a]; else if (q[a] >= nn[a]) q[a] -= nn[a]; }
            if (q[a] < 0 || q[a] >= nn[a]) outside = 1;
          }
          const uint8_t f = outside ? SB_EXCLUDED : s->flags[SS(idi)(s, q[0], q[1], q[2])];
          if (f == SB_EXCLUDED) { ix -= d6[k][0]; iy -= d6[k][1]; iz -= d6[k][2]; }
        }
        long long best = n;
        #define SFLAG_AT(X, Y, Z, OUT)                                                       \
          do {                                                                              \
            int q_[3] = {(X), (Y), (Z)}, o_ = 0;                                            \
            for (int a_ = 0; a_ < 3; ++a_) {                                                \
              if (s->per[a_]) { if (q_[a_] < 0) q_[a_] += nn[a_]; else if (q_[a_] >= nn[a_]) q_[a_] -= nn[a_]; } \
              if (q_[a_] < 0 || q_[a_] >= nn[a_]) o_ = 1;                                   \
            }                                                                               \
            (OUT) = o_ ? SB_EXCLUDED : s->flags[SS(idi)(s, q_[0], q_[1], q_[2])];          \
          } while (0)
        if (ix || iy || iz) {
          uint8_t f;
          SFLAG_AT(x + ix, y + iy, z + iz, f);
          if (f == SB_BULK) best = SS(idi)(s, x + ix, y + iy, z + iz);
        }
        if (best == n)
          for (int k = 0; k < 6; ++k) {
            uint8_t f;
            SFLAG_AT(x + d6[k][0], y + d6[k][1], z + d6[k][2], f);
            if (f == SB_BULK) { best = SS(idi)(s, x + d6[k][0], y + d6[k][1], z + d6[k][2]); break; }
          }
        #undef SFLAG_AT
        s->don[n] = best;
      }
  s->has_outflow = nout > 0;
}
/* initialize_field (:175-190): T per PADDED node (Dirichlet nodes take their wall value). */
void SF(initialize_field)(void* h, const double* T) {
  SS(solver)* s = (SS(solver)*)h;
  s->t = 0;
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    SS(neighbours)(s, n, nb);
    const R Tn = (s->flags[n] == SB_DIRICHLET) ? s->wall[n] : (R)T[n];
    s->field[n] = Tn;
    for (int i = 0; i < s->Q; ++i) *SS(slot)(s, 0, n, nb, i) = SS(eq)(s, i, Tn - s->T_ref, 0, 0, 0);
  }
}
void SF(initialize)(void* h, double T0) {
  SS(solver)* s = (SS(solver)*)h;
  double* T = (double*)malloc((size_t)s->n_padded * sizeof(double));
  for (long long n = 0; n < s->n_padded; ++n) T[n] = T0;
  SF(initialize_field)(h, T);
  free(T);
}
/* run_step<P> (:302-372) then outflow_kernel<P> (:393-419). */
void SF(step)(void* h, int nsteps) {
  SS(solver)* s = (SS(solver)*)h;
  for (int t = 0; t < nsteps; ++t) {
    const int par = (int)(s->t % 2);
#pragma omp parallel for schedule(static)
    for (long long n = 0; n < s->n_padded; ++n) {
      const uint8_t flag = s->flags[n];
      if (flag == SB_EXCLUDED || flag == SB_OUTFLOW || flag == SB_ADIABATIC) continue;
      long long nb[27];
      R g[27];
      SS(neighbours)(s, n, nb);
      SS(load_all)(s, par, n, nb, g);
      const R vx = s->have_u ? s->ux[n] : (R)0;
      const R vy = s->have_u ? s->uy[n] : (R)0;
      const R vz = s->have_u ? s->uz[n] : (R)0;
      if (flag == SB_MOMENT) {
        SS(impose_moment)(s, g, s->wall[n] - s->T_ref, s->unk[n]);
        const R dTm = SS(deviation)(s, g);
        SS(collide)(s, g, dTm, vx, vy, vz, SS(omega_at)(s, n));
        s->field[n] = s->T_ref + dTm;
        SS(store_all)(s, par, n, nb, g);
        continue;
      }
      if (flag == SB_DIRICHLET) {
        const R Tw = s->wall[n] - s->T_ref;
        R o[27];
        o[0] = -g[0] + (R)2 * SS(w)(s, 0) * Tw;
        for (int i = 1; i < s->Q; i += 2) {
          o[i] = -g[i + 1] + (R)2 * SS(w)(s, i) * Tw;
          o[i + 1] = -g[i] + (R)2 * SS(w)(s, i + 1) * Tw;
        }
        SS(store_all)(s, par, n, nb, o);
        continue;
      }
      if (flag == SB_SPECULAR) SS(mirror_faces)(s, g, s->spec[n]);
      const R dT = SS(deviation)(s, g);
      SS(collide)(s, g, dT, vx, vy, vz, SS(omega_at)(s, n));
      s->field[n] = s->T_ref + dT;
      SS(store_all)(s, par, n, nb, g);
    }
    if (s->has_outflow)
      for (long long n = 0; n < s->n_padded; ++n) {
        if (s->flags[n] != SB_OUTFLOW) continue;
        const long long src = s->don[n];
        if (src == n) continue;
        long long nb[27];
        SS(neighbours)(s, n, nb);
        const R dT = s->field[src] - s->T_ref;
        const R vx = s->have_u ? s->ux[n] : (R)0;
        const R vy = s->have_u ? s->uy[n] : (R)0;
        const R vz = s->have_u ? s->uz[n] : (R)0;
        R o[27];
        for (int i = 0; i < s->Q; ++i) o[i] = SS(eq)(s, i, dT, vx, vy, vz);
        SS(store_all)(s, par, n, nb, o);
        s->field[n] = s->T_ref + dT;
      }
    ++s->t;
  }
}
/* add_source (:198-200, 421-437): per interior node, on Bulk and Specular nodes. */
void SF(add_source)(void* h, const double* dC) {
  SS(solver)* s = (SS(solver)*)h;
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x) {
        const long long n = SS(idi)(s, x, y, z);
        const uint8_t f = s->flags[n];
        if (f != SB_BULK && f != SB_SPECULAR) continue;
        const R d = (R)dC[((size_t)z * s->ny + y) * s->nx + x];
        if (d == (R)0) continue;
        SS(neighbours)(s, n, nb);
        for (int i = 0; i < s->Q; ++i) {
          R* p = SS(slot)(s, par, n, nb, i);
          *p = *p + SS(w)(s, i) * d;
        }
      }
}
/* field_kernel (:375-391): compute_field. */
void SF(compute_field)(void* h) {
  SS(solver)* s = (SS(solver)*)h;
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    const uint8_t flag = s->flags[n];
    if (flag == SB_EXCLUDED) { s->field[n] = 0; continue; }
    if (flag == SB_DIRICHLET || flag == SB_MOMENT) { s->field[n] = s->wall[n]; continue; }
    if (flag == SB_ADIABATIC) { s->field[n] = 0; continue; }
    if (flag == SB_OUTFLOW) continue;
    R g[27];
    SS(neighbours)(s, n, nb);
    SS(load_all)(s, par, n, nb, g);
    if (flag == SB_SPECULAR) SS(mirror_faces)(s, g, s->spec[n]);
    s->field[n] = s->T_ref + SS(deviation)(s, g);
  }
}
/* temperature(): the field per interior node, as it stands. */
void SF(field)(void* h, double* T) {
  SS(solver)* s = (SS(solver)*)h;
  for (int z = 0; z < s->nz; ++z)
    for (int y = 0; y < s->ny; ++y)
      for (int x = 0; x < s->nx; ++x)
        T[((size_t)z * s->ny + y) * s->nx + x] = (double)s->field[SS(idi)(s, x, y, z)];
}
/* total_population (:209-218). */
double SF(total)(void* h) {
  SS(solver)* s = (SS(solver)*)h;
  R acc = 0;
  for (long long k = 0; k < s->n_padded * s->Q; ++k) acc += s->g[k];
  return (double)acc;
}
/* logical populations per padded node (gather / seed for tests). */
void SF(gather)(void* h, double* out) {
  SS(solver)* s = (SS(solver)*)h;
  const int par = (int)(s->t % 2);
  long long nb[27];
  for (long long n = 0; n < s->n_padded; ++n) {
    SS(neighbours)(s, n, nb);
    for (int i = 0; i < s->Q; ++i) out[n * s->Q + i] = (double)*SS(slot)(s, par, n, nb, i);
  }
}
long long SF(n_padded)(void* h) { return ((SS(solver)*)h)->n_padded; }
long long SF(timestep)(void* h) { return ((SS(solver)*)h)->t; }

#undef SF
#undef SS
#undef SC
#undef SC_
