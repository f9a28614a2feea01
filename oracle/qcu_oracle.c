/*
 * CPU oracle for the Wilson-clover hot path - TEST INFRASTRUCTURE ONLY.
 * See qcu_oracle.h for the layouts and for what pins this restatement.
 * Every routine cites the reference file:line (paths inside cg_inverter/) whose
 * behaviour it restates. Nothing in the product library calls this file.
 */
#include "qcu_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* ------------------------------------------------------------------------- */
/* lattice geometry                                                          */
/* ------------------------------------------------------------------------- */
typedef struct {
  int Lx, Ly, Lz, Lt, Lxh;
  size_t V, Vh;
} geom_t;

static geom_t geom(const int L[4]) {
  geom_t g;
  g.Lx = L[0]; g.Ly = L[1]; g.Lz = L[2]; g.Lt = L[3];
  g.Lxh = L[0] / 2;
  g.V = (size_t)L[0] * L[1] * L[2] * L[3];
  g.Vh = g.V / 2;
  return g;
}

/* checkerboard index of the site; coordinates are (x/2, y, z, t) as in
 * include/qcu_point.cuh:70-72 */
static inline size_t cb_index(const geom_t* g, int xh, int y, int z, int t) {
  return (((size_t)t * g->Lz + z) * g->Ly + y) * g->Lxh + xh;
}
static inline void cb_coords(const geom_t* g, size_t s, int* xh, int* y, int* z, int* t) {
  *xh = (int)(s % g->Lxh); s /= g->Lxh;
  *y = (int)(s % g->Ly); s /= g->Ly;
  *z = (int)(s % g->Lz); s /= g->Lz;
  *t = (int)s;
}

/* Neighbour of a checkerboard site in direction mu (0..3), forward (fb=1) or
 * backward (fb=0). Restates Point::move, include/qcu_point.cuh:20-63: the x
 * step moves x/2 only when eo != parity (forward) or eo == parity (backward),
 * with eo = (y+z+t)&1, and every step wraps periodically. */
static inline size_t cb_move(const geom_t* g, int parity, int xh, int y, int z, int t, int mu, int fb) {
  int eo = (y + z + t) & 1;
  switch (mu) {
    case 0:
      if (fb) xh = xh + (eo != parity) * (1 + (xh == g->Lxh - 1) * (-g->Lxh));
      else xh = xh + (eo == parity) * (-1 + (xh == 0) * g->Lxh);
      break;
    case 1: y = fb ? (y + 1 == g->Ly ? 0 : y + 1) : (y == 0 ? g->Ly - 1 : y - 1); break;
    case 2: z = fb ? (z + 1 == g->Lz ? 0 : z + 1) : (z == 0 ? g->Lz - 1 : z - 1); break;
    default: t = fb ? (t + 1 == g->Lt ? 0 : t + 1) : (t == 0 ? g->Lt - 1 : t - 1); break;
  }
  return cb_index(g, xh, y, z, t);
}

/* index of the full-lattice site (x,y,z,t) in [parity][cb] order */
static inline void full_to_cb(const geom_t* g, int x, int y, int z, int t, int* parity, size_t* s) {
  x = (x % g->Lx + g->Lx) % g->Lx;
  y = (y % g->Ly + g->Ly) % g->Ly;
  z = (z % g->Lz + g->Lz) % g->Lz;
  t = (t % g->Lt + g->Lt) % g->Lt;
  *parity = (x + y + z + t) & 1;
  *s = cb_index(g, x >> 1, y, z, t);
}

/* ------------------------------------------------------------------------- */
/* SU(3) helpers                                                              */
/* ------------------------------------------------------------------------- */
/* row 3 = conj(row 1 x row 2), src/qcu_clover_dslash.cu:11-16 */
static inline void su3_reconstruct(cplx u[9]) {
  u[6] = conj(u[1] * u[5] - u[2] * u[4]);
  u[7] = conj(u[2] * u[3] - u[0] * u[5]);
  u[8] = conj(u[0] * u[4] - u[1] * u[3]);
}
/* loads the first two rows of a link and rebuilds the third, as the reference
 * does for every link it uses (src/qcu_clover_dslash.cu:102-108, 119-124) */
static inline void load_link(cplx u[9], const double* gauge, const geom_t* g, int mu, int parity, size_t s) {
  const cplx* src = (const cplx*)gauge + (((size_t)mu * 2 + parity) * g->Vh + s) * 9;
  for (int i = 0; i < 6; i++) u[i] = src[i];
  su3_reconstruct(u);
}
static inline void load_link_full(cplx u[9], const double* gauge, const geom_t* g, int mu, int x, int y, int z, int t) {
  int p; size_t s;
  full_to_cb(g, x, y, z, t, &p, &s);
  load_link(u, gauge, g, mu, p, s);
}
static inline void mat_mul(cplx r[9], const cplx a[9], const cplx b[9]) {
  cplx t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      cplx acc = 0;
      for (int k = 0; k < 3; k++) acc += a[i * 3 + k] * b[k * 3 + j];
      t[i * 3 + j] = acc;
    }
  memcpy(r, t, sizeof(t));
}
static inline void mat_dag(cplx r[9], const cplx a[9]) {
  cplx t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) t[i * 3 + j] = conj(a[j * 3 + i]);
  memcpy(r, t, sizeof(t));
}
static inline void mat_vec(cplx o[3], const cplx u[9], const cplx v[3]) {
  for (int i = 0; i < 3; i++) o[i] = u[i * 3 + 0] * v[0] + u[i * 3 + 1] * v[1] + u[i * 3 + 2] * v[2];
}
static inline void mat_dag_vec(cplx o[3], const cplx u[9], const cplx v[3]) {
  for (int i = 0; i < 3; i++) o[i] = conj(u[0 * 3 + i]) * v[0] + conj(u[1 * 3 + i]) * v[1] + conj(u[2 * 3 + i]) * v[2];
}

/* ------------------------------------------------------------------------- */
/* counter-based random numbers (SplitMix64 streams)                          */
/* ------------------------------------------------------------------------- */
/* Each generated object (a link, a spinor site) owns one stream keyed by
 * (seed, object index), so the values do not depend on the order or the
 * number of threads that generate them. The CUDA generator in the product
 * library uses the same streams. */
static inline uint64_t sm64_next(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline uint64_t stream_init(uint64_t seed, uint64_t object) {
  uint64_t s = seed ^ 0xD1B54A32D192ED03ull;
  s += object * 0x632BE59BD9B4E019ull;
  (void)sm64_next(&s);
  return s;
}
static inline double unif01(uint64_t* s) { return (double)(sm64_next(s) >> 11) * 0x1.0p-53; }
/* Box-Muller pair of N(0,1) */
static inline void gauss2(uint64_t* s, double* a, double* b) {
  double u1 = 1.0 - unif01(s); /* (0,1] */
  double u2 = unif01(s);
  double r = sqrt(-2.0 * log(u1));
  double th = 6.283185307179586476925286766559 * u2;
  *a = r * cos(th);
  *b = r * sin(th);
}

/* U = exp(i*eps*H) by scaling and squaring of a degree-12 Taylor series, then
 * reunitarised: Gram-Schmidt on rows 1-2, row 3 = conj(row1 x row2). H is
 * traceless Hermitian: diagonal = three N(0,1) minus their mean, each
 * off-diagonal entry N(0,1) + i N(0,1). */
static void su3_from_stream(cplx u[9], uint64_t* st, double eps) {
  double g[10];
  for (int k = 0; k < 5; k++) gauss2(st, &g[2 * k], &g[2 * k + 1]);
  cplx H[9];
  double mean = (g[0] + g[1] + g[2]) / 3.0;
  H[0] = g[0] - mean; H[4] = g[1] - mean; H[8] = g[2] - mean;
  H[1] = g[3] + I * g[4]; H[3] = conj(H[1]);
  H[2] = g[5] + I * g[6]; H[6] = conj(H[2]);
  H[5] = g[7] + I * g[8]; H[7] = conj(H[5]);
  cplx X[9];
  double nrm = 0;
  for (int i = 0; i < 9; i++) {
    X[i] = I * eps * H[i];
    nrm += creal(X[i]) * creal(X[i]) + cimag(X[i]) * cimag(X[i]);
  }
  nrm = sqrt(nrm);
  int k = 0;
  while (nrm > 0.25 && k < 30) { nrm *= 0.5; k++; }
  double sc = ldexp(1.0, -k);
  for (int i = 0; i < 9; i++) X[i] *= sc;
  /* Horner: E = I + X(I + X/2(I + X/3(...(I + X/12)))) */
  cplx E[9];
  for (int i = 0; i < 9; i++) E[i] = (i % 4 == 0) ? 1.0 : 0.0;
  for (int n = 12; n >= 1; n--) {
    cplx T[9];
    mat_mul(T, X, E);
    for (int i = 0; i < 9; i++) E[i] = ((i % 4 == 0) ? 1.0 : 0.0) + T[i] / (double)n;
  }
  for (int s = 0; s < k; s++) mat_mul(E, E, E);
  /* Gram-Schmidt rows 0 and 1 */
  double n0 = 0;
  for (int j = 0; j < 3; j++) n0 += creal(E[j]) * creal(E[j]) + cimag(E[j]) * cimag(E[j]);
  n0 = 1.0 / sqrt(n0);
  for (int j = 0; j < 3; j++) u[j] = E[j] * n0;
  cplx ip = 0;
  for (int j = 0; j < 3; j++) ip += conj(u[j]) * E[3 + j];
  cplx r1[3];
  for (int j = 0; j < 3; j++) r1[j] = E[3 + j] - ip * u[j];
  double n1 = 0;
  for (int j = 0; j < 3; j++) n1 += creal(r1[j]) * creal(r1[j]) + cimag(r1[j]) * cimag(r1[j]);
  n1 = 1.0 / sqrt(n1);
  for (int j = 0; j < 3; j++) u[3 + j] = r1[j] * n1;
  su3_reconstruct(u);
}

void orc_gauge_random(double* gauge, const int L[4], uint64_t seed, double eps) {
  geom_t g = geom(L);
  size_t nlinks = 4 * g.V;
#pragma omp parallel for schedule(static)
  for (size_t l = 0; l < nlinks; l++) {
    uint64_t st = stream_init(seed, l);
    su3_from_stream((cplx*)gauge + l * 9, &st, eps);
  }
}

void orc_gauge_unit(double* gauge, const int L[4]) {
  geom_t g = geom(L);
  size_t nlinks = 4 * g.V;
  cplx* u = (cplx*)gauge;
  for (size_t l = 0; l < nlinks; l++)
    for (int i = 0; i < 9; i++) u[l * 9 + i] = (i % 4 == 0) ? 1.0 : 0.0;
}

void orc_su3_random_field(double* gfield, const int L[4], uint64_t seed) {
  geom_t g = geom(L);
#pragma omp parallel for schedule(static)
  for (size_t l = 0; l < g.V; l++) {
    uint64_t st = stream_init(seed ^ 0x5bd1e995ull, l);
    su3_from_stream((cplx*)gfield + l * 9, &st, 1.0);
  }
}

/* U'_mu(x) = g(x) U_mu(x) g(x+mu)^dag, g stored per site in [parity][cb][3][3] */
void orc_gauge_transform(double* out, const double* gauge, const double* gf, const int L[4]) {
  geom_t g = geom(L);
  const cplx* G = (const cplx*)gf;
#pragma omp parallel for schedule(static)
  for (size_t l = 0; l < 4 * g.V; l++) {
    int mu = (int)(l / g.V);
    size_t rem = l % g.V;
    int parity = (int)(rem / g.Vh);
    size_t s = rem % g.Vh;
    int xh, y, z, t;
    cb_coords(&g, s, &xh, &y, &z, &t);
    size_t sn = cb_move(&g, parity, xh, y, z, t, mu, 1);
    cplx u[9], gd[9], tmp[9];
    const cplx* src = (const cplx*)gauge + l * 9;
    for (int i = 0; i < 9; i++) u[i] = src[i];
    mat_dag(gd, G + ((size_t)(1 - parity) * g.Vh + sn) * 9);
    mat_mul(tmp, G + ((size_t)parity * g.Vh + s) * 9, u);
    mat_mul(tmp, tmp, gd);
    memcpy((cplx*)out + l * 9, tmp, sizeof(tmp));
  }
}

void orc_gauge_pure(double* gauge, const int L[4], uint64_t seed) {
  geom_t g = geom(L);
  double* gf = (double*)malloc(sizeof(cplx) * 9 * g.V);
  orc_su3_random_field(gf, L, seed);
  orc_gauge_unit(gauge, L);
  double* tmp = (double*)malloc(sizeof(cplx) * 9 * 4 * g.V);
  orc_gauge_transform(tmp, gauge, gf, L);
  memcpy(gauge, tmp, sizeof(cplx) * 9 * 4 * g.V);
  free(tmp);
  free(gf);
}

void orc_spinor_random(double* psi, size_t nsites, uint64_t seed) {
#pragma omp parallel for schedule(static)
  for (size_t s = 0; s < nsites; s++) {
    uint64_t st = stream_init(seed ^ 0xA0761D6478BD642Full, s);
    for (int k = 0; k < 12; k++) gauss2(&st, &psi[s * 24 + 2 * k], &psi[s * 24 + 2 * k + 1]);
  }
}

void orc_spinor_transform(double* out, const double* psi, const double* gf, const int L[4]) {
  geom_t g = geom(L);
#pragma omp parallel for schedule(static)
  for (size_t s = 0; s < g.V; s++) {
    const cplx* G = (const cplx*)gf + s * 9;
    const cplx* in = (const cplx*)psi + s * 12;
    cplx* o = (cplx*)out + s * 12;
    cplx v[3], w[3];
    for (int sp = 0; sp < 4; sp++) {
      for (int c = 0; c < 3; c++) v[c] = in[sp * 3 + c];
      mat_vec(w, G, v);
      for (int c = 0; c < 3; c++) o[sp * 3 + c] = w[c];
    }
  }
}

/* ------------------------------------------------------------------------- */
/* hopping term, src/qcu_clover_dslash.cu:570-772                            */
/* ------------------------------------------------------------------------- */
/* D psi(x) = sum_mu (1 - f gamma_mu) U_mu(x) psi(x+mu) + (1 + f gamma_mu) U_mu(x-mu)^dag psi(x-mu)
 * with f = +1 (dagger = 0) or -1 (dagger = 1), DeGrand-Rossi gamma matrices.
 * Each direction is written as the reference writes it: a two-component
 * projection h0, h1, a colour multiply, and the spin reconstruction. */
static void hop_site(cplx out[12], const double* in_half, const double* gauge, const geom_t* g,
                     int parity, size_t s, double f, double bc_t) {
  int xh, y, z, t;
  cb_coords(g, s, &xh, &y, &z, &t);
  const cplx* in = (const cplx*)in_half;
  cplx u[9], h0[3], h1[3], a[3], b[3];
  const cplx fi = f * I;
  for (int k = 0; k < 12; k++) out[k] = 0;
  for (int mu = 0; mu < 4; mu++) {
    /* forward */
    size_t n = cb_move(g, parity, xh, y, z, t, mu, 1);
    load_link(u, gauge, g, mu, parity, s);
    const cplx* p = in + n * 12;
    double ph = (mu == 3 && t == g->Lt - 1) ? bc_t : 1.0;
    for (int c = 0; c < 3; c++) {
      switch (mu) {
        case 0: h0[c] = p[c] - fi * p[9 + c]; h1[c] = p[3 + c] - fi * p[6 + c]; break;
        case 1: h0[c] = p[c] + f * p[9 + c]; h1[c] = p[3 + c] - f * p[6 + c]; break;
        case 2: h0[c] = p[c] - fi * p[6 + c]; h1[c] = p[3 + c] + fi * p[9 + c]; break;
        default: h0[c] = p[c] - f * p[6 + c]; h1[c] = p[3 + c] - f * p[9 + c]; break;
      }
      h0[c] *= ph; h1[c] *= ph;
    }
    mat_vec(a, u, h0);
    mat_vec(b, u, h1);
    for (int c = 0; c < 3; c++) {
      out[c] += a[c];
      out[3 + c] += b[c];
      switch (mu) {
        case 0: out[6 + c] += fi * b[c]; out[9 + c] += fi * a[c]; break;
        case 1: out[6 + c] -= f * b[c]; out[9 + c] += f * a[c]; break;
        case 2: out[6 + c] += fi * a[c]; out[9 + c] -= fi * b[c]; break;
        default: out[6 + c] -= f * a[c]; out[9 + c] -= f * b[c]; break;
      }
    }
    /* backward: link of the neighbour (parity 1-parity), daggered */
    n = cb_move(g, parity, xh, y, z, t, mu, 0);
    load_link(u, gauge, g, mu, 1 - parity, n);
    p = in + n * 12;
    ph = (mu == 3 && t == 0) ? bc_t : 1.0;
    for (int c = 0; c < 3; c++) {
      switch (mu) {
        case 0: h0[c] = p[c] + fi * p[9 + c]; h1[c] = p[3 + c] + fi * p[6 + c]; break;
        case 1: h0[c] = p[c] - f * p[9 + c]; h1[c] = p[3 + c] + f * p[6 + c]; break;
        case 2: h0[c] = p[c] + fi * p[6 + c]; h1[c] = p[3 + c] - fi * p[9 + c]; break;
        default: h0[c] = p[c] + f * p[6 + c]; h1[c] = p[3 + c] + f * p[9 + c]; break;
      }
      h0[c] *= ph; h1[c] *= ph;
    }
    mat_dag_vec(a, u, h0);
    mat_dag_vec(b, u, h1);
    for (int c = 0; c < 3; c++) {
      out[c] += a[c];
      out[3 + c] += b[c];
      switch (mu) {
        case 0: out[6 + c] -= fi * b[c]; out[9 + c] -= fi * a[c]; break;
        case 1: out[6 + c] += f * b[c]; out[9 + c] -= f * a[c]; break;
        case 2: out[6 + c] -= fi * a[c]; out[9 + c] += fi * b[c]; break;
        default: out[6 + c] += f * a[c]; out[9 + c] += f * b[c]; break;
      }
    }
  }
}

void orc_dslash(double* out_half, const double* in_half, const double* gauge, const int L[4],
                int parity, int dagger, double bc_t) {
  geom_t g = geom(L);
  double f = dagger ? -1.0 : 1.0;
#pragma omp parallel for schedule(static)
  for (size_t s = 0; s < g.Vh; s++) hop_site((cplx*)out_half + s * 12, in_half, gauge, &g, parity, s, f, bc_t);
}

/* ------------------------------------------------------------------------- */
/* clover term                                                                */
/* ------------------------------------------------------------------------- */
/* Spin structure of tensorProductAddition, src/qcu_clover_dslash.cu:210-267:
 * for plane (mu,nu) and row spin s the entry goes to column spin kCol[pl][s]
 * with phase kPhase[pl][s]; every entry is scaled by 2*coef. */
static const int kPlaneMu[6] = {0, 0, 0, 1, 1, 2};
static const int kPlaneNu[6] = {1, 2, 3, 2, 3, 3};
static const int kCol[6][4] = {{0, 1, 2, 3}, {1, 0, 3, 2}, {1, 0, 3, 2}, {1, 0, 3, 2}, {1, 0, 3, 2}, {0, 1, 2, 3}};
static const double kPhRe[6][4] = {{0, 0, 0, 0}, {-1, 1, -1, 1}, {0, 0, 0, 0}, {0, 0, 0, 0}, {-1, 1, 1, -1}, {0, 0, 0, 0}};
static const double kPhIm[6][4] = {{-1, 1, -1, 1}, {0, 0, 0, 0}, {1, 1, -1, -1}, {-1, -1, -1, -1}, {0, 0, 0, 0}, {1, -1, -1, 1}};

/* Q_munu(x) = F1+F2+F3+F4, the four leaves of src/qcu_clover_dslash.cu:329-413:
 *  F1 = U_mu(x) U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
 *  F2 = U_nu(x) U_mu(x-mu+nu)^dag U_nu(x-mu)^dag U_mu(x-mu)
 *  F3 = U_mu(x-mu)^dag U_nu(x-mu-nu)^dag U_mu(x-mu-nu) U_nu(x-nu)
 *  F4 = U_nu(x-nu)^dag U_mu(x-nu) U_nu(x+mu-nu) U_mu(x)^dag
 * The reference reads the shifted links from 32 shifted copies of the gauge
 * field (src/qcu_communicator.cu:755-980, 1270-1297); on one rank those are
 * plain periodic shifts, which is what direct neighbour indexing gives. */
static void clover_leaves(cplx Q[9], const double* gauge, const geom_t* g, int x, int y, int z, int t, int mu, int nu) {
  int dm[4] = {0, 0, 0, 0}, dn[4] = {0, 0, 0, 0};
  dm[mu] = 1; dn[nu] = 1;
#define LNK(out, d, ox, oy, oz, ot) load_link_full(out, gauge, g, d, x + (ox), y + (oy), z + (oz), t + (ot))
  cplx a[9], b[9], c[9], d[9], r[9];
  for (int i = 0; i < 9; i++) Q[i] = 0;
  /* F1 */
  LNK(a, mu, 0, 0, 0, 0);
  LNK(b, nu, dm[0], dm[1], dm[2], dm[3]);
  LNK(c, mu, dn[0], dn[1], dn[2], dn[3]);
  LNK(d, nu, 0, 0, 0, 0);
  mat_mul(r, a, b); mat_dag(c, c); mat_mul(r, r, c); mat_dag(d, d); mat_mul(r, r, d);
  for (int i = 0; i < 9; i++) Q[i] += r[i];
  /* F2 */
  LNK(a, nu, 0, 0, 0, 0);
  LNK(b, mu, -dm[0] + dn[0], -dm[1] + dn[1], -dm[2] + dn[2], -dm[3] + dn[3]);
  LNK(c, nu, -dm[0], -dm[1], -dm[2], -dm[3]);
  LNK(d, mu, -dm[0], -dm[1], -dm[2], -dm[3]);
  mat_dag(b, b); mat_mul(r, a, b); mat_dag(c, c); mat_mul(r, r, c); mat_mul(r, r, d);
  for (int i = 0; i < 9; i++) Q[i] += r[i];
  /* F3 */
  LNK(a, mu, -dm[0], -dm[1], -dm[2], -dm[3]);
  LNK(b, nu, -dm[0] - dn[0], -dm[1] - dn[1], -dm[2] - dn[2], -dm[3] - dn[3]);
  LNK(c, mu, -dm[0] - dn[0], -dm[1] - dn[1], -dm[2] - dn[2], -dm[3] - dn[3]);
  LNK(d, nu, -dn[0], -dn[1], -dn[2], -dn[3]);
  mat_dag(a, a); mat_dag(b, b); mat_mul(r, a, b); mat_mul(r, r, c); mat_mul(r, r, d);
  for (int i = 0; i < 9; i++) Q[i] += r[i];
  /* F4 */
  LNK(a, nu, -dn[0], -dn[1], -dn[2], -dn[3]);
  LNK(b, mu, -dn[0], -dn[1], -dn[2], -dn[3]);
  LNK(c, nu, dm[0] - dn[0], dm[1] - dn[1], dm[2] - dn[2], dm[3] - dn[3]);
  LNK(d, mu, 0, 0, 0, 0);
  mat_dag(a, a); mat_mul(r, a, b); mat_mul(r, r, c); mat_dag(d, d); mat_mul(r, r, d);
  for (int i = 0; i < 9; i++) Q[i] += r[i];
#undef LNK
}

/* A = 1 + csw*T with T = (-1/16)*2*sum_{mu<nu} (spin phase) x (Q - Q^dag),
 * src/qcu_clover_dslash.cu:415-458 and :537-540; csw = 1 is the reference. */
void orc_clover_build(double* clover, const double* gauge, const int L[4], double csw) {
  geom_t g = geom(L);
#pragma omp parallel for schedule(static)
  for (size_t l = 0; l < g.V; l++) {
    int parity = (int)(l / g.Vh);
    size_t s = l % g.Vh;
    int xh, y, z, t;
    cb_coords(&g, s, &xh, &y, &z, &t);
    int x = 2 * xh + ((y + z + t + parity) & 1);
    cplx T[2][36];
    for (int i = 0; i < 72; i++) (&T[0][0])[i] = 0;
    for (int pl = 0; pl < 6; pl++) {
      cplx Q[9], G[9];
      clover_leaves(Q, gauge, &g, x, y, z, t, kPlaneMu[pl], kPlaneNu[pl]);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) G[i * 3 + j] = Q[i * 3 + j] - conj(Q[j * 3 + i]);
      for (int sp = 0; sp < 4; sp++) {
        int blk = sp / 2, r0 = (sp % 2) * 3, c0 = (kCol[pl][sp] % 2) * 3;
        cplx ph = (kPhRe[pl][sp] + I * kPhIm[pl][sp]) * (-1.0 / 16.0) * 2.0 * csw;
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) T[blk][(r0 + i) * 6 + c0 + j] += ph * G[i * 3 + j];
      }
    }
    cplx* dst = (cplx*)clover + l * 72;
    for (int b = 0; b < 2; b++)
      for (int i = 0; i < 36; i++) dst[b * 36 + i] = T[b][i] + ((i % 7 == 0) ? 1.0 : 0.0);
  }
}

/* Gauss-Jordan inverse of a 6x6 complex matrix with partial pivoting
 * (the reference's inverseMatrix, src/qcu_clover_dslash.cu:42-100, pivots only
 * on an exact zero; for a nonsingular block both give the same inverse). */
static int inv6(cplx out[36], const cplx in[36]) {
  cplx a[6][12];
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 12; j++) a[i][j] = (j < 6) ? in[i * 6 + j] : ((j - 6 == i) ? 1.0 : 0.0);
  for (int c = 0; c < 6; c++) {
    int piv = c;
    double best = cabs(a[c][c]);
    for (int r = c + 1; r < 6; r++)
      if (cabs(a[r][c]) > best) { best = cabs(a[r][c]); piv = r; }
    if (best == 0.0) return -1;
    if (piv != c)
      for (int j = 0; j < 12; j++) { cplx tmp = a[c][j]; a[c][j] = a[piv][j]; a[piv][j] = tmp; }
    cplx d = 1.0 / a[c][c];
    for (int j = 0; j < 12; j++) a[c][j] *= d;
    for (int r = 0; r < 6; r++) {
      if (r == c) continue;
      cplx m = a[r][c];
      for (int j = 0; j < 12; j++) a[r][j] -= m * a[c][j];
    }
  }
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) out[i * 6 + j] = a[i][6 + j];
  return 0;
}

int orc_clover_invert(double* inv, const double* clover, size_t nsites) {
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
  for (size_t s = 0; s < 2 * nsites; s++)
    bad += inv6((cplx*)inv + s * 36, (const cplx*)clover + s * 36) != 0;
  return bad;
}

/* gpuCloverCalculate, src/qcu_clover_dslash.cu:461-506 */
void orc_clover_apply(double* psi, const double* mat, size_t nsites) {
#pragma omp parallel for schedule(static)
  for (size_t s = 0; s < nsites; s++) {
    cplx* v = (cplx*)psi + s * 12;
    const cplx* m = (const cplx*)mat + s * 72;
    cplx o[12];
    for (int b = 0; b < 2; b++)
      for (int i = 0; i < 6; i++) {
        cplx acc = 0;
        for (int j = 0; j < 6; j++) acc += m[b * 36 + i * 6 + j] * v[b * 6 + j];
        o[b * 6 + i] = acc;
      }
    memcpy(v, o, sizeof(o));
  }
}

/* ------------------------------------------------------------------------- */
/* BLAS, src/qcu_complex_computation.cu:10-133                                */
/* ------------------------------------------------------------------------- */
void orc_cdot(const double* x, const double* y, size_t n, double out[2]) {
  double re = 0, im = 0;
#pragma omp parallel for schedule(static) reduction(+ : re, im)
  for (size_t i = 0; i < n; i++) {
    double xr = x[2 * i], xi = x[2 * i + 1], yr = y[2 * i], yi = y[2 * i + 1];
    re += xr * yr + xi * yi;
    im += xr * yi - xi * yr;
  }
  out[0] = re; out[1] = im;
}
void orc_caxpy(double* y, const double* x, const double a[2], size_t n) {
  cplx A = a[0] + I * a[1];
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) ((cplx*)y)[i] += ((const cplx*)x)[i] * A;
}
void orc_cscale(double* x, const double a[2], size_t n) {
  cplx A = a[0] + I * a[1];
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < n; i++) ((cplx*)x)[i] = A * ((cplx*)x)[i];
}

/* ------------------------------------------------------------------------- */
/* reference compositions, src/qcu_clover_dslash.cu:902-1049                  */
/* ------------------------------------------------------------------------- */
/* out_p = A^-1_p D_{p,1-p} in_{1-p} for both parities (cloverDslashOneRound :990) */
static void clover_dslash_round(double* out, const double* in, const double* gauge, const double* clover_inv,
                                const geom_t* g, const int L[4], int dagger) {
  for (int p = 0; p < 2; p++) {
    double* o = out + (size_t)p * g->Vh * 24;
    orc_dslash(o, in + (size_t)(1 - p) * g->Vh * 24, gauge, L, p, dagger, 1.0);
    orc_clover_apply(o, clover_inv + (size_t)p * g->Vh * 144, g->Vh);
  }
}

/* fullCloverDslashOneRound (:948): out = A (in - A^-1 D in) = A in - D in */
void orc_full_dslash_ref(double* out, const double* in, const double* gauge, const double* clover,
                         const double* clover_inv, const int L[4], int dagger) {
  geom_t g = geom(L);
  clover_dslash_round(out, in, gauge, clover_inv, &g, L, dagger);
  const double m1[2] = {-1, 0}, p1[2] = {1, 0};
  orc_cscale(out, m1, g.V * 12);
  orc_caxpy(out, in, p1, g.V * 12);
  for (int p = 0; p < 2; p++) orc_clover_apply(out + (size_t)p * g.Vh * 24, clover + (size_t)p * g.Vh * 144, g.Vh);
}

/* newFullCloverDslashOneRound (:1013): out = in - A^-1 D in */
void orc_new_full_ref(double* out, const double* in, const double* gauge, const double* clover_inv,
                      const int L[4], int dagger) {
  geom_t g = geom(L);
  clover_dslash_round(out, in, gauge, clover_inv, &g, L, dagger);
  const double m1[2] = {-1, 0}, p1[2] = {1, 0};
  orc_cscale(out, m1, g.V * 12);
  orc_caxpy(out, in, p1, g.V * 12);
}

/* MmV_one_round (:1044): (1 - A^-1 D^dag)(1 - A^-1 D) in */
void orc_mmv_ref(double* out, const double* in, const double* gauge, const double* clover_inv, const int L[4]) {
  geom_t g = geom(L);
  double* tmp = (double*)malloc(sizeof(double) * 24 * g.V);
  orc_new_full_ref(tmp, in, gauge, clover_inv, L, 0);
  orc_new_full_ref(out, tmp, gauge, clover_inv, L, 1);
  free(tmp);
}

/* invertCloverDslash (:902): in place on out, parity by parity */
void orc_invert_clover_ref(double* out, const double* clover_inv, const int L[4]) {
  geom_t g = geom(L);
  for (int p = 0; p < 2; p++) orc_clover_apply(out + (size_t)p * g.Vh * 24, clover_inv + (size_t)p * g.Vh * 144, g.Vh);
}

static inline double cnorm_of(const double c[2]) { return sqrt(c[0] * c[0] + c[1] * c[1]); }

/* cg_inverter + cg + if_converge, src/cg_inverter.cu:125-146, 181-256, 260-369.
 * Complex alpha = <r,r>/<p,Ap>, beta = <r',r'>/<r,r>; the convergence test is
 * |<r,r>| < 1e-23 on the residual from BEFORE the update (:225), taken after x
 * has already moved; at most V iterations. */
int orc_cg_inverter_ref(double* x, const double* b, const double* gauge, const int L[4], int maxiter, int* converged) {
  geom_t g = geom(L);
  size_t n = g.V * 12;
  if (maxiter <= 0) maxiter = (int)g.V;
  double* clover = (double*)malloc(sizeof(double) * 144 * g.V);
  double* cinv = (double*)malloc(sizeof(double) * 144 * g.V);
  orc_clover_build(clover, gauge, L, 1.0);
  orc_clover_invert(cinv, clover, g.V);
  double* nb = (double*)malloc(sizeof(double) * 2 * n);
  double* tmp = (double*)malloc(sizeof(double) * 2 * n);
  double* r = (double*)malloc(sizeof(double) * 2 * n);
  double* p = (double*)malloc(sizeof(double) * 2 * n);
  double* ap = (double*)malloc(sizeof(double) * 2 * n);
  double* r2 = (double*)malloc(sizeof(double) * 2 * n);
  memset(x, 0, sizeof(double) * 2 * n);
  memcpy(tmp, b, sizeof(double) * 2 * n);
  orc_invert_clover_ref(tmp, cinv, L);
  orc_new_full_ref(nb, tmp, gauge, cinv, L, 1);
  orc_mmv_ref(ap, x, gauge, cinv, L);
  memcpy(r, nb, sizeof(double) * 2 * n);
  const double m1[2] = {-1, 0};
  orc_caxpy(r, ap, m1, n);
  memcpy(p, r, sizeof(double) * 2 * n);
  double d[2];
  *converged = 0;
  orc_cdot(r, r, n, d);
  int it = 0;
  if (cnorm_of(d) < 1e-23) { *converged = 1; goto done; }
  for (it = 0; it < maxiter;) {
    double num[2], den[2];
    orc_cdot(r, r, n, num);
    orc_mmv_ref(ap, p, gauge, cinv, L);
    orc_cdot(p, ap, n, den);
    cplx alpha = (num[0] + I * num[1]) / (den[0] + I * den[1]);
    double a[2] = {creal(alpha), cimag(alpha)};
    orc_caxpy(x, p, a, n);
    memcpy(r2, r, sizeof(double) * 2 * n);
    double ma[2] = {-a[0], -a[1]};
    orc_caxpy(r2, ap, ma, n);
    it++;
    orc_cdot(r, r, n, d);
    if (cnorm_of(d) < 1e-23) { *converged = 1; break; }
    double rr2[2];
    orc_cdot(r2, r2, n, rr2);
    cplx beta = (rr2[0] + I * rr2[1]) / (num[0] + I * num[1]);
    double bb[2] = {creal(beta), cimag(beta)};
    orc_cscale(p, bb, n);
    const double one[2] = {1, 0};
    orc_caxpy(p, r2, one, n);
    memcpy(r, r2, sizeof(double) * 2 * n);
  }
done:
  free(clover); free(cinv); free(nb); free(tmp); free(r); free(p); free(ap); free(r2);
  return it;
}

/* ------------------------------------------------------------------------- */
/* extended physics: M = A - kappa D with A = 1 + kappa*c_sw*T                */
/* ------------------------------------------------------------------------- */
void orc_apply_full(double* out, const double* in, const double* gauge, const double* clover,
                    const int L[4], double kappa, double bc_t, int dagger) {
  geom_t g = geom(L);
  double* tmp = (double*)malloc(sizeof(double) * 24 * g.Vh);
  for (int p = 0; p < 2; p++) {
    double* o = out + (size_t)p * g.Vh * 24;
    orc_dslash(tmp, in + (size_t)(1 - p) * g.Vh * 24, gauge, L, p, dagger, bc_t);
    memcpy(o, in + (size_t)p * g.Vh * 24, sizeof(double) * 24 * g.Vh);
    orc_clover_apply(o, clover + (size_t)p * g.Vh * 144, g.Vh);
    const double mk[2] = {-kappa, 0};
    orc_caxpy(o, tmp, mk, g.Vh * 12);
  }
  free(tmp);
}

/* Mhat x = x - k^2 A_ee^-1 D_eo A_oo^-1 D_oe x;
 * Mhat^dag y = y - k^2 D^dag_eo A_oo^-1 D^dag_oe A_ee^-1 y */
void orc_schur_apply(double* out, const double* in, const double* gauge, const double* cinv,
                     const int L[4], double kappa, double bc_t, int dagger) {
  geom_t g = geom(L);
  size_t nh = g.Vh * 12;
  double* t1 = (double*)malloc(sizeof(double) * 2 * nh);
  double* t2 = (double*)malloc(sizeof(double) * 2 * nh);
  const double* cee = cinv;
  const double* coo = cinv + g.Vh * 144;
  if (!dagger) {
    orc_dslash(t1, in, gauge, L, 1, 0, bc_t);
    orc_clover_apply(t1, coo, g.Vh);
    orc_dslash(t2, t1, gauge, L, 0, 0, bc_t);
    orc_clover_apply(t2, cee, g.Vh);
  } else {
    memcpy(t2, in, sizeof(double) * 2 * nh);
    orc_clover_apply(t2, cee, g.Vh);
    orc_dslash(t1, t2, gauge, L, 1, 1, bc_t);
    orc_clover_apply(t1, coo, g.Vh);
    orc_dslash(t2, t1, gauge, L, 0, 1, bc_t);
  }
  memcpy(out, in, sizeof(double) * 2 * nh);
  const double a[2] = {-kappa * kappa, 0};
  orc_caxpy(out, t2, a, nh);
  free(t1); free(t2);
}

static double norm2_real(const double* x, size_t n) {
  double d[2];
  orc_cdot(x, x, n, d);
  return d[0];
}

/* CG on Mhat^dag Mhat x_e = Mhat^dag bhat with a prebuilt clover A and its
 * inverse, stopping on the true residual of the full system, |b - M x|/|b| <
 * tol. The full residual is measured at checks only: at x = 0, and whenever
 * the iterated normal-equation residual |r|^2 falls below the level at which
 * the true residual is predicted at tol/2, the prediction using the ratio
 * q = |b - M x| / |Mhat^dag (bhat - Mhat x_e)| of the last check (the
 * convergence trigger of the B200 library's FP64 solve, so both stop by the
 * same rule). After a failed check the recursion restarts from the
 * recomputed residual, keeping the search direction with
 * beta = |r_new|^2 / |r_old|^2. The CG iteration itself is the plain CGNR
 * recursion of the reference's cg (src/cg_inverter.cu:181-256) on the
 * Hermitian normal operator. */
int orc_solve_schur_cl(double* x, const double* b, const double* gauge, const double* clover,
                       const double* cinv, const int L[4], double kappa, double bc_t, double tol,
                       int maxiter, double* true_res, int* checks) {
  geom_t g = geom(L);
  size_t nh = g.Vh * 12, n = g.V * 12;
  double* bh = (double*)malloc(sizeof(double) * 2 * nh);
  double* t = (double*)malloc(sizeof(double) * 2 * nh);
  double* r = (double*)malloc(sizeof(double) * 2 * nh);
  double* p = (double*)malloc(sizeof(double) * 2 * nh);
  double* y = (double*)malloc(sizeof(double) * 2 * nh);
  double* z = (double*)malloc(sizeof(double) * 2 * nh);
  double* full = (double*)malloc(sizeof(double) * 2 * n);
  const double* be = b;
  const double* bo = b + nh * 2;
  const double kk[2] = {kappa, 0};
  /* bhat = A_ee^-1 (b_e + kappa D_eo A_oo^-1 b_o) */
  memcpy(t, bo, sizeof(double) * 2 * nh);
  orc_clover_apply(t, cinv + g.Vh * 144, g.Vh);
  orc_dslash(bh, t, gauge, L, 0, 0, bc_t);
  memcpy(t, be, sizeof(double) * 2 * nh);
  orc_caxpy(t, bh, kk, nh);
  memcpy(bh, t, sizeof(double) * 2 * nh);
  orc_clover_apply(bh, cinv, g.Vh);
  double b2 = norm2_real(b, n);
  memset(x, 0, sizeof(double) * 2 * n);
  double* xe = x;
  double* xo = x + 2 * nh;
  int iters = 0, nchk = 0;
  double res = 1.0, rr = 0.0;
  memset(p, 0, sizeof(double) * 2 * nh);
  for (;;) {
    /* check: x_o = A_oo^-1 (b_o + kappa D_oe x_e), then |b - M x| */
    orc_dslash(t, xe, gauge, L, 1, 0, bc_t);
    memcpy(xo, bo, sizeof(double) * 2 * nh);
    orc_caxpy(xo, t, kk, nh);
    orc_clover_apply(xo, cinv + g.Vh * 144, g.Vh);
    orc_apply_full(full, x, gauge, clover, L, kappa, bc_t, 0);
    for (size_t i = 0; i < 2 * n; i++) full[i] = b[i] - full[i];
    const double ar2 = norm2_real(full, n);
    res = b2 > 0 ? sqrt(ar2 / b2) : 0.0;
    nchk++;
    if (res < tol || iters >= maxiter || !isfinite(res)) break;
    /* r = Mhat^dag (bhat - Mhat x_e) */
    orc_schur_apply(y, xe, gauge, cinv, L, kappa, bc_t, 0);
    for (size_t i = 0; i < 2 * nh; i++) y[i] = bh[i] - y[i];
    orc_schur_apply(r, y, gauge, cinv, L, kappa, bc_t, 1);
    const double ne2 = norm2_real(r, nh);
    const double beta = rr > 0 ? ne2 / rr : 0.0;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < 2 * nh; i++) p[i] = r[i] + beta * p[i];
    rr = ne2;
    const double q = sqrt(fmax(ar2, 1e-300) / fmax(ne2, 1e-300));
    const double target = 0.5 * tol * sqrt(b2) / q;
    while (rr > target * target && iters < maxiter) {
      orc_schur_apply(y, p, gauge, cinv, L, kappa, bc_t, 0);
      double pap = norm2_real(y, nh);
      orc_schur_apply(z, y, gauge, cinv, L, kappa, bc_t, 1);
      double alpha = rr / pap;
      const double pa[2] = {alpha, 0}, ma[2] = {-alpha, 0};
      orc_caxpy(xe, p, pa, nh);
      orc_caxpy(r, z, ma, nh);
      double rr_new = norm2_real(r, nh);
      double bt = rr_new / rr;
      rr = rr_new;
#pragma omp parallel for schedule(static)
      for (size_t i = 0; i < 2 * nh; i++) p[i] = r[i] + bt * p[i];
      iters++;
    }
  }
  if (true_res) *true_res = res;
  if (checks) *checks = nchk;
  free(bh); free(t); free(r); free(p); free(y); free(z); free(full);
  return iters;
}

int orc_solve_schur(double* x, const double* b, const double* gauge, const int L[4], double kappa,
                    double csw, double bc_t, double tol, int maxiter, double* true_res) {
  geom_t g = geom(L);
  double* clover = (double*)malloc(sizeof(double) * 144 * g.V);
  double* cinv = (double*)malloc(sizeof(double) * 144 * g.V);
  orc_clover_build(clover, gauge, L, kappa * csw);
  orc_clover_invert(cinv, clover, g.V);
  int it = orc_solve_schur_cl(x, b, gauge, clover, cinv, L, kappa, bc_t, tol, maxiter, true_res, NULL);
  free(clover); free(cinv);
  return it;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}
