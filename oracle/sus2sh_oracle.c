/*
 * Oracle (test infrastructure only): FP64 CPU evaluation of SUS2-SH site
 * energies, forces and per-atom virials.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this library; the product path never
 * does.
 *
 * Restates the reference algorithm of hu-yanxiao/GPUMD-SUS2-SH
 * (src/force/sus2_sh.cu) in its simplest correct form:
 *   neighbours   every image j with |r_j - r_i + shift|^2 < rc^2 (strict),
 *                i == j allowed for non-zero images      (:7668-7769)
 *   radial       x = tanh(scal (r - s)/2) (or z/sqrt(1+z^2)),
 *                R = s_pair (r - rc)^2 sum_n c_n T_n(x)   (:3171-3220, :2484-2517)
 *                computed in FP64 throughout (no FP32 tables)
 *   harmonics    Y_lm = c P_lm(x,y,z) / r^l, gradient by the quotient rule
 *                (:2782-2808, :3032-3169)
 *   basics       B_b = sum_j R_mu(b) Y_lm(b)               (:3486-3550)
 *   products     flat, in file order, M[t] += c M[l] M[r]  (:4813-4821)
 *   energy       E_i = shift_t + c_t + c_t sum_s w_s M[map_s]   (:4823-4832)
 *   adjoint      g[map_s] += c_t w_s, then products reversed (:4830-4845)
 *   forces       dE = sum_b g_b (R' d/r Y + R grad Y); F_i += dE, F_j -= dE,
 *                W_i -= d (x) dE, order xx yy zz xy xz yz yx zx zy (:6388-6445)
 * Outputs are assigned.  OpenMP over centre atoms.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int S, L, K, rb, kmu, M, nbasic, nscalar, nprod;
  int kind; /* radial basis: 0 Chebyshev of tanh, 1 Chebyshev of the rational map, 2 Laguerre of log1p */
  double rc;
  const double* radial;   /* [kmu][rb] */
  const double* scal;     /* [S*S][kmu] */
  const double* rshift;   /* [S*S][kmu] */
  const double* pscale;   /* [S*S] */
  const int* basic_mu;    /* [nbasic] */
  const int* basic_y;     /* [nbasic] flat harmonic index l*l+l+m */
  const int* prod_l;
  const int* prod_r;
  const int* prod_t;
  const double* prod_c;   /* [nprod] */
  const int* map;         /* [nscalar] */
  const double* w;        /* [nscalar] */
  const double* shift_e;  /* [S] */
  const double* species;  /* [S] */
} OracleModel;

/* ---- real harmonics: value c*P/r^l and gradient ------------------------- */
/* P and grad P for each (l, m), homogeneous Cartesian polynomials. */
static void poly(int idx, double x, double y, double z, double* p, double* gx, double* gy, double* gz) {
  const double x2 = x * x, y2 = y * y, z2 = z * z;
  switch (idx) {
    case 0: *p = 1; *gx = 0; *gy = 0; *gz = 0; return;
    case 1: *p = y; *gx = 0; *gy = 1; *gz = 0; return;
    case 2: *p = z; *gx = 0; *gy = 0; *gz = 1; return;
    case 3: *p = x; *gx = 1; *gy = 0; *gz = 0; return;
    case 4: *p = x * y; *gx = y; *gy = x; *gz = 0; return;
    case 5: *p = y * z; *gx = 0; *gy = z; *gz = y; return;
    case 6: *p = 2 * z2 - x2 - y2; *gx = -2 * x; *gy = -2 * y; *gz = 4 * z; return;
    case 7: *p = x * z; *gx = z; *gy = 0; *gz = x; return;
    case 8: *p = x2 - y2; *gx = 2 * x; *gy = -2 * y; *gz = 0; return;
    case 9: *p = 3 * x2 * y - y * y2; *gx = 6 * x * y; *gy = 3 * x2 - 3 * y2; *gz = 0; return;
    case 10: *p = x * y * z; *gx = y * z; *gy = x * z; *gz = x * y; return;
    case 11: *p = 4 * y * z2 - x2 * y - y * y2; *gx = -2 * x * y; *gy = 4 * z2 - x2 - 3 * y2; *gz = 8 * y * z; return;
    case 12: *p = 2 * z * z2 - 3 * x2 * z - 3 * y2 * z; *gx = -6 * x * z; *gy = -6 * y * z; *gz = 6 * z2 - 3 * x2 - 3 * y2; return;
    case 13: *p = 4 * x * z2 - x * x2 - x * y2; *gx = 4 * z2 - 3 * x2 - y2; *gy = -2 * x * y; *gz = 8 * x * z; return;
    case 14: *p = x2 * z - y2 * z; *gx = 2 * x * z; *gy = -2 * y * z; *gz = x2 - y2; return;
    case 15: *p = x * x2 - 3 * x * y2; *gx = 3 * x2 - 3 * y2; *gy = -6 * x * y; *gz = 0; return;
    case 16: *p = x * x2 * y - x * y * y2; *gx = 3 * x2 * y - y * y2; *gy = x * x2 - 3 * x * y2; *gz = 0; return;
    case 17: *p = 3 * x2 * y * z - y * y2 * z; *gx = 6 * x * y * z; *gy = 3 * x2 * z - 3 * y2 * z; *gz = 3 * x2 * y - y * y2; return;
    case 18: *p = 6 * x * y * z2 - x * x2 * y - x * y * y2;
      *gx = 6 * y * z2 - 3 * x2 * y - y * y2; *gy = 6 * x * z2 - x * x2 - 3 * x * y2; *gz = 12 * x * y * z; return;
    case 19: *p = 4 * y * z * z2 - 3 * x2 * y * z - 3 * y * y2 * z;
      *gx = -6 * x * y * z; *gy = 4 * z * z2 - 3 * x2 * z - 9 * y2 * z; *gz = 12 * y * z2 - 3 * x2 * y - 3 * y * y2; return;
    case 20: {
      const double q = x2 + y2;
      *p = 8 * z2 * z2 - 24 * z2 * q + 3 * q * q;
      *gx = -48 * x * z2 + 12 * x * q; *gy = -48 * y * z2 + 12 * y * q; *gz = 32 * z * z2 - 48 * z * q; return;
    }
    case 21: *p = 4 * x * z * z2 - 3 * x * x2 * z - 3 * x * y2 * z;
      *gx = 4 * z * z2 - 9 * x2 * z - 3 * y2 * z; *gy = -6 * x * y * z; *gz = 12 * x * z2 - 3 * x * x2 - 3 * x * y2; return;
    case 22: *p = 6 * x2 * z2 - 6 * y2 * z2 - x2 * x2 + y2 * y2;
      *gx = 12 * x * z2 - 4 * x * x2; *gy = -12 * y * z2 + 4 * y * y2; *gz = 12 * x2 * z - 12 * y2 * z; return;
    case 23: *p = x * x2 * z - 3 * x * y2 * z; *gx = 3 * x2 * z - 3 * y2 * z; *gy = -6 * x * y * z; *gz = x * x2 - 3 * x * y2; return;
    case 24: *p = x2 * x2 - 6 * x2 * y2 + y2 * y2; *gx = 4 * x * x2 - 12 * x * y2; *gy = -12 * x2 * y + 4 * y * y2; *gz = 0; return;
    default: *p = 0; *gx = *gy = *gz = 0; return;
  }
}

static double ycoef(int idx) {
  const double pi = 3.14159265358979323846;
  switch (idx) {
    case 0: return 0.5 / sqrt(pi);
    case 1: case 2: case 3: return 0.5 * sqrt(3.0 / pi);
    case 4: case 5: case 7: return 0.5 * sqrt(15.0 / pi);
    case 6: return 0.25 * sqrt(5.0 / pi);
    case 8: return 0.25 * sqrt(15.0 / pi);
    case 9: case 15: return 0.25 * sqrt(35.0 / (2.0 * pi));
    case 10: return 0.5 * sqrt(105.0 / pi);
    case 11: case 13: return 0.25 * sqrt(21.0 / (2.0 * pi));
    case 12: return 0.25 * sqrt(7.0 / pi);
    case 14: return 0.25 * sqrt(105.0 / pi);
    case 16: return 0.75 * sqrt(35.0 / pi);
    case 17: case 23: return 0.75 * sqrt(35.0 / (2.0 * pi));
    case 18: return 0.75 * sqrt(5.0 / pi);
    case 19: case 21: return 0.75 * sqrt(5.0 / (2.0 * pi));
    case 20: return 0.1875 / sqrt(pi);
    case 22: return 0.375 * sqrt(5.0 / pi);
    case 24: return 0.1875 * sqrt(35.0 / pi);
    default: return 0.0;
  }
}

static int l_of(int idx) { return idx < 1 ? 0 : idx < 4 ? 1 : idx < 9 ? 2 : idx < 16 ? 3 : 4; }

static double fact(int n) {
  double f = 1.0;
  for (int k = 2; k <= n; ++k) f *= k;
  return f;
}

static double binom(int n, int k) { return fact(n) / (fact(k) * fact(n - k)); }

/* l = 5, 6 from the closed form of the complex solid harmonic (Rodrigues'
 * formula for P_l differentiated m times, no Condon-Shortley phase):
 *   r^l P_l^m(cos t) e^{imp} = (x + iy)^m sum_k a_k z^(l-2k-m) r^(2k),
 *   a_k = 2^-l (-1)^k C(l,k) C(2l-2k,l) (l-2k)!/(l-2k-m)!,
 * real harmonics Y_l0 = N_l0 Re, (Y_l,m, Y_l,-m) = sqrt2 N_lm (Re, Im),
 * N_lm^2 = (2l+1)/(4 pi) (l-m)!/(l+m)!; divided by r^l with the quotient rule
 * for the gradient. */
static void solid_closed_form(int l, double x, double y, double z, double* Y, double* dY) {
  const double pi = 3.14159265358979323846;
  const double r2 = x * x + y * y + z * z, r = sqrt(r2);
  const double rl = pow(r, -l), drl = -l * rl / r2;
  for (int m = 0; m <= l; ++m) {
    /* w = (x + iy)^m and its gradient (m (x+iy)^(m-1) (1, i, 0)) */
    double wre = 1.0, wim = 0.0, pre = 1.0, pim = 0.0; /* p = (x+iy)^(m-1) */
    for (int k = 0; k < m; ++k) {
      pre = wre;
      pim = wim;
      const double a = wre * x - wim * y, b = wre * y + wim * x;
      wre = a;
      wim = b;
    }
    double gw_re[3] = {0, 0, 0}, gw_im[3] = {0, 0, 0};
    if (m > 0) {
      gw_re[0] = m * pre;  gw_im[0] = m * pim;
      gw_re[1] = -m * pim; gw_im[1] = m * pre;
    }
    double sv = 0.0, gs[3] = {0, 0, 0};
    for (int k = 0; 2 * k <= l - m; ++k) {
      const int e = l - 2 * k - m;
      const double a = ldexp(1.0, -l) * ((k & 1) ? -1.0 : 1.0) * binom(l, k) * binom(2 * l - 2 * k, l) *
                       fact(l - 2 * k) / fact(e);
      const double ze = pow(z, e), rk = pow(r2, k);
      sv += a * ze * rk;
      const double dze = e > 0 ? e * pow(z, e - 1) : 0.0;
      const double drk = k > 0 ? k * pow(r2, k - 1) : 0.0;
      gs[0] += a * ze * drk * 2.0 * x;
      gs[1] += a * ze * drk * 2.0 * y;
      gs[2] += a * (dze * rk + ze * drk * 2.0 * z);
    }
    double nrm = sqrt((2 * l + 1) / (4.0 * pi) * fact(l - m) / fact(l + m));
    if (m > 0) nrm *= sqrt(2.0);
    const double qre = wre * sv, qim = wim * sv;
    const double q[3] = {x, y, z};
    const int ip = l * l + l + m, in = l * l + l - m;
    Y[ip] = nrm * qre * rl;
    if (m > 0) Y[in] = nrm * qim * rl;
    if (dY) {
      for (int a = 0; a < 3; ++a) {
        const double gre = gw_re[a] * sv + wre * gs[a], gim = gw_im[a] * sv + wim * gs[a];
        dY[3 * ip + a] = nrm * (gre * rl + qre * drl * q[a]);
        if (m > 0) dY[3 * in + a] = nrm * (gim * rl + qim * drl * q[a]);
      }
    }
  }
}

/* Y[idx] and dY[3*idx+a] at displacement d (not normalised), l <= 6. */
void oracle_real_sh(int L, double x, double y, double z, double* Y, double* dY) {
  const double r2 = x * x + y * y + z * z;
  const double r = sqrt(r2);
  for (int l = 5; l <= L; ++l) solid_closed_form(l, x, y, z, Y, dY);
  const int C = (L < 4 ? (L + 1) * (L + 1) : 25);
  for (int idx = 0; idx < C; ++idx) {
    double p, gx, gy, gz;
    poly(idx, x, y, z, &p, &gx, &gy, &gz);
    const int l = l_of(idx);
    const double c = ycoef(idx);
    const double rl = pow(r, -l);
    Y[idx] = c * p * rl;
    if (dY) {
      const double dr = -l * rl / r2;  /* d(r^-l)/dx_a = -l r^(-l-2) x_a */
      dY[3 * idx + 0] = c * (gx * rl + p * dr * x);
      dY[3 * idx + 1] = c * (gy * rl + p * dr * y);
      dY[3 * idx + 2] = c * (gz * rl + p * dr * z);
    }
  }
}

/* R_mu and dR_mu/dr for one pair (FP64).  Chebyshev kinds
   (sus2_sh.cu:3171-3297): R = f sum_n c_n T_n(xi), xi = tanh(z) or
   z / sqrt(1 + z^2), z = scal (r - shift) / 2.  Laguerre kind
   (sus2_sh.cu:3299-3352): R = f exp(-u/2) sum_n c_n L_n(u),
   u = scal log(1 + r / rho), rho = max(shift, 1e-8).  f = s_pair (r - rc)^2. */
void oracle_radial(const OracleModel* m, int pair, double r, double* R, double* dR) {
  const double dr = r - m->rc;
  const double f = m->pscale[pair] * dr * dr;
  const double df = 2.0 * m->pscale[pair] * dr;
  double t[32], dt[32];
  for (int mu = 0; mu < m->kmu; ++mu) {
    const double sc = m->scal[pair * m->kmu + mu];
    const double sh = m->rshift[pair * m->kmu + mu];
    double x, dxdr, env = 1.0, denv = 0.0;
    if (m->kind == 2) {
      const double rho = sh > 1.0e-8 ? sh : 1.0e-8;
      x = sc * log1p(r / rho);
      dxdr = sc / (rho + r);
      env = exp(-0.5 * x);
      denv = -0.5 * dxdr * env;
      t[0] = 1.0;
      dt[0] = 0.0;
      if (m->rb > 1) {
        t[1] = 1.0 - x;
        dt[1] = -1.0;
      }
      for (int n = 1; n + 1 < m->rb; ++n) {
        t[n + 1] = ((2.0 * n + 1.0 - x) * t[n] - n * t[n - 1]) / (n + 1.0);
        dt[n + 1] = ((2.0 * n + 1.0 - x) * dt[n] - t[n] - n * dt[n - 1]) / (n + 1.0);
      }
    } else {
      const double z = 0.5 * sc * (r - sh);
      if (m->kind == 1) {
        const double q = 1.0 / sqrt(1.0 + z * z);
        x = z * q;
        dxdr = 0.5 * sc * q * q * q;
      } else {
        x = tanh(z);
        dxdr = 0.5 * sc * (1.0 - x * x);
      }
      t[0] = 1.0;
      dt[0] = 0.0;
      if (m->rb > 1) {
        t[1] = x;
        dt[1] = 1.0;
      }
      for (int n = 2; n < m->rb; ++n) {
        t[n] = 2.0 * x * t[n - 1] - t[n - 2];
        dt[n] = 2.0 * t[n - 1] + 2.0 * x * dt[n - 1] - dt[n - 2];
      }
    }
    double s = 0.0, sd = 0.0;
    for (int n = 0; n < m->rb; ++n) {
      s += m->radial[mu * m->rb + n] * t[n];
      sd += m->radial[mu * m->rb + n] * dt[n];
    }
    R[mu] = f * env * s;
    if (dR) dR[mu] = (df * env + f * denv) * s + f * env * sd * dxdr;
  }
}

/* ---- neighbours ---------------------------------------------------------- */
typedef struct {
  int j;
  double d[3];
} Edge;

typedef struct {
  double h[9], hinv[9];
  int pbc[3];
  int n[3];       /* cells */
  int reach[3];   /* image range for brute force */
  int use_cells;
} Geo;

static void inv3(const double* h, double* o) {
  const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
                     h[2] * (h[3] * h[7] - h[4] * h[6]);
  const double id = 1.0 / det;
  o[0] = (h[4] * h[8] - h[5] * h[7]) * id;
  o[1] = (h[2] * h[7] - h[1] * h[8]) * id;
  o[2] = (h[1] * h[5] - h[2] * h[4]) * id;
  o[3] = (h[5] * h[6] - h[3] * h[8]) * id;
  o[4] = (h[0] * h[8] - h[2] * h[6]) * id;
  o[5] = (h[2] * h[3] - h[0] * h[5]) * id;
  o[6] = (h[3] * h[7] - h[4] * h[6]) * id;
  o[7] = (h[1] * h[6] - h[0] * h[7]) * id;
  o[8] = (h[0] * h[4] - h[1] * h[3]) * id;
}

static void geo_init(Geo* g, const double* h, const int* pbc, double rc) {
  memcpy(g->h, h, sizeof(g->h));
  inv3(h, g->hinv);
  const double a[3] = {h[0], h[3], h[6]}, b[3] = {h[1], h[4], h[7]}, c[3] = {h[2], h[5], h[8]};
  const double* v[3][2] = {{b, c}, {c, a}, {a, b}};
  const double vol = fabs(a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
                          a[2] * (b[0] * c[1] - b[1] * c[0]));
  g->use_cells = 1;
  for (int d = 0; d < 3; ++d) {
    const double* u = v[d][0];
    const double* w = v[d][1];
    const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
    const double thick = vol / sqrt(cx * cx + cy * cy + cz * cz);
    g->pbc[d] = pbc[d] ? 1 : 0;
    g->reach[d] = g->pbc[d] ? (int)ceil(rc / thick) : 0;
    if (g->reach[d] < 1 && g->pbc[d]) g->reach[d] = 1;
    int n = (int)floor(thick / rc);
    if (n < 1) n = 1;
    if (n > 512) n = 512;
    g->n[d] = n;
    if (g->pbc[d] && n < 3) g->use_cells = 0;
  }
}

/* Collects the neighbours of every atom; returns per-atom arrays. */
typedef struct {
  int* start;  /* [N+1] */
  Edge* e;
} NList;

static void frac(const Geo* g, const double* p, double* s) {
  for (int a = 0; a < 3; ++a) s[a] = g->hinv[3 * a] * p[0] + g->hinv[3 * a + 1] * p[1] + g->hinv[3 * a + 2] * p[2];
}

static int build_nlist(const Geo* g, int N, const double* pos, double rc, NList* out) {
  const double rc2 = rc * rc;
  int* cnt = (int*)calloc((size_t)N + 1, sizeof(int));
  Edge** per = (Edge**)calloc((size_t)N, sizeof(Edge*));
  int* capv = (int*)calloc((size_t)N, sizeof(int));
  if (!cnt || !per || !capv) return -1;
  int ncell = 1, *cstart = NULL, *catoms = NULL, *cell_of = NULL;
  if (g->use_cells) {
    ncell = g->n[0] * g->n[1] * g->n[2];
    cstart = (int*)calloc((size_t)ncell + 1, sizeof(int));
    catoms = (int*)malloc(sizeof(int) * (size_t)N);
    cell_of = (int*)malloc(sizeof(int) * (size_t)N);
    for (int i = 0; i < N; ++i) {
      double p[3] = {pos[i], pos[i + N], pos[i + 2 * N]}, s[3];
      frac(g, p, s);
      int c[3];
      for (int a = 0; a < 3; ++a) {
        if (g->pbc[a]) s[a] -= floor(s[a]);
        c[a] = (int)floor(s[a] * g->n[a]);
        if (c[a] < 0) c[a] = 0;
        if (c[a] >= g->n[a]) c[a] = g->n[a] - 1;
      }
      cell_of[i] = (c[2] * g->n[1] + c[1]) * g->n[0] + c[0];
      cstart[cell_of[i] + 1]++;
    }
    for (int c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    int* fillp = (int*)malloc(sizeof(int) * (size_t)ncell);
    memcpy(fillp, cstart, sizeof(int) * (size_t)ncell);
    for (int i = 0; i < N; ++i) catoms[fillp[cell_of[i]]++] = i;
    free(fillp);
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < N; ++i) {
    const double pi[3] = {pos[i], pos[i + N], pos[i + 2 * N]};
    int k = 0, cap = 64;
    Edge* e = (Edge*)malloc(sizeof(Edge) * cap);
    if (g->use_cells) {
      /* wrapped fractional coordinate of i decides its cell; neighbours are
       * searched through the 27 surrounding cells with explicit images */
      double s[3];
      frac(g, pi, s);
      int ci[3];
      double wi[3];
      for (int a = 0; a < 3; ++a) {
        wi[a] = g->pbc[a] ? floor(s[a]) : 0.0;
        double t = s[a] - wi[a];
        ci[a] = (int)floor(t * g->n[a]);
        if (ci[a] < 0) ci[a] = 0;
        if (ci[a] >= g->n[a]) ci[a] = g->n[a] - 1;
      }
      for (int oz = -1; oz <= 1; ++oz)
        for (int oy = -1; oy <= 1; ++oy)
          for (int ox = -1; ox <= 1; ++ox) {
            int o[3] = {ox, oy, oz}, cc[3], sh[3];
            int skip = 0;
            for (int a = 0; a < 3; ++a) {
              int v = ci[a] + o[a];
              sh[a] = 0;
              if (g->pbc[a]) {
                if (v < 0) { v += g->n[a]; sh[a] = -1; }
                else if (v >= g->n[a]) { v -= g->n[a]; sh[a] = 1; }
              } else if (v < 0 || v >= g->n[a]) {
                skip = 1;
              }
              cc[a] = v;
            }
            if (skip) continue;
            const int c = (cc[2] * g->n[1] + cc[1]) * g->n[0] + cc[0];
            for (int q = cstart[c]; q < cstart[c + 1]; ++q) {
              const int j = catoms[q];
              const double pj[3] = {pos[j], pos[j + N], pos[j + 2 * N]};
              double sj[3];
              frac(g, pj, sj);
              double t[3];
              for (int a = 0; a < 3; ++a) {
                const double wj = g->pbc[a] ? floor(sj[a]) : 0.0;
                /* image of j: wrapped j shifted by the cell-wrap, relative to wrapped i */
                t[a] = (double)sh[a] - wj + wi[a];
              }
              double d[3];
              for (int a = 0; a < 3; ++a)
                d[a] = pj[a] - pi[a] + g->h[3 * a] * t[0] + g->h[3 * a + 1] * t[1] + g->h[3 * a + 2] * t[2];
              if (j == i && t[0] == 0 && t[1] == 0 && t[2] == 0) continue;
              const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
              if (r2 < rc2) {
                if (k == cap) { cap *= 2; e = (Edge*)realloc(e, sizeof(Edge) * cap); }
                e[k].j = j;
                e[k].d[0] = d[0]; e[k].d[1] = d[1]; e[k].d[2] = d[2];
                ++k;
              }
            }
          }
    } else {
      for (int j = 0; j < N; ++j) {
        const double d0[3] = {pos[j] - pi[0], pos[j + N] - pi[1], pos[j + 2 * N] - pi[2]};
        for (int tx = -g->reach[0]; tx <= g->reach[0]; ++tx)
          for (int ty = -g->reach[1]; ty <= g->reach[1]; ++ty)
            for (int tz = -g->reach[2]; tz <= g->reach[2]; ++tz) {
              if (j == i && tx == 0 && ty == 0 && tz == 0) continue;
              double d[3];
              for (int a = 0; a < 3; ++a)
                d[a] = d0[a] + g->h[3 * a] * tx + g->h[3 * a + 1] * ty + g->h[3 * a + 2] * tz;
              const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
              if (r2 < rc2) {
                if (k == cap) { cap *= 2; e = (Edge*)realloc(e, sizeof(Edge) * cap); }
                e[k].j = j;
                e[k].d[0] = d[0]; e[k].d[1] = d[1]; e[k].d[2] = d[2];
                ++k;
              }
            }
      }
    }
    per[i] = e;
    capv[i] = k;
  }
  out->start = (int*)malloc(sizeof(int) * ((size_t)N + 1));
  out->start[0] = 0;
  for (int i = 0; i < N; ++i) out->start[i + 1] = out->start[i] + capv[i];
  out->e = (Edge*)malloc(sizeof(Edge) * ((size_t)out->start[N] + 1));
  for (int i = 0; i < N; ++i) {
    memcpy(out->e + out->start[i], per[i], sizeof(Edge) * (size_t)capv[i]);
    free(per[i]);
  }
  free(per);
  free(capv);
  free(cnt);
  free(cstart);
  free(catoms);
  free(cell_of);
  return 0;
}

/* ---- energy / forces / virial -------------------------------------------- */
/* center (optional): only atoms with center[i] != 0 are centres: their site
   energies, the forces of those energies on every atom, and their virials;
   the other atoms (ghosts of a spatial decomposition) get pe = vir = 0. */
int oracle_efs_centers(const OracleModel* m, int N, const double* h, const int* pbc, const int* type,
                       const double* pos, const unsigned char* center, double* pe, double* f, double* vir,
                       int nthreads);

int oracle_efs(const OracleModel* m, int N, const double* h, const int* pbc, const int* type,
               const double* pos, double* pe, double* f, double* vir, int nthreads) {
  return oracle_efs_centers(m, N, h, pbc, type, pos, NULL, pe, f, vir, nthreads);
}

int oracle_efs_centers(const OracleModel* m, int N, const double* h, const int* pbc, const int* type,
                       const double* pos, const unsigned char* center, double* pe, double* f, double* vir,
                       int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int nt = omp_get_max_threads();
#else
  (void)nthreads;
  const int nt = 1;
#endif
  Geo g;
  geo_init(&g, h, pbc, m->rc);
  NList nl;
  if (build_nlist(&g, N, pos, m->rc, &nl) != 0) return -1;
  double* fbuf = (double*)calloc((size_t)nt * 3 * N, sizeof(double));
  if (!fbuf) return -1;
  const int C = (m->L + 1) * (m->L + 1);
#pragma omp parallel
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
    double* fl = fbuf + (size_t)tid * 3 * N;
    double* Mv = (double*)malloc(sizeof(double) * m->M);
    double* gv = (double*)malloc(sizeof(double) * m->M);
    double R[64], dR[64], Y[49], dY[147];
#pragma omp for schedule(dynamic, 32)
    for (int i = 0; i < N; ++i) {
      const int ti = type[i];
      if (center && !center[i]) {
        pe[i] = 0.0;
        for (int k = 0; k < 9; ++k) vir[(size_t)k * N + i] = 0.0;
        continue;
      }
      memset(Mv, 0, sizeof(double) * m->M);
      for (int q = nl.start[i]; q < nl.start[i + 1]; ++q) {
        const Edge* e = nl.e + q;
        const double r = sqrt(e->d[0] * e->d[0] + e->d[1] * e->d[1] + e->d[2] * e->d[2]);
        oracle_radial(m, ti * m->S + type[e->j], r, R, NULL);
        oracle_real_sh(m->L, e->d[0], e->d[1], e->d[2], Y, NULL);
        for (int b = 0; b < m->nbasic; ++b) Mv[b] += R[m->basic_mu[b]] * Y[m->basic_y[b]];
      }
      for (int p = 0; p < m->nprod; ++p) Mv[m->prod_t[p]] += m->prod_c[p] * Mv[m->prod_l[p]] * Mv[m->prod_r[p]];
      const double ct = m->species[ti];
      double E = m->shift_e[ti] + ct;
      memset(gv, 0, sizeof(double) * m->M);
      for (int s = 0; s < m->nscalar; ++s) {
        E += ct * m->w[s] * Mv[m->map[s]];
        gv[m->map[s]] += ct * m->w[s];
      }
      pe[i] = E;
      for (int p = m->nprod - 1; p >= 0; --p) {
        const double gt = gv[m->prod_t[p]] * m->prod_c[p];
        gv[m->prod_l[p]] += gt * Mv[m->prod_r[p]];
        gv[m->prod_r[p]] += gt * Mv[m->prod_l[p]];
      }
      double w9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int q = nl.start[i]; q < nl.start[i + 1]; ++q) {
        const Edge* e = nl.e + q;
        const double dx = e->d[0], dy = e->d[1], dz = e->d[2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        oracle_radial(m, ti * m->S + type[e->j], r, R, dR);
        oracle_real_sh(m->L, dx, dy, dz, Y, dY);
        double ex = 0, ey = 0, ez = 0;
        for (int b = 0; b < m->nbasic; ++b) {
          const double a = gv[b];
          if (a == 0.0) continue;
          const int mu = m->basic_mu[b], y = m->basic_y[b];
          ex += a * (dR[mu] * dx / r * Y[y] + R[mu] * dY[3 * y + 0]);
          ey += a * (dR[mu] * dy / r * Y[y] + R[mu] * dY[3 * y + 1]);
          ez += a * (dR[mu] * dz / r * Y[y] + R[mu] * dY[3 * y + 2]);
        }
        fl[i] += ex;
        fl[i + N] += ey;
        fl[i + 2 * N] += ez;
        fl[e->j] -= ex;
        fl[e->j + N] -= ey;
        fl[e->j + 2 * N] -= ez;
        w9[0] -= dx * ex;
        w9[1] -= dy * ey;
        w9[2] -= dz * ez;
        w9[3] -= dx * ey;
        w9[4] -= dx * ez;
        w9[5] -= dy * ez;
        w9[6] -= dy * ex;
        w9[7] -= dz * ex;
        w9[8] -= dz * ey;
      }
      for (int k = 0; k < 9; ++k) vir[(size_t)k * N + i] = w9[k];
    }
    free(Mv);
    free(gv);
  }
  for (int a = 0; a < 3 * N; ++a) {
    double s = 0.0;
    for (int t = 0; t < nt; ++t) s += fbuf[(size_t)t * 3 * N + a];
    f[a] = s;
  }
  (void)C;
  free(fbuf);
  free(nl.start);
  free(nl.e);
  return 0;
}

/* Basic moments only (for kernel-level parity checks): B[b*N+i]. */
int oracle_basics(const OracleModel* m, int N, const double* h, const int* pbc, const int* type,
                  const double* pos, double* B, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  Geo g;
  geo_init(&g, h, pbc, m->rc);
  NList nl;
  if (build_nlist(&g, N, pos, m->rc, &nl) != 0) return -1;
#pragma omp parallel for schedule(dynamic, 32)
  for (int i = 0; i < N; ++i) {
    double R[64], Y[49];
    for (int b = 0; b < m->nbasic; ++b) B[(size_t)b * N + i] = 0.0;
    for (int q = nl.start[i]; q < nl.start[i + 1]; ++q) {
      const Edge* e = nl.e + q;
      const double r = sqrt(e->d[0] * e->d[0] + e->d[1] * e->d[1] + e->d[2] * e->d[2]);
      oracle_radial(m, type[i] * m->S + type[e->j], r, R, NULL);
      oracle_real_sh(m->L, e->d[0], e->d[1], e->d[2], Y, NULL);
      for (int b = 0; b < m->nbasic; ++b) B[(size_t)b * N + i] += R[m->basic_mu[b]] * Y[m->basic_y[b]];
    }
  }
  free(nl.start);
  free(nl.e);
  return 0;
}

/* Neighbour count per atom within rc (for neighbour-list parity). */
int oracle_neighbor_counts(int N, const double* h, const int* pbc, const double* pos, double rc, int* counts) {
  Geo g;
  geo_init(&g, h, pbc, rc);
  NList nl;
  if (build_nlist(&g, N, pos, rc, &nl) != 0) return -1;
  for (int i = 0; i < N; ++i) counts[i] = nl.start[i + 1] - nl.start[i];
  free(nl.start);
  free(nl.e);
  return 0;
}

/* Site energies and basic-moment adjoints dE_i/dB_b(i) from given basics
 * B[b*N+i] (flat products, sus2_sh.cu:4813-4845); G[b*N+i] assigned. */
int oracle_cg_energy(const OracleModel* m, int N, const int* type, const double* B, double* pe, double* G) {
  int fail = 0;
#pragma omp parallel
  {
    double* Mv = (double*)malloc(sizeof(double) * m->M);
    double* gv = (double*)malloc(sizeof(double) * m->M);
    if (!Mv || !gv) fail = 1;
#pragma omp for schedule(static)
    for (int i = 0; i < N; ++i) {
      if (!Mv || !gv) continue;
      memset(Mv, 0, sizeof(double) * m->M);
      memset(gv, 0, sizeof(double) * m->M);
      for (int b = 0; b < m->nbasic; ++b) Mv[b] = B[(size_t)b * N + i];
      for (int p = 0; p < m->nprod; ++p) Mv[m->prod_t[p]] += m->prod_c[p] * Mv[m->prod_l[p]] * Mv[m->prod_r[p]];
      const int ti = type[i];
      const double ct = m->species[ti];
      double E = m->shift_e[ti] + ct;
      for (int s = 0; s < m->nscalar; ++s) {
        E += ct * m->w[s] * Mv[m->map[s]];
        gv[m->map[s]] += ct * m->w[s];
      }
      for (int p = m->nprod - 1; p >= 0; --p) {
        const double gt = gv[m->prod_t[p]] * m->prod_c[p];
        gv[m->prod_l[p]] += gt * Mv[m->prod_r[p]];
        gv[m->prod_r[p]] += gt * Mv[m->prod_l[p]];
      }
      pe[i] = E;
      for (int b = 0; b < m->nbasic; ++b) G[(size_t)b * N + i] = gv[b];
    }
    free(Mv);
    free(gv);
  }
  return fail ? -1 : 0;
}

/* ---- ZBL short-range term ------------------------------------------------
 * Restates src/force/sus2_zbl_common.cuh:18-225 (pair function, covalent
 * radii, pair cutoff tables) and gpu_sh_apply_zbl (sus2_sh.cu:7522-7627):
 * every listed pair with r < outer(ti,tj) puts E/2 on atom i, dE = E'/2 d/r,
 * F_i += dE, F_j -= dE, W_i -= d (x) dE.  Outputs are accumulated (+=) onto
 * the SUS2 outputs of oracle_efs.  Test infrastructure only.               */

static const double kOracleCovalent[94] = {
    0.426667, 0.613333, 1.6,      1.25333,  1.02667,  1.0,      0.946667, 0.84,     0.853333, 0.893333,
    1.86667,  1.66667,  1.50667,  1.38667,  1.46667,  1.36,     1.32,     1.28,     2.34667,  2.05333,
    1.77333,  1.62667,  1.61333,  1.46667,  1.42667,  1.38667,  1.33333,  1.32,     1.34667,  1.45333,
    1.49333,  1.45333,  1.53333,  1.46667,  1.52,     1.56,     2.52,     2.22667,  1.96,     1.85333,
    1.76,     1.65333,  1.53333,  1.50667,  1.50667,  1.44,     1.53333,  1.64,     1.70667,  1.68,
    1.68,     1.64,     1.76,     1.74667,  2.78667,  2.34667,  2.16,     1.96,     2.10667,  2.09333,
    2.08,     2.06667,  2.01333,  2.02667,  2.01333,  2.0,      1.98667,  1.98667,  1.97333,  2.04,
    1.94667,  1.82667,  1.74667,  1.64,     1.57333,  1.54667,  1.48,     1.49333,  1.50667,  1.76,
    1.73333,  1.73333,  1.81333,  1.74667,  1.84,     1.89333,  2.68,     2.41333,  2.22667,  2.10667,
    2.02667,  2.04,     2.05333,  2.06667};

double oracle_zbl_covalent_radius(int z) { return (z >= 1 && z <= 94) ? kOracleCovalent[z - 1] : 0.0; }

/* Energy and dE/dr of one pair (screened Coulomb, four-exponential universal
 * screening, cosine switch between inner and outer). */
void oracle_zbl_pair(int zi, int zj, double r, double inner, double outer, double* e, double* de) {
  *e = 0.0;
  *de = 0.0;
  if (zi <= 0 || zj <= 0 || r <= 0.0 || outer <= 0.0 || r >= outer) return;
  static const double amp[4] = {0.18175, 0.50986, 0.28022, 0.02817};
  static const double rate[4] = {3.1998, 0.94229, 0.4029, 0.20162};
  const double ainv = 2.134563 * (pow((double)zi, 0.23) + pow((double)zj, 0.23));
  const double x = ainv * r;
  double phi = 0.0, dphi = 0.0;
  for (int q = 0; q < 4; ++q) {
    const double ex = exp(-rate[q] * x);
    phi += amp[q] * ex;
    dphi -= amp[q] * rate[q] * ainv * ex;
  }
  const double k = 14.3996454784255 * (double)zi * (double)zj;
  const double e0 = k * phi / r, de0 = k * (dphi / r - phi / (r * r));
  double s = 1.0, ds = 0.0;
  if (r > inner) {
    const double w = 3.141592653589793238462643383279502884 / (outer - inner);
    s = 0.5 * cos(w * (r - inner)) + 0.5;
    ds = -0.5 * w * sin(w * (r - inner));
  }
  *e = s * e0;
  *de = s * de0 + ds * e0;
}

/* Per species pair cutoffs [S*S]; 0 on success, else a code naming the
 * failed check (1 no species, 2 inner < 0, 3 outer <= 0, 4 factor < 0.5,
 * 5 outer <= inner, 6 atomic number out of range, 7 pair inner >= outer). */
int oracle_zbl_tables(int S, const int* z, double inner, double outer, int typewise, double factor, double* pin,
                      double* pout) {
  if (S <= 0) return 1;
  if (inner < 0.0) return 2;
  if (outer <= 0.0) return 3;
  if (typewise) {
    if (factor < 0.5) return 4;
  } else if (outer <= inner) {
    return 5;
  }
  for (int a = 0; a < S; ++a)
    for (int b = 0; b < S; ++b) {
      const double ra = oracle_zbl_covalent_radius(z[a]), rb = oracle_zbl_covalent_radius(z[b]);
      if (z[a] <= 0 || z[b] <= 0 || (typewise && (ra <= 0.0 || rb <= 0.0))) return 6;
      double lo = inner, hi = outer;
      if (typewise) {
        lo = 0.0;
        hi = factor * (ra + rb);
        if (hi > outer) hi = outer;
      }
      if (hi <= lo) return 7;
      pin[a * S + b] = lo;
      pout[a * S + b] = hi;
    }
  return 0;
}

int oracle_zbl_efs(int S, const int* z, const double* pin, const double* pout, int N, const double* h,
                   const int* pbc, const int* type, const double* pos, double* pe, double* f, double* vir,
                   int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int nt = omp_get_max_threads();
#else
  (void)nthreads;
  const int nt = 1;
#endif
  double rmax = 0.0;
  for (int p = 0; p < S * S; ++p)
    if (pout[p] > rmax) rmax = pout[p];
  if (rmax <= 0.0) return -1;
  Geo g;
  geo_init(&g, h, pbc, rmax);
  NList nl;
  if (build_nlist(&g, N, pos, rmax, &nl) != 0) return -1;
  double* fbuf = (double*)calloc((size_t)nt * 3 * N, sizeof(double));
  if (!fbuf) return -1;
#pragma omp parallel
  {
#ifdef _OPENMP
    double* fl = fbuf + (size_t)omp_get_thread_num() * 3 * N;
#else
    double* fl = fbuf;
#endif
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < N; ++i) {
      const int ti = type[i];
      double e = 0.0, w9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int q = nl.start[i]; q < nl.start[i + 1]; ++q) {
        const Edge* ed = nl.e + q;
        const int p = ti * S + type[ed->j];
        const double dx = ed->d[0], dy = ed->d[1], dz = ed->d[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 <= 0.0 || r2 >= pout[p] * pout[p]) continue;
        const double r = sqrt(r2);
        double v, dv;
        oracle_zbl_pair(z[ti], z[type[ed->j]], r, pin[p], pout[p], &v, &dv);
        e += 0.5 * v;
        const double c = 0.5 * dv / r;
        const double ex = c * dx, ey = c * dy, ez = c * dz;
        fl[i] += ex;
        fl[i + N] += ey;
        fl[i + 2 * N] += ez;
        fl[ed->j] -= ex;
        fl[ed->j + N] -= ey;
        fl[ed->j + 2 * N] -= ez;
        w9[0] -= dx * ex;
        w9[1] -= dy * ey;
        w9[2] -= dz * ez;
        w9[3] -= dx * ey;
        w9[4] -= dx * ez;
        w9[5] -= dy * ez;
        w9[6] -= dy * ex;
        w9[7] -= dz * ex;
        w9[8] -= dz * ey;
      }
      pe[i] += e;
      for (int k = 0; k < 9; ++k) vir[(size_t)k * N + i] += w9[k];
    }
  }
  for (int a = 0; a < 3 * N; ++a) {
    double s = 0.0;
    for (int t = 0; t < nt; ++t) s += fbuf[(size_t)t * 3 * N + a];
    f[a] += s;
  }
  free(fbuf);
  free(nl.start);
  free(nl.e);
  return 0;
}

/* ---- two-layer mu-body gate ---------------------------------------------
 * Restates the gate path of SUS2_SH::compute (sus2_sh.cu:9821-10120) in its
 * plain form: first-layer moments Mg from the gate radial coefficients and
 * every product; signals h_mu (mu-body-linear-combo: b_p = sum_{body(q)=p}
 * w_q s_q, h_mu = sum_p c_{mu,p} b_p; mu-scalar-full: h_mu = sum_q W_{mu,q}
 * s_q); G = 1 + A tanh(a_t h), D = A a_t (1 - tanh^2) per atom (:4565-4662);
 * main moments with R_mu(r_ij) G_{j,mu} (:4247-4314); forces from the main
 * adjoints with G_j, dE/dh_{j,mu} += D_{j,mu} R_mu sum g Y (:6077-6121);
 * seeds and reverse products on Mg (:4664-4727); first-layer forces with the
 * gate radial coefficients (:6695-6790).  Outputs assigned.                */
typedef struct {
  int mode;               /* 1 mu-body-linear-combo, 2 mu-scalar-full */
  int nbody, nq;
  double amplitude;
  const double* radial;   /* [kmu][rb] */
  const double* additive; /* [S] */
  const int* q_moment;    /* [nq] */
  const int* q_body;      /* [nq] */
  const double* weights;  /* full [kmu][nq]; combo [nq] */
  const double* body_mix; /* combo [kmu][nbody] */
} OracleGate;

static void moments_of_atom(const OracleModel* m, const NList* nl, int i, const int* type, const double* gmul,
                            double* Mv) {
  double R[64], Y[49];
  const int ti = type[i];
  memset(Mv, 0, sizeof(double) * m->M);
  for (int q = nl->start[i]; q < nl->start[i + 1]; ++q) {
    const Edge* e = nl->e + q;
    const double r = sqrt(e->d[0] * e->d[0] + e->d[1] * e->d[1] + e->d[2] * e->d[2]);
    oracle_radial(m, ti * m->S + type[e->j], r, R, NULL);
    if (gmul)
      for (int mu = 0; mu < m->kmu; ++mu) R[mu] *= gmul[(size_t)e->j * m->kmu + mu];
    oracle_real_sh(m->L, e->d[0], e->d[1], e->d[2], Y, NULL);
    for (int b = 0; b < m->nbasic; ++b) Mv[b] += R[m->basic_mu[b]] * Y[m->basic_y[b]];
  }
  for (int p = 0; p < m->nprod; ++p) Mv[m->prod_t[p]] += m->prod_c[p] * Mv[m->prod_l[p]] * Mv[m->prod_r[p]];
}

/* Edge forces of basic adjoints gb on atom i (radial of model m, optional
 * gate multipliers of the neighbour and dE/dh accumulation). */
static void edge_forces(const OracleModel* m, const NList* nl, int i, int N, const int* type, const double* gb,
                        const double* gmul, const double* gder, double* adjh, double* fl, double* vir) {
  double R[64], dR[64], Y[49], dY[147];
  const int ti = type[i];
  double w9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int q = nl->start[i]; q < nl->start[i + 1]; ++q) {
    const Edge* e = nl->e + q;
    const double dx = e->d[0], dy = e->d[1], dz = e->d[2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    oracle_radial(m, ti * m->S + type[e->j], r, R, dR);
    oracle_real_sh(m->L, dx, dy, dz, Y, dY);
    if (adjh) {
      for (int b = 0; b < m->nbasic; ++b) {
        const int mu = m->basic_mu[b];
        adjh[(size_t)e->j * m->kmu + mu] += gb[b] * R[mu] * Y[m->basic_y[b]] * gder[(size_t)e->j * m->kmu + mu];
      }
    }
    double ex = 0, ey = 0, ez = 0;
    for (int b = 0; b < m->nbasic; ++b) {
      const int mu = m->basic_mu[b], y = m->basic_y[b];
      const double a = gb[b] * (gmul ? gmul[(size_t)e->j * m->kmu + mu] : 1.0);
      if (a == 0.0) continue;
      ex += a * (dR[mu] * dx / r * Y[y] + R[mu] * dY[3 * y + 0]);
      ey += a * (dR[mu] * dy / r * Y[y] + R[mu] * dY[3 * y + 1]);
      ez += a * (dR[mu] * dz / r * Y[y] + R[mu] * dY[3 * y + 2]);
    }
    fl[i] += ex;
    fl[i + N] += ey;
    fl[i + 2 * N] += ez;
    fl[e->j] -= ex;
    fl[e->j + N] -= ey;
    fl[e->j + 2 * N] -= ez;
    w9[0] -= dx * ex;
    w9[1] -= dy * ey;
    w9[2] -= dz * ez;
    w9[3] -= dx * ey;
    w9[4] -= dx * ez;
    w9[5] -= dy * ez;
    w9[6] -= dy * ex;
    w9[7] -= dz * ex;
    w9[8] -= dz * ey;
  }
  for (int k = 0; k < 9; ++k) vir[(size_t)k * N + i] += w9[k];
}

int oracle_efs_gate(const OracleModel* m, const OracleGate* g, int N, const double* h, const int* pbc,
                    const int* type, const double* pos, double* pe, double* f, double* vir, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int nt = omp_get_max_threads();
#else
  (void)nthreads;
  const int nt = 1;
#endif
  const int K = m->kmu;
  Geo geo;
  geo_init(&geo, h, pbc, m->rc);
  NList nl;
  if (build_nlist(&geo, N, pos, m->rc, &nl) != 0) return -1;
  OracleModel mg = *m;
  mg.radial = g->radial;
  double* Mg = (double*)malloc(sizeof(double) * (size_t)N * m->M);
  double* gmul = (double*)malloc(sizeof(double) * (size_t)N * K);
  double* gder = (double*)malloc(sizeof(double) * (size_t)N * K);
  double* gmain = (double*)malloc(sizeof(double) * (size_t)N * m->nbasic);
  double* gfirst = (double*)malloc(sizeof(double) * (size_t)N * m->nbasic);
  double* adjh_t = (double*)calloc((size_t)nt * N * K, sizeof(double));
  double* fbuf = (double*)calloc((size_t)nt * 3 * N, sizeof(double));
  if (!Mg || !gmul || !gder || !gmain || !gfirst || !adjh_t || !fbuf) return -1;
  memset(vir, 0, sizeof(double) * 9 * (size_t)N);
  /* 1. first layer: moments, signals, multipliers */
#pragma omp parallel for schedule(dynamic, 32)
  for (int i = 0; i < N; ++i) {
    double* Mv = Mg + (size_t)i * m->M;
    moments_of_atom(&mg, &nl, i, type, NULL, Mv);
    double hmu[64], body[64];
    if (g->mode == 1) {
      for (int b = 0; b < g->nbody; ++b) body[b] = 0.0;
      for (int q = 0; q < g->nq; ++q) body[g->q_body[q]] += g->weights[q] * Mv[g->q_moment[q]];
      for (int mu = 0; mu < K; ++mu) {
        hmu[mu] = 0.0;
        for (int b = 0; b < g->nbody; ++b) hmu[mu] += g->body_mix[mu * g->nbody + b] * body[b];
      }
    } else {
      for (int mu = 0; mu < K; ++mu) {
        hmu[mu] = 0.0;
        for (int q = 0; q < g->nq; ++q) hmu[mu] += g->weights[mu * g->nq + q] * Mv[g->q_moment[q]];
      }
    }
    const double a = g->additive[type[i]];
    for (int mu = 0; mu < K; ++mu) {
      const double th = tanh(a * hmu[mu]);
      gmul[(size_t)i * K + mu] = 1.0 + g->amplitude * th;
      gder[(size_t)i * K + mu] = g->amplitude * a * (1.0 - th * th);
    }
  }
  /* 2. main layer: energies and basic adjoints */
#pragma omp parallel
  {
    double* Mv = (double*)malloc(sizeof(double) * m->M);
    double* gv = (double*)malloc(sizeof(double) * m->M);
#pragma omp for schedule(dynamic, 32)
    for (int i = 0; i < N; ++i) {
      moments_of_atom(m, &nl, i, type, gmul, Mv);
      const int ti = type[i];
      const double ct = m->species[ti];
      double E = m->shift_e[ti] + ct;
      memset(gv, 0, sizeof(double) * m->M);
      for (int s = 0; s < m->nscalar; ++s) {
        E += ct * m->w[s] * Mv[m->map[s]];
        gv[m->map[s]] += ct * m->w[s];
      }
      pe[i] = E;
      for (int p = m->nprod - 1; p >= 0; --p) {
        const double gt = gv[m->prod_t[p]] * m->prod_c[p];
        gv[m->prod_l[p]] += gt * Mv[m->prod_r[p]];
        gv[m->prod_r[p]] += gt * Mv[m->prod_l[p]];
      }
      memcpy(gmain + (size_t)i * m->nbasic, gv, sizeof(double) * m->nbasic);
    }
    free(Mv);
    free(gv);
  }
  /* 3. main forces with gate multipliers; dE/dh per thread */
#pragma omp parallel
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
#pragma omp for schedule(dynamic, 32)
    for (int i = 0; i < N; ++i)
      edge_forces(m, &nl, i, N, type, gmain + (size_t)i * m->nbasic, gmul, gder, adjh_t + (size_t)tid * N * K,
                  fbuf + (size_t)tid * 3 * N, vir);
  }
  for (size_t a = 0; a < (size_t)N * K; ++a)
    for (int t = 1; t < nt; ++t) adjh_t[a] += adjh_t[(size_t)t * N * K + a];
  /* 4. seeds and reverse products on the first layer */
#pragma omp parallel
  {
    double* gv = (double*)malloc(sizeof(double) * m->M);
#pragma omp for schedule(dynamic, 32)
    for (int i = 0; i < N; ++i) {
      const double* Mv = Mg + (size_t)i * m->M;
      const double* adj = adjh_t + (size_t)i * K;
      memset(gv, 0, sizeof(double) * m->M);
      if (g->mode == 1) {
        double body[64];
        for (int b = 0; b < g->nbody; ++b) {
          body[b] = 0.0;
          for (int mu = 0; mu < K; ++mu) body[b] += adj[mu] * g->body_mix[mu * g->nbody + b];
        }
        for (int q = 0; q < g->nq; ++q) gv[g->q_moment[q]] += body[g->q_body[q]] * g->weights[q];
      } else {
        for (int q = 0; q < g->nq; ++q) {
          double seed = 0.0;
          for (int mu = 0; mu < K; ++mu) seed += adj[mu] * g->weights[mu * g->nq + q];
          gv[g->q_moment[q]] += seed;
        }
      }
      for (int p = m->nprod - 1; p >= 0; --p) {
        const double gt = gv[m->prod_t[p]] * m->prod_c[p];
        gv[m->prod_l[p]] += gt * Mv[m->prod_r[p]];
        gv[m->prod_r[p]] += gt * Mv[m->prod_l[p]];
      }
      memcpy(gfirst + (size_t)i * m->nbasic, gv, sizeof(double) * m->nbasic);
    }
    free(gv);
  }
  /* 5. first-layer forces */
#pragma omp parallel
  {
#ifdef _OPENMP
    const int tid = omp_get_thread_num();
#else
    const int tid = 0;
#endif
#pragma omp for schedule(dynamic, 32)
    for (int i = 0; i < N; ++i)
      edge_forces(&mg, &nl, i, N, type, gfirst + (size_t)i * m->nbasic, NULL, NULL, NULL,
                  fbuf + (size_t)tid * 3 * N, vir);
  }
  for (int a = 0; a < 3 * N; ++a) {
    double s = 0.0;
    for (int t = 0; t < nt; ++t) s += fbuf[(size_t)t * 3 * N + a];
    f[a] = s;
  }
  free(Mg);
  free(gmul);
  free(gder);
  free(gmain);
  free(gfirst);
  free(adjh_t);
  free(fbuf);
  free(nl.start);
  free(nl.e);
  return 0;
}
