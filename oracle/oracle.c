/* CPU oracle: plain-C restatement of ExaHyPE's generic nonlinear ADER-DG kernels.
 * TEST INFRASTRUCTURE ONLY (see oracle.h). Every function names the reference code it restates;
 * paths are relative to the ExaHyPE-Engine checkout.
 */
#include "oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXN 16
#define MAXV 16

/* ------------------------------------------------------------------------------------------ */
/* DG operator tables                                                                          */
/* Maths: Miscellaneous/aderdg/aderdg.py:14-195 (BaseFunc1d, assembleStiffnessMatrix, K1, dudx) */
/* and generateLookupTable.py:146-182; evaluated here in long double.                          */
/* ------------------------------------------------------------------------------------------ */

static long double legendre_p(int n, long double x, long double* dp) {
  long double p0 = 1.0L, p1 = x;
  if (n == 0) { *dp = 0.0L; return 1.0L; }
  for (int k = 2; k <= n; k++) {
    long double p2 = ((2.0L * k - 1.0L) * x * p1 - (k - 1.0L) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  *dp = n * (x * p1 - p0) / (x * x - 1.0L);
  return p1;
}

/* Gauss-Legendre nodes/weights on [0,1], ascending (generated/GaussLegendreBasis.csnippet order). */
static void gauss_legendre(int n, long double* x, long double* w) {
  for (int i = 0; i < n; i++) {
    long double r = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (n + 0.5L));
    long double dp = 0;
    for (int it = 0; it < 100; it++) {
      long double p = legendre_p(n, r, &dp);
      long double dr = p / dp;
      r -= dr;
      if (fabsl(dr) < 1e-22L) break;
    }
    legendre_p(n, r, &dp);
    long double wi = 2.0L / ((1.0L - r * r) * dp * dp);
    /* r descends with i, so x = (1-r)/2 ascends on [0,1] */
    x[i] = 0.5L * (1.0L - r);
    w[i] = 0.5L * wi;
  }
  if (n == 1) { x[0] = 0.5L; w[0] = 1.0L; }
}

/* Lagrange basis phi_m(xi) and phi_m'(xi) on nodes xin (aderdg.py:14-51). */
static void base_func(int n, const long double* xin, long double xi, long double* phi, long double* dphi) {
  for (int m = 0; m < n; m++) {
    phi[m] = 1.0L;
    dphi[m] = 0.0L;
    for (int j = 0; j < n; j++)
      if (j != m) phi[m] *= (xi - xin[j]) / (xin[m] - xin[j]);
    for (int i = 0; i < n; i++) {
      if (i == m) continue;
      long double tmp = 1.0L;
      for (int j = 0; j < n; j++) {
        if (j == i || j == m) continue;
        tmp *= (xi - xin[j]) / (xin[m] - xin[j]);
      }
      dphi[m] += tmp / (xin[m] - xin[i]);
    }
  }
}

int exo_tables(int order, double* nodes, double* weights, double* Kxi, double* iK1, double* dudx, double* F0,
               double* F1) {
  const int n = order + 1;
  if (n < 1 || n > MAXN) return -1;
  long double x[MAXN], w[MAXN], phi[MAXN], dphi[MAXN];
  long double K[MAXN][MAXN], A[MAXN][2 * MAXN];
  gauss_legendre(n, x, w);
  /* Kxi[k][l] = sum_i w_i phi_k'(x_i) phi_l(x_i)   (aderdg.py:53-78) */
  for (int k = 0; k < n; k++)
    for (int l = 0; l < n; l++) K[k][l] = 0.0L;
  for (int i = 0; i < n; i++) {
    base_func(n, x, x[i], phi, dphi);
    for (int k = 0; k < n; k++)
      for (int l = 0; l < n; l++) K[k][l] += w[i] * dphi[k] * phi[l];
  }
  /* K1 = phi(1) phi(1)^T - Kxi, iK1 = K1^{-1}   (aderdg.py:134-159) */
  long double p1[MAXN], p0[MAXN];
  base_func(n, x, 1.0L, p1, dphi);
  base_func(n, x, 0.0L, p0, dphi);
  for (int k = 0; k < n; k++)
    for (int l = 0; l < n; l++) {
      A[k][l] = p1[k] * p1[l] - K[k][l];
      A[k][n + l] = (k == l) ? 1.0L : 0.0L;
    }
  for (int c = 0; c < n; c++) { /* Gauss-Jordan with partial pivoting */
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (fabsl(A[r][c]) > fabsl(A[piv][c])) piv = r;
    if (piv != c)
      for (int j = 0; j < 2 * n; j++) { long double t = A[c][j]; A[c][j] = A[piv][j]; A[piv][j] = t; }
    long double d = A[c][c];
    for (int j = 0; j < 2 * n; j++) A[c][j] /= d;
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      long double f = A[r][c];
      for (int j = 0; j < 2 * n; j++) A[r][j] -= f * A[c][j];
    }
  }
  for (int i = 0; i < n; i++) {
    if (nodes) nodes[i] = (double)x[i];
    if (weights) weights[i] = (double)w[i];
    if (F0) F0[i] = (double)p0[i];
    if (F1) F1[i] = (double)p1[i];
    for (int j = 0; j < n; j++) {
      if (Kxi) Kxi[i * n + j] = (double)K[i][j];
      if (iK1) iK1[i * n + j] = (double)A[i][n + j];
      /* dudx = M^{-1} Kxi^T with the diagonal GL mass matrix M = diag(w) (aderdg.py:177-195) */
      if (dudx) dudx[i * n + j] = (double)(K[j][i] / w[i]);
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* PDE terms (L0 user hooks)                                                                   */
/* ------------------------------------------------------------------------------------------ */

/* Euler, gamma = 1.4: ApplicationExamples/Euler/Euler_ADERDG/EulerSolver_ADERDG.cpp:61-146. */
static void euler_flux(int dim, const double* Q, double* F /*[d][5]*/) {
  const double gamma = 1.4;
  const double irho = 1. / Q[0];
  const double j2 = dim == 3 ? Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3] : Q[1] * Q[1] + Q[2] * Q[2];
  const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
  for (int d = 0; d < dim; d++) {
    double* f = F + 5 * d;
    const double un = Q[1 + d];
    f[0] = un;
    f[1] = irho * Q[1] * un;
    f[2] = irho * Q[2] * un;
    f[3] = irho * Q[3] * un;
    f[1 + d] += p;
    f[4] = irho * (Q[4] + p) * un;
  }
}
static void euler_eig(int dim, const double* Q, int d, double* lambda) {
  const double gamma = 1.4;
  const double irho = 1. / Q[0];
  const double j2 = dim == 3 ? Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3] : Q[1] * Q[1] + Q[2] * Q[2];
  const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
  const double u_n = Q[d + 1] * irho;
  const double c = sqrt(gamma * p * irho);
  for (int m = 0; m < 5; m++) lambda[m] = u_n;
  lambda[0] -= c;
  lambda[4] += c;
}

/* Shallow water (h, hu, hv, b): ApplicationExamples/SWE/SWE_ADERDG/MySWESolver.cpp:103-152, g=9.81. */
static const double SWE_G = 9.81;
static void swe_flux(int dim, const double* Q, double* F) {
  const double ih = 1. / Q[0];
  double* f = F;
  double* g = F + 4;
  f[0] = Q[1];
  f[1] = Q[1] * Q[1] * ih + 0.5 * SWE_G * Q[0] * Q[0];
  f[2] = Q[1] * Q[2] * ih;
  f[3] = 0.0;
  g[0] = Q[2];
  g[1] = Q[1] * Q[2] * ih;
  g[2] = Q[2] * Q[2] * ih + 0.5 * SWE_G * Q[0] * Q[0];
  g[3] = 0.0;
  if (dim == 3) memset(F + 8, 0, 4 * sizeof(double));
}
static void swe_eig(const double* Q, int d, double* lambda) {
  const double c = sqrt(SWE_G * Q[0]);
  const double ih = 1. / Q[0];
  const double u_n = Q[d + 1] * ih;
  lambda[0] = u_n + c;
  lambda[1] = u_n - c;
  lambda[2] = u_n;
  lambda[3] = 0.0;
}
static void swe_ncp(const double* Q, const double* gradQ /*[d][4]*/, double* BgradQ) {
  BgradQ[0] = 0.0;
  BgradQ[1] = SWE_G * Q[0] * gradQ[0 * 4 + 3];
  BgradQ[2] = SWE_G * Q[0] * gradQ[1 * 4 + 3];
  BgradQ[3] = 0.0;
}

/* Linear acoustics in flux form with per-node parameters Q[4] = rho, Q[5] = c (new functor;
 * the reference's acoustic app uses the linear kernels): F_d = (rho c^2 u_d, p/rho e_d). */
static void acoustic_flux(int dim, const double* Q, double* F) {
  const double rho = Q[4], cc = Q[5];
  const double K = rho * cc * cc;
  const double pr = Q[0] / rho;
  for (int d = 0; d < dim; d++) {
    double* f = F + 4 * d;
    f[0] = K * Q[1 + d];
    f[1] = d == 0 ? pr : 0.0;
    f[2] = d == 1 ? pr : 0.0;
    f[3] = d == 2 ? pr : 0.0;
  }
}
/* Linear elasticity, velocity-stress form, per-node rho, cp, cs (Q[9..11]) in flux form. */
static void elastic_flux(int dim, const double* Q, double* F) {
  const double rho = Q[9], cp = Q[10], cs = Q[11];
  const double mu = rho * cs * cs;
  const double lam = rho * cp * cp - 2.0 * mu;
  const double ir = 1.0 / rho;
  const double sg[3][3] = {{Q[3], Q[6], Q[7]}, {Q[6], Q[4], Q[8]}, {Q[7], Q[8], Q[5]}};
  for (int d = 0; d < dim; d++) {
    double* f = F + 9 * d;
    f[0] = -sg[0][d] * ir;
    f[1] = -sg[1][d] * ir;
    f[2] = -sg[2][d] * ir;
    const double vd = Q[d];
    f[3] = -(lam * vd + (d == 0 ? 2.0 * mu * vd : 0.0));
    f[4] = -(lam * vd + (d == 1 ? 2.0 * mu * vd : 0.0));
    f[5] = -(lam * vd + (d == 2 ? 2.0 * mu * vd : 0.0));
    f[6] = -mu * ((d == 0 ? Q[1] : 0.0) + (d == 1 ? Q[0] : 0.0));
    f[7] = -mu * ((d == 0 ? Q[2] : 0.0) + (d == 2 ? Q[0] : 0.0));
    f[8] = -mu * ((d == 1 ? Q[2] : 0.0) + (d == 2 ? Q[1] : 0.0));
  }
}

void exo_flux(const exo_cfg* c, const double* Q, double* F) {
  switch (c->pde) {
    case EXO_PDE_EULER: euler_flux(c->dim, Q, F); break;
    case EXO_PDE_SWE: swe_flux(c->dim, Q, F); break;
    case EXO_PDE_ACOUSTIC: acoustic_flux(c->dim, Q, F); break;
    case EXO_PDE_ELASTIC: elastic_flux(c->dim, Q, F); break;
    default: memset(F, 0, sizeof(double) * c->dim * c->nvar);
  }
}
void exo_eigenvalues(const exo_cfg* c, const double* Q, int d, double* lambda) {
  switch (c->pde) {
    case EXO_PDE_EULER: euler_eig(c->dim, Q, d, lambda); break;
    case EXO_PDE_SWE: swe_eig(Q, d, lambda); break;
    case EXO_PDE_ACOUSTIC:
      lambda[0] = -Q[5]; lambda[1] = 0.0; lambda[2] = 0.0; lambda[3] = Q[5];
      break;
    case EXO_PDE_ELASTIC: {
      const double cp = Q[10], cs = Q[11];
      const double l[9] = {-cp, -cs, -cs, 0.0, 0.0, 0.0, cs, cs, cp};
      memcpy(lambda, l, sizeof(l));
      break;
    }
    default: memset(lambda, 0, sizeof(double) * c->nvar);
  }
}

/* Regularised point source on variable src[7]: amplitude * Ricker(t - t0; f0) * Gaussian of
 * width src[6] around (src[0..2]), normalised to unit mass; cells whose centre is farther than
 * 6 widths plus a cell diagonal receive none (the same truncation as the device kernels). */
static double point_source(const exo_cfg* c, const double* x, double t) {
  const double pi = 3.14159265358979323846;
  double r2 = 0.0;
  for (int d = 0; d < c->dim; d++) r2 += (x[d] - c->src[d]) * (x[d] - c->src[d]);
  const double w = c->src[6];
  const double a = pi * c->src[3] * (t - c->src[4]);
  const double ricker = (1.0 - 2.0 * a * a) * exp(-a * a);
  const double norm = c->dim == 3 ? 1.0 / (15.749609945722419 * w * w * w) : 1.0 / (6.283185307179586 * w * w);
  return c->src[5] * ricker * exp(-0.5 * r2 / (w * w)) * norm;
}
static int source_near(const exo_cfg* c, const double* centre, const double* dx) {
  double r2 = 0.0, h2 = 0.0;
  for (int d = 0; d < c->dim; d++) {
    r2 += (centre[d] - c->src[d]) * (centre[d] - c->src[d]);
    h2 += dx[d] * dx[d];
  }
  const double reach = 6.0 * c->src[6] + sqrt(h2);
  return r2 <= reach * reach;
}
static void exo_ncp(const exo_cfg* c, const double* Q, const double* gradQ, double* BgradQ) {
  switch (c->pde) {
    case EXO_PDE_SWE: swe_ncp(Q, gradQ, BgradQ); break;
    default: memset(BgradQ, 0, sizeof(double) * c->nvar);
  }
}
/* Reflective wall: mirrored normal momentum, flux of the mirrored state
 * (MySWESolver.cpp:43-62; the same construction for Euler). */
void exo_boundary_wall(const exo_cfg* c, double* FOut, double* QOut, const double* QIn, int normal) {
  const int D = c->nvar + c->npar;
  double F[3 * MAXV];
  memcpy(QOut, QIn, sizeof(double) * D);
  if (c->pde == EXO_PDE_ELASTIC) {
    for (int k = 0; k < 3; k++) QOut[k] = -QOut[k];
  } else {
    QOut[1 + normal] = -QOut[1 + normal];
  }
  exo_flux(c, QOut, F);
  memcpy(FOut, F + normal * c->nvar, sizeof(double) * c->nvar);
}
/* outflow: boundaryValues returning the inner state and its flux */
static void exo_boundary_outflow(const exo_cfg* c, double* FOut, double* QOut, const double* QIn, int normal) {
  const int D = c->nvar + c->npar;
  double F[3 * MAXV];
  memcpy(QOut, QIn, sizeof(double) * D);
  exo_flux(c, QOut, F);
  memcpy(FOut, F + normal * c->nvar, sizeof(double) * c->nvar);
}

/* ------------------------------------------------------------------------------------------ */
/* Geometry helpers: node p has coordinates (z,y,x) in 3D or (y,x) in 2D, x fastest.           */
/* coord[dir] is the coordinate along axis dir (0=x,1=y,2=z).                                  */
/* ------------------------------------------------------------------------------------------ */
typedef struct {
  int dim, n, v, D, nd, nf;
  double w[MAXN], x[MAXN], Kxi[MAXN * MAXN], iK1[MAXN * MAXN], dudx[MAXN * MAXN], F0[MAXN], F1[MAXN];
} geo;

static void geo_init(geo* g, const exo_cfg* c) {
  g->dim = c->dim;
  g->n = c->order + 1;
  g->v = c->nvar;
  g->D = c->nvar + c->npar;
  g->nd = g->dim == 3 ? g->n * g->n * g->n : g->n * g->n;
  g->nf = g->dim == 3 ? g->n * g->n : g->n;
  exo_tables(c->order, g->x, g->w, g->Kxi, g->iK1, g->dudx, g->F0, g->F1);
}
static inline void node_coords(const geo* g, int p, int* co) {
  co[0] = p % g->n;
  co[1] = (p / g->n) % g->n;
  co[2] = g->dim == 3 ? p / (g->n * g->n) : 0;
}
static inline int node_index(const geo* g, const int* co) {
  return g->dim == 3 ? (co[2] * g->n + co[1]) * g->n + co[0] : co[1] * g->n + co[0];
}
static inline int axis_stride(const geo* g, int dir) { return dir == 0 ? 1 : (dir == 1 ? g->n : g->n * g->n); }
/* tangential coordinates of a node w.r.t. direction dir, slower axis first */
static inline void tangential(const geo* g, int dir, const int* co, int* a, int* b) {
  if (g->dim == 2) { *a = co[dir == 0 ? 1 : 0]; *b = 0; return; }
  if (dir == 0) { *a = co[2]; *b = co[1]; }
  else if (dir == 1) { *a = co[2]; *b = co[0]; }
  else { *a = co[1]; *b = co[0]; }
}
/* product of weights over the tangential coordinates, slower axis first */
static inline double w_tan(const geo* g, int dir, const int* co) {
  int a, b;
  tangential(g, dir, co, &a, &b);
  return g->dim == 3 ? g->w[a] * g->w[b] : g->w[a];
}
/* product of spatial weights, slowest axis first (z,y,x) */
static inline double w_space(const geo* g, const int* co) {
  return g->dim == 3 ? g->w[co[2]] * g->w[co[1]] * g->w[co[0]] : g->w[co[1]] * g->w[co[0]];
}
/* offset of a face-node (a,b) inside one face block */
static inline int face_node(const geo* g, int a, int b) { return g->dim == 3 ? a * g->n + b : a; }
/* lFhi block for direction dir stores the node with the normal coordinate fastest */
static inline int lfhi_index(const geo* g, int dir, const int* co) {
  int a, b;
  tangential(g, dir, co, &a, &b);
  return g->dim == 3 ? (a * g->n + b) * g->n + co[dir] : a * g->n + co[dir];
}

/* ------------------------------------------------------------------------------------------ */
/* Space-time predictor: 3d/spaceTimePredictorNonlinear.cpph:39-433 (Picard loop), :441-515    */
/* (time averaging), :517-687 (extrapolation), :816-864 (entry); 2D analogue 2d/...:38-597.    */
/* Source term (:323-367): S = algebraicSource(x_node, t + node_i dt) - NCP; the point source   */
/* of the acoustic / elastic systems is the only algebraicSource here (zero for Euler / SWE).  */
/* ------------------------------------------------------------------------------------------ */
int exo_predictor(const exo_cfg* c, const double* luh, const double* centre, const double* dx, double t,
                  double dt, double* lQi, double* lFi, double* lQhi, double* lFhi, double* lQhbnd,
                  double* lFhbnd, int* sweeps) {
  geo g;
  geo_init(&g, c);
  const int n = g.n, v = g.v, D = g.D, nd = g.nd, dim = g.dim, nf = g.nf;
  const int useNCP = c->use_ncp;
  const int useSource = c->has_src; /* the lFi source block exists (zero far from the source) */
  const int srcOn = c->has_src && source_near(c, centre, dx);
  const int srcVar = (int)c->src[7];
  double invDx[3];
  for (int d = 0; d < dim; d++) invDx[d] = 1.0 / dx[d];
  const int maxIter = c->max_picard > 0 ? c->max_picard : 2 * n;
  double* rhs = (double*)malloc(sizeof(double) * n * nd * v);
  double* gradQ = (double*)malloc(sizeof(double) * nd * dim * v);
  /* lQi[p][t][D], lFi[t][p][d+1][v] */
#define LQI(p, tt, m) lQi[((p) * n + (tt)) * D + (m)]
#define LFI(tt, p, dd, m) lFi[(((tt) * nd + (p)) * (dim + 1) + (dd)) * v + (m)]
#define RHS(tt, p, m) rhs[((tt) * nd + (p)) * v + (m)]
  /* 1. trivial initial guess (:71-82) */
  for (int p = 0; p < nd; p++)
    for (int tt = 0; tt < n; tt++)
      for (int m = 0; m < D; m++) LQI(p, tt, m) = luh[p * D + m];
  int iter = 0, converged = 0, nsweeps = 0;
  for (; iter < maxIter; iter++) {
    nsweeps++;
    for (int i = 0; i < n; i++) { /* time node */
      /* gradients via dudx (:111-175), only with NCP */
      if (useNCP) {
        memset(gradQ, 0, sizeof(double) * nd * dim * v);
        for (int dd = 0; dd < dim; dd++) {
          const int s = axis_stride(&g, dd);
          for (int p = 0; p < nd; p++) {
            int co[3];
            node_coords(&g, p, co);
            const int l = co[dd];
            const int base = p - l * s;
            for (int m = 0; m < v; m++)
              for (int nn = 0; nn < n; nn++)
                gradQ[(p * dim + dd) * v + m] += 1.0 * invDx[dd] * LQI(base + nn * s, i, m) * g.dudx[l * n + nn];
          }
        }
      }
      /* fluxes (:196-227) */
      for (int p = 0; p < nd; p++) {
        double F[3 * MAXV];
        exo_flux(c, &LQI(p, i, 0), F);
        for (int dd = 0; dd < dim; dd++)
          for (int m = 0; m < v; m++) LFI(i, p, dd, m) = F[dd * v + m];
      }
      /* rhs0 = w_space F0[i] luh (:231-246) */
      for (int p = 0; p < nd; p++) {
        int co[3];
        node_coords(&g, p, co);
        const double weight = w_space(&g, co);
        for (int m = 0; m < v; m++) RHS(i, p, m) = weight * g.F0[i] * luh[p * D + m];
      }
      /* flux contractions, x then y then z (:248-321) */
      for (int dd = 0; dd < dim; dd++) {
        const int s = axis_stride(&g, dd);
        for (int p = 0; p < nd; p++) {
          int co[3];
          node_coords(&g, p, co);
          int a, b;
          tangential(&g, dd, co, &a, &b);
          const double weight = dim == 3 ? g.w[i] * g.w[a] * g.w[b] : g.w[i] * g.w[a];
          const double updateSize = weight * dt * invDx[dd];
          const int l = co[dd];
          const int base = p - l * s;
          for (int m = 0; m < v; m++)
            for (int nn = 0; nn < n; nn++)
              RHS(i, p, m) -= updateSize * LFI(i, base + nn * s, dd, m) * g.Kxi[nn * n + l];
        }
      }
      /* source / NCP (:323-367) */
      if (useNCP || useSource) {
        for (int p = 0; p < nd; p++) {
          int co[3];
          node_coords(&g, p, co);
          const double weight = dim == 3 ? g.w[i] * g.w[co[2]] * g.w[co[1]] * g.w[co[0]]
                                         : g.w[i] * g.w[co[1]] * g.w[co[0]];
          const double updateSize = weight * dt;
          double* S = &LFI(i, p, dim, 0);
          for (int m = 0; m < v; m++) S[m] = 0.0;
          if (srcOn) {
            double x[3];
            for (int dd = 0; dd < dim; dd++) x[dd] = centre[dd] + dx[dd] * (g.x[co[dd]] - 0.5);
            S[srcVar] = point_source(c, x, t + g.x[i] * dt);
          }
          if (useNCP) {
            double ncp[MAXV];
            exo_ncp(c, &LQI(p, i, 0), &gradQ[p * dim * v], ncp);
            for (int m = 0; m < v; m++) S[m] -= ncp[m];
          }
          for (int m = 0; m < v; m++) RHS(i, p, m) += updateSize * S[m];
        }
      }
    }
    /* time solve with iK1 and the residual (:370-405) */
    double sq_res = 0.0;
    for (int p = 0; p < nd; p++) {
      int co[3];
      node_coords(&g, p, co);
      const double iweight = 1.0 / w_space(&g, co);
      for (int l = 0; l < n; l++)
        for (int m = 0; m < v; m++) {
          double q = 0;
          for (int nn = 0; nn < n; nn++) q += iweight * RHS(nn, p, m) * g.iK1[l * n + nn];
          const double r = q - LQI(p, l, m);
          sq_res += r * r;
          LQI(p, l, m) = q;
        }
    }
    /* exit condition (:407-412), tolerance 1e-7 squared */
    if (c->max_picard <= 0 && sq_res < 1e-7 * 1e-7) {
      converged = 1;
      break;
    }
  }
  int ret = iter;
  if (dim == 2) ret = converged ? maxIter + 2 : maxIter; /* 2d/...:303-305 quirk */
  if (sweeps) *sweeps = nsweeps;

  /* time averaging (:441-515): lQhi, lFhi (direction-permuted blocks), lShi */
  memset(lQhi, 0, sizeof(double) * nd * D);
  memset(lFhi, 0, sizeof(double) * (dim + 1) * nd * v);
  for (int p = 0; p < nd; p++) {
    int co[3];
    node_coords(&g, p, co);
    for (int m = 0; m < v; m++)
      for (int tt = 0; tt < n; tt++) {
        for (int dd = 0; dd < dim; dd++)
          lFhi[dd * nd * v + lfhi_index(&g, dd, co) * v + m] += LFI(tt, p, dd, m) * g.w[tt];
        if (useNCP || useSource) lFhi[dim * nd * v + p * v + m] += LFI(tt, p, dim, m) * g.w[tt];
      }
    for (int m = 0; m < D; m++)
      for (int tt = 0; tt < n; tt++) lQhi[p * D + m] += LQI(p, tt, m) * g.w[tt];
  }
  /* extrapolation to the faces (:517-687) */
  memset(lQhbnd, 0, sizeof(double) * 2 * dim * nf * D);
  memset(lFhbnd, 0, sizeof(double) * 2 * dim * nf * v);
  for (int dd = 0; dd < dim; dd++) {
    const int s = axis_stride(&g, dd);
    /* 2D x faces extrapolate only the nVar evolved entries of lQhbnd (2d/...:436-445 quirk) */
    const int nQ = (dim == 2 && dd == 0) ? v : D;
    for (int p = 0; p < nd; p++) {
      int co[3];
      node_coords(&g, p, co);
      if (co[dd] != 0) continue;
      int a, b;
      tangential(&g, dd, co, &a, &b);
      const int fn = face_node(&g, a, b);
      for (int l = 0; l < n; l++) {
        int cl[3] = {co[0], co[1], co[2]};
        cl[dd] = l;
        const int q = p + l * s;
        for (int m = 0; m < v; m++) {
          const double f = lFhi[dd * nd * v + lfhi_index(&g, dd, cl) * v + m];
          lFhbnd[((2 * dd + 0) * nf + fn) * v + m] += f * g.F0[l];
          lFhbnd[((2 * dd + 1) * nf + fn) * v + m] += f * g.F1[l];
        }
        for (int m = 0; m < nQ; m++) {
          lQhbnd[((2 * dd + 0) * nf + fn) * D + m] += lQhi[q * D + m] * g.F0[l];
          lQhbnd[((2 * dd + 1) * nf + fn) * D + m] += lQhi[q * D + m] * g.F1[l];
        }
      }
    }
  }
  free(rhs);
  free(gradQ);
#undef LQI
#undef LFI
#undef RHS
  return ret;
}

/* Volume integral, time-averaged branch: 3d/volumeIntegralNonlinear.cpph:133-223, 2d/...:115-176. */
void exo_volume(const exo_cfg* c, double* lduh, const double* lFhi, const double* dx) {
  geo g;
  geo_init(&g, c);
  const int n = g.n, v = g.v, nd = g.nd, dim = g.dim;
  memset(lduh, 0, sizeof(double) * nd * v);
  for (int dd = 0; dd < dim; dd++) {
    const double invDx = 1.0 / dx[dd];
    for (int p = 0; p < nd; p++) {
      int co[3];
      node_coords(&g, p, co);
      const double updateSize = w_tan(&g, dd, co) * invDx;
      const int k = co[dd];
      for (int m = 0; m < v; m++)
        for (int mm = 0; mm < n; mm++) {
          int cm[3] = {co[0], co[1], co[2]};
          cm[dd] = mm;
          lduh[p * v + m] += g.Kxi[k * n + mm] * lFhi[dd * nd * v + lfhi_index(&g, dd, cm) * v + m] * updateSize;
        }
    }
  }
  if (c->use_ncp || c->has_src) {
    for (int p = 0; p < nd; p++) {
      int co[3];
      node_coords(&g, p, co);
      const double weight = w_space(&g, co);
      for (int m = 0; m < v; m++) lduh[p * v + m] += weight * lFhi[dim * nd * v + p * v + m];
    }
  }
}

/* Rusanov flux with face-averaged smax: 3d/riemannSolverNonlinear.cpph:37-128,
 * averageRiemannInputs RiemannSolverUtils.h:152-177. FL/FR are in/out. */
void exo_riemann(const exo_cfg* c, double* FL, double* FR, const double* QL, const double* QR,
                 const double* dx, int direction) {
  (void)dx;
  geo g;
  geo_init(&g, c);
  const int n = g.n, v = g.v, D = g.D, nf = g.nf, dim = g.dim;
  double QavL[MAXV] = {0}, QavR[MAXV] = {0};
  for (int a = 0; a < (dim == 3 ? n : 1); a++)
    for (int b = 0; b < n; b++) {
      const double wab = dim == 3 ? g.w[a] * g.w[b] : g.w[b];
      const int fn = dim == 3 ? a * n + b : b;
      for (int k = 0; k < D; k++) {
        QavL[k] += wab * QL[fn * D + k];
        QavR[k] += wab * QR[fn * D + k];
      }
    }
  double LL[MAXV], LR[MAXV];
  exo_eigenvalues(c, QavL, direction, LL);
  exo_eigenvalues(c, QavR, direction, LR);
  double sL = 0, sR = 0;
  for (int m = 0; m < v; m++) {
    LL[m] = fabs(LL[m]);
    LR[m] = fabs(LR[m]);
  }
  sL = LL[0];
  sR = LR[0];
  for (int m = 1; m < v; m++) {
    if (LL[m] > sL) sL = LL[m];
    if (LR[m] > sR) sR = LR[m];
  }
  const double smax = sL > sR ? sL : sR;
  for (int fn = 0; fn < nf; fn++) {
    double ncp[MAXV] = {0};
    if (c->use_ncp) {
      double gradQ[3 * MAXV] = {0};
      double Qavg[MAXV];
      for (int l = 0; l < v; l++) gradQ[direction * v + l] = QR[fn * D + l] - QL[fn * D + l];
      for (int l = 0; l < D; l++) Qavg[l] = 0.5 * (QR[fn * D + l] + QL[fn * D + l]);
      exo_ncp(c, Qavg, gradQ, ncp);
    }
    for (int k = 0; k < v; k++) {
      const int i = fn * v + k;
      FL[i] = 0.5 * (FR[i] + FL[i]) - 0.5 * smax * (QR[fn * D + k] - QL[fn * D + k]);
      if (c->use_ncp) {
        FR[i] = FL[i] - 0.5 * ncp[k];
        FL[i] = FL[i] + 0.5 * ncp[k];
      } else {
        FR[i] = FL[i];
      }
    }
  }
}

/* Surface integral over all faces: 3d/surfaceIntegralNonlinear.cpph:21-90, 2d/...:26-74. */
void exo_surface(const exo_cfg* c, double* lduh, const double* lFhbnd, const double* dx) {
  geo g;
  geo_init(&g, c);
  const int v = g.v, nd = g.nd, dim = g.dim, nf = g.nf;
  for (int dd = 0; dd < dim; dd++) {
    const double invDx = 1.0 / dx[dd];
    for (int p = 0; p < nd; p++) {
      int co[3], a, b;
      node_coords(&g, p, co);
      tangential(&g, dd, co, &a, &b);
      const int fn = face_node(&g, a, b);
      const double updateSize = w_tan(&g, dd, co) * invDx;
      const int k = co[dd];
      for (int m = 0; m < v; m++)
        lduh[p * v + m] -= (lFhbnd[((2 * dd + 1) * nf + fn) * v + m] * g.F1[k] -
                            lFhbnd[((2 * dd + 0) * nf + fn) * v + m] * g.F0[k]) * updateSize;
    }
  }
}

/* Single-face lifting: 3d/faceIntegralNonlinear.cpph:21-103. */
void exo_face(const exo_cfg* c, double* lduh, const double* lFhbnd_face, int direction, int orientation,
              const double* dx) {
  geo g;
  geo_init(&g, c);
  const int v = g.v, nd = g.nd;
  const double scaling = 1.0 / dx[direction] * (2.0 * orientation - 1.0);
  const double* Fc = orientation ? g.F1 : g.F0;
  for (int p = 0; p < nd; p++) {
    int co[3], a, b;
    node_coords(&g, p, co);
    tangential(&g, direction, co, &a, &b);
    const double scaledWeight = w_tan(&g, direction, co) * scaling;
    for (int m = 0; m < v; m++)
      lduh[p * v + m] -= scaledWeight * Fc[co[direction]] * lFhbnd_face[face_node(&g, a, b) * v + m];
  }
}

/* luh = luhOld + dt/w_ijk * lduh for the evolved variables: 3d/solutionUpdate.cpph:28-67. */
void exo_update(const exo_cfg* c, double* luh, const double* luhOld, const double* lduh, double dt) {
  geo g;
  geo_init(&g, c);
  for (int p = 0; p < g.nd; p++) {
    int co[3];
    node_coords(&g, p, co);
    const double updateSize = dt / w_space(&g, co);
    for (int m = 0; m < g.v; m++) luh[p * g.D + m] = luhOld[p * g.D + m] + lduh[p * g.v + m] * updateSize;
  }
}

/* CFL: 3d/stableTimeStepSize.cpph:14-62. */
double exo_dt(const exo_cfg* c, const double* luh, const double* dx) {
  geo g;
  geo_init(&g, c);
  double dt = DBL_MAX;
  const double cflPNPM = c->cfl * c->pnpm;
  for (int p = 0; p < g.nd; p++) {
    double den = 0.0;
    for (int d = 0; d < g.dim; d++) {
      double lambda[MAXV];
      exo_eigenvalues(c, luh + p * g.D, d, lambda);
      double mx = 0.0;
      for (int m = 0; m < g.v; m++) mx = fmax(fabs(lambda[m]), mx);
      den += mx * (1.0 / dx[d]);
    }
    const double cand = cflPNPM / den;
    if (cand < dt) dt = cand;
  }
  return dt;
}

/* ------------------------------------------------------------------------------------------ */
/* Uniform patch driver, global non-fused order (ADERDGSolver.cpp:887-947, 1190-1258;           */
/* boundary faces through boundaryConditions + Riemann as glue :307-350).                      */
/* ------------------------------------------------------------------------------------------ */
int exo_run(const exo_cfg* c, const int* ncell, const double* offset, const double* size, int walls,
            double* luh, int nsteps, double t0, double fixed_dt, double* t_out, double* dts, int* picard,
            int nthreads) {
  geo g;
  geo_init(&g, c);
  const int dim = g.dim, v = g.v, D = g.D, nd = g.nd, nf = g.nf, n = g.n;
  const int nx = ncell[0], ny = ncell[1], nz = dim == 3 ? ncell[2] : 1;
  const long nc = (long)nx * ny * nz;
  const double dx[3] = {size[0] / nx, size[1] / ny, dim == 3 ? size[2] / nz : 1.0};
  const long sQ = 2L * dim * nf * D, sF = 2L * dim * nf * v;
  double* lduh = (double*)malloc(sizeof(double) * nc * nd * v);
  double* lQhbnd = (double*)malloc(sizeof(double) * nc * sQ);
  double* lFhbnd = (double*)malloc(sizeof(double) * nc * sF);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  double t = t0;
  for (int step = 0; step < nsteps; step++) {
    double dt = DBL_MAX;
    if (fixed_dt > 0) {
      dt = fixed_dt;
    } else {
#pragma omp parallel for reduction(min : dt) schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        double d = exo_dt(c, luh + ci * nd * D, dx);
        if (d < dt) dt = d;
      }
    }
#pragma omp parallel
    {
      double* lQi = (double*)malloc(sizeof(double) * nd * n * D);
      double* lFi = (double*)malloc(sizeof(double) * n * nd * (dim + 1) * v);
      double* lQhi = (double*)malloc(sizeof(double) * nd * D);
      double* lFhi = (double*)malloc(sizeof(double) * (dim + 1) * nd * v);
#pragma omp for schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        const int ix = ci % nx, iy = (ci / nx) % ny, iz = (int)(ci / ((long)nx * ny));
        double centre[3] = {offset[0] + (ix + 0.5) * dx[0], offset[1] + (iy + 0.5) * dx[1],
                            dim == 3 ? offset[2] + (iz + 0.5) * dx[2] : 0.0};
        int sw = 0;
        exo_predictor(c, luh + ci * nd * D, centre, dx, t, dt, lQi, lFi, lQhi, lFhi, lQhbnd + ci * sQ,
                      lFhbnd + ci * sF, &sw);
        if (picard) picard[(long)step * nc + ci] = sw;
        exo_volume(c, lduh + ci * nd * v, lFhi, dx);
      }
      free(lQi); free(lFi); free(lQhi); free(lFhi);
    }
    for (int d = 0; d < dim; d++) {
#pragma omp parallel for schedule(static)
      for (long ci = 0; ci < nc; ci++) {
        const int ix = ci % nx, iy = (ci / nx) % ny, iz = (int)(ci / ((long)nx * ny));
        int j[3] = {ix, iy, iz};
        const int lim = d == 0 ? nx : (d == 1 ? ny : nz);
        j[d] += 1;
        double* FL = lFhbnd + ci * sF + (2 * d + 1) * nf * v;
        const double* QL = lQhbnd + ci * sQ + (2 * d + 1) * nf * D;
        double QOut[MAXN * MAXN * MAXV], FOut[MAXN * MAXN * MAXV];
        if (j[d] == lim) {
          if (walls) {
            for (int f = 0; f < nf; f++) {
              if (walls == 3)
                exo_boundary_outflow(c, FOut + f * v, QOut + f * D, QL + f * D, d);
              else
                exo_boundary_wall(c, FOut + f * v, QOut + f * D, QL + f * D, d);
            }
            exo_riemann(c, FL, FOut, QL, QOut, dx, d);
          } else {
            j[d] = 0;
          }
        }
        if (j[d] < lim) {
          const long c2 = ((long)j[2] * ny + j[1]) * nx + j[0];
          exo_riemann(c, FL, lFhbnd + c2 * sF + 2 * d * nf * v, QL, lQhbnd + c2 * sQ + 2 * d * nf * D, dx, d);
        }
        const int k = d == 0 ? ix : (d == 1 ? iy : iz);
        if (walls && k == 0) {
          double* FRb = lFhbnd + ci * sF + 2 * d * nf * v;
          const double* QRb = lQhbnd + ci * sQ + 2 * d * nf * D;
          for (int f = 0; f < nf; f++) {
            if (walls == 3)
              exo_boundary_outflow(c, FOut + f * v, QOut + f * D, QRb + f * D, d);
            else
              exo_boundary_wall(c, FOut + f * v, QOut + f * D, QRb + f * D, d);
          }
          exo_riemann(c, FOut, FRb, QOut, QRb, dx, d);
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (long ci = 0; ci < nc; ci++) {
      exo_surface(c, lduh + ci * nd * v, lFhbnd + ci * sF, dx);
      exo_update(c, luh + ci * nd * D, luh + ci * nd * D, lduh + ci * nd * v, dt);
    }
    if (dts) dts[step] = dt;
    t += dt;
  }
  if (t_out) *t_out = t;
  free(lduh);
  free(lQhbnd);
  free(lFhbnd);
  return 0;
}
