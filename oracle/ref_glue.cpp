// Checker glue around the reference's OWN generic ADER-DG kernels.
//
// This file is test infrastructure: it is compiled (by oracle/Makefile) together with the
// unmodified reference headers ExaHyPE/kernels/aderdg/generic/Kernels.h and
// ExaHyPE/kernels/GaussLegendreBasis.cpp, read in place from the reference checkout, into
// oracle/_ref/libexaref{2,3}d.so. Only tests and bench.py's CPU baseline load it. It plays the
// role of the toolkit-generated glue (Toolkit/exahype/toolkit/templates/solvers/
// AbstractGenericADERDGSolverImplementation.template:104-361): a SolverType with the static
// contract of AbstractGenericADERDGSolverHeader.template:34-68 plus extern "C" wrappers.
//
// Build with -DDIMENSIONS=2 or -DDIMENSIONS=3.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "kernels/GaussLegendreBasis.h"
#include "kernels/KernelUtils.h"
#include "kernels/aderdg/generic/Kernels.h"

namespace exaref {

// ADER-DG PNPM table by order (Toolkit/exahype/toolkit/solverController.py:17).
constexpr double kPNPM[10] = {1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015};

// Compressible Euler, gamma = 1.4 (ApplicationExamples/Euler/Euler_ADERDG/EulerSolver_ADERDG.cpp:61-146).
// nVar = 5 in 2D and 3D (the 2D app carries the unused z-momentum).
struct EulerPDE {
  static constexpr int NumberOfVariables = 5;
  static void flux(const double* const Q, double** const F) {
    constexpr double gamma = 1.4;
    const double irho = 1. / Q[0];
#if DIMENSIONS == 3
    const double j2 = Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3];
#else
    const double j2 = Q[1] * Q[1] + Q[2] * Q[2];
#endif
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
    F[0][0] = Q[1];
    F[0][1] = irho * Q[1] * Q[1] + p;
    F[0][2] = irho * Q[2] * Q[1];
    F[0][3] = irho * Q[3] * Q[1];
    F[0][4] = irho * (Q[4] + p) * Q[1];
    F[1][0] = Q[2];
    F[1][1] = irho * Q[1] * Q[2];
    F[1][2] = irho * Q[2] * Q[2] + p;
    F[1][3] = irho * Q[3] * Q[2];
    F[1][4] = irho * (Q[4] + p) * Q[2];
#if DIMENSIONS == 3
    F[2][0] = Q[3];
    F[2][1] = irho * Q[1] * Q[3];
    F[2][2] = irho * Q[2] * Q[3];
    F[2][3] = irho * Q[3] * Q[3] + p;
    F[2][4] = irho * (Q[4] + p) * Q[3];
#endif
  }
  static void eigenvalues(const double* const Q, const int direction, double* const lambda) {
    constexpr double gamma = 1.4;
    const double irho = 1. / Q[0];
#if DIMENSIONS == 3
    const double j2 = Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3];
#else
    const double j2 = Q[1] * Q[1] + Q[2] * Q[2];
#endif
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
    const double u_n = Q[direction + 1] * irho;
    const double c = std::sqrt(gamma * p * irho);
    std::fill_n(lambda, 5, u_n);
    lambda[0] -= c;
    lambda[4] += c;
  }
  static void nonConservativeProduct(const double* const, const double* const, double* const BgradQ) {
    std::fill_n(BgradQ, 5, 0.0);
  }
  // Reflective wall (used only by boundary tests).
  static void wall(const double* QIn, int normal, double* QOut) {
    std::copy_n(QIn, 5, QOut);
    QOut[1 + normal] = -QOut[1 + normal];
  }
};

// Shallow water with bathymetry as 4th variable (ApplicationExamples/SWE/SWE_ADERDG/MySWESolver.cpp:103-152),
// reflective wall boundary (:43-62). grav = 9.81.
struct SWEPDE {
  static constexpr int NumberOfVariables = 4;
  static constexpr double grav = 9.81;
  static void flux(const double* const Q, double** const F) {
    const double ih = 1. / Q[0];
    F[0][0] = Q[1];
    F[0][1] = Q[1] * Q[1] * ih + 0.5 * grav * Q[0] * Q[0];
    F[0][2] = Q[1] * Q[2] * ih;
    F[0][3] = 0.0;
    F[1][0] = Q[2];
    F[1][1] = Q[1] * Q[2] * ih;
    F[1][2] = Q[2] * Q[2] * ih + 0.5 * grav * Q[0] * Q[0];
    F[1][3] = 0.0;
#if DIMENSIONS == 3
    F[2][0] = F[2][1] = F[2][2] = F[2][3] = 0.0;
#endif
  }
  static void eigenvalues(const double* const Q, const int d, double* const lambda) {
    const double c = std::sqrt(grav * Q[0]);
    const double ih = 1. / Q[0];
    const double u_n = Q[d + 1] * ih;
    lambda[0] = u_n + c;
    lambda[1] = u_n - c;
    lambda[2] = u_n;
    lambda[3] = 0.0;
  }
  static void nonConservativeProduct(const double* const Q, const double* const gradQ, double* const BgradQ) {
    BgradQ[0] = 0.0;
    BgradQ[1] = grav * Q[0] * gradQ[0 * 4 + 3];
    BgradQ[2] = grav * Q[0] * gradQ[1 * 4 + 3];
    BgradQ[3] = 0.0;
  }
  static void wall(const double* QIn, int normal, double* QOut) {
    std::copy_n(QIn, 4, QOut);
    QOut[1 + normal] = -QOut[1 + normal];
  }
};

// Linear acoustics in flux form with per-node parameters rho = Q[4], c = Q[5]; the nonlinear
// functors the GPU path uses for this system (the reference's acoustic app is linear-only).
struct AcousticPDE {
  static constexpr int NumberOfVariables = 4;
  static constexpr bool HasSource = true;
  static void flux(const double* const Q, double** const F) {
    const double rho = Q[4], c = Q[5];
    const double K = rho * c * c;
    const double pr = Q[0] / rho;
    for (int d = 0; d < DIMENSIONS; d++) {
      F[d][0] = K * Q[1 + d];
      F[d][1] = d == 0 ? pr : 0.0;
      F[d][2] = d == 1 ? pr : 0.0;
      F[d][3] = d == 2 ? pr : 0.0;
    }
  }
  static void eigenvalues(const double* const Q, const int, double* const lambda) {
    lambda[0] = -Q[5];
    lambda[1] = 0.0;
    lambda[2] = 0.0;
    lambda[3] = Q[5];
  }
  static void nonConservativeProduct(const double* const, const double* const, double* const B) {
    std::fill_n(B, 4, 0.0);
  }
  static void wall(const double* QIn, int normal, double* QOut) {
    std::copy_n(QIn, 4, QOut);
    QOut[1 + normal] = -QOut[1 + normal];
  }
};

// Linear elasticity, velocity-stress form (v1 v2 v3 s11 s22 s33 s12 s13 s23), per-node
// rho, cp, cs = Q[9..11], in flux form.
struct ElasticPDE {
  static constexpr int NumberOfVariables = 9;
  static constexpr bool HasSource = true;
  static void flux(const double* const Q, double** const F) {
    const double rho = Q[9], cp = Q[10], cs = Q[11];
    const double mu = rho * cs * cs;
    const double lam = rho * cp * cp - 2.0 * mu;
    const double ir = 1.0 / rho;
    const double sg[3][3] = {{Q[3], Q[6], Q[7]}, {Q[6], Q[4], Q[8]}, {Q[7], Q[8], Q[5]}};
    for (int d = 0; d < DIMENSIONS; d++) {
      double* f = F[d];
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
  static void eigenvalues(const double* const Q, const int, double* const lambda) {
    const double cp = Q[10], cs = Q[11];
    const double l[9] = {-cp, -cs, -cs, 0.0, 0.0, 0.0, cs, cs, cp};
    std::copy_n(l, 9, lambda);
  }
  static void nonConservativeProduct(const double* const, const double* const, double* const B) {
    std::fill_n(B, 9, 0.0);
  }
  static void wall(const double* QIn, int, double* QOut) {
    std::copy_n(QIn, 9, QOut);
    for (int k = 0; k < 3; k++) QOut[k] = -QOut[k];
  }
};

// Advection-diffusion of three scalars with their own velocities and diffusivities: the test
// system of the viscous-flux path (useViscousFlux). viscousFlux F_d[m] = a_m,d Q[m] - nu_m dQ[m]/dx_d
// (gradQ[d][m] as the predictor passes it, 3d/spaceTimePredictorNonlinear.cpph:206-208);
// viscousEigenvalues nu_m. The GPU functor of the tests defines the same system.
struct AdvDiffPDE {
  static constexpr int NumberOfVariables = 3;
  static constexpr bool HasSource = false;
  static constexpr double a[3][3] = {{0.3, -0.2, 0.1}, {-0.5, 0.25, 0.4}, {0.0, 0.6, -0.3}};
  static constexpr double nu[3] = {0.01, 0.005, 0.02};
  static void flux(const double* const Q, double** const F) {
    for (int d = 0; d < DIMENSIONS; d++)
      for (int m = 0; m < 3; m++) F[d][m] = a[m][d] * Q[m];
  }
  static void viscousFlux(const double* const Q, const double* const gradQ, double** const F) {
    for (int d = 0; d < DIMENSIONS; d++)
      for (int m = 0; m < 3; m++) F[d][m] = a[m][d] * Q[m] - nu[m] * gradQ[d * 3 + m];
  }
  static void eigenvalues(const double* const, const int d, double* const lambda) {
    for (int m = 0; m < 3; m++) lambda[m] = a[m][d];
  }
  static void viscousEigenvalues(const double* const, const int, double* const lambda) {
    for (int m = 0; m < 3; m++) lambda[m] = nu[m];
  }
  static void nonConservativeProduct(const double* const, const double* const, double* const B) {
    std::fill_n(B, 3, 0.0);
  }
  static void wall(const double* QIn, int, double* QOut) { std::copy_n(QIn, 3, QOut); }
};
constexpr double AdvDiffPDE::a[3][3];
constexpr double AdvDiffPDE::nu[3];

// The same three advected scalars with a space-, time- and state-dependent algebraic source: the
// test system of the algebraicSource path (useSource). The GPU functor of the tests defines the same
// system.
struct AdvReactPDE {
  static constexpr int NumberOfVariables = 3;
  static constexpr bool HasSource = true;
  static void flux(const double* const Q, double** const F) { AdvDiffPDE::flux(Q, F); }
  static void eigenvalues(const double* const Q, const int d, double* const lambda) {
    AdvDiffPDE::eigenvalues(Q, d, lambda);
  }
  // x: 3 coordinates (z = 0 in 2D)
  static void algebraicSource(const double* x, double t, const double* const Q, double* S) {
    const double pi = 3.14159265358979323846;
    S[0] = -0.5 * Q[0] + 0.2 * Q[1] + 0.1 * std::sin(2.0 * pi * (x[0] + 2.0 * x[1] + 3.0 * x[2]) - t);
    S[1] = -0.3 * Q[1] * Q[2];
    S[2] = 0.05 * std::cos(2.0 * pi * x[0]) - 0.4 * Q[2];
  }
  static void nonConservativeProduct(const double* const, const double* const, double* const B) {
    std::fill_n(B, 3, 0.0);
  }
  static void wall(const double* QIn, int, double* QOut) { std::copy_n(QIn, 3, QOut); }
};

// Point source of the acoustic / elastic solvers (x, y, z, f0, t0, amplitude, width, variable):
// a unit-mass Gaussian of the given width times a Ricker wavelet, acting only on cells whose
// centre is within 6 widths plus a cell diagonal (the per-cell truncation the GPU path and the
// C restatement use). algebraicSource sees only the node, so the cell's verdict is handed to it
// through a thread-local flag set before each predictor call.
double g_src[8] = {0, 0, 0, 0, 0, 0, 1, 0};
int g_src_active = 0;
int g_bc_mode = 1;  // 1 reflective wall, 3 outflow
thread_local int tl_src_on = 0;

inline bool source_near(const double* centre, const double* dx) {
  if (!g_src_active) return false;
  double r2 = 0.0, h2 = 0.0;
  for (int d = 0; d < DIMENSIONS; d++) {
    r2 += (centre[d] - g_src[d]) * (centre[d] - g_src[d]);
    h2 += dx[d] * dx[d];
  }
  const double reach = 6.0 * g_src[6] + std::sqrt(h2);
  return r2 <= reach * reach;
}
inline double point_source(const double* x, double t) {
  const double pi = 3.14159265358979323846;
  double r2 = 0.0;
  for (int d = 0; d < DIMENSIONS; d++) r2 += (x[d] - g_src[d]) * (x[d] - g_src[d]);
  const double w = g_src[6];
  const double a = pi * g_src[3] * (t - g_src[4]);
  const double ricker = (1.0 - 2.0 * a * a) * std::exp(-a * a);
  const double norm = DIMENSIONS == 3 ? 1.0 / (15.749609945722419 * w * w * w) : 1.0 / (6.283185307179586 * w * w);
  return g_src[5] * ricker * std::exp(-0.5 * r2 / (w * w)) * norm;
}

// FIXED selects the reference's UseMaxPicardIterations mode: Order+1 sweeps, no residual test.
template <class PDE, int ORDER, int NPAR, bool FIXED = false>
struct RefSolver {
  static constexpr int Order = ORDER;
  static constexpr int NumberOfVariables = PDE::NumberOfVariables;
  static constexpr int NumberOfParameters = NPAR;
  static constexpr int MaxPicardIterations = ORDER + 1;
  static constexpr bool UseMaxPicardIterations = FIXED;
  static constexpr double CFL = 0.9;
  static constexpr double PNPM = kPNPM[ORDER];
  static constexpr bool UseLobattoBasis = false;
  static double** weights;
  static double** nodes;
  static double*** Kxi;
  static double*** dudx;
  static double*** iK1;
  static double*** FCoeff;

  void flux(const double* const Q, double** const F) { PDE::flux(Q, F); }
  void eigenvalues(const double* const Q, const int d, double* const l) { PDE::eigenvalues(Q, d, l); }
  void nonConservativeProduct(const double* const Q, const double* const g, double* const b) {
    PDE::nonConservativeProduct(Q, g, b);
  }
  void algebraicSource(const tarch::la::Vector<DIMENSIONS, double>& x, double t, const double* const,
                       double* S) {
    std::fill_n(S, NumberOfVariables, 0.0);
    if (tl_src_on) {
      double xs[3] = {0, 0, 0};
      for (int d = 0; d < DIMENSIONS; d++) xs[d] = x[d];
      S[(int)g_src[7]] = point_source(xs, t);
    }
  }
  void viscousFlux(const double* const, const double* const, double**) {}
  void viscousEigenvalues(const double* const, const int, double* const l) {
    std::fill_n(l, NumberOfVariables, 0.0);
  }
  // Reflective wall (mirrored normal momentum) or outflow (the inner state), and the flux of
  // that ghost state.
  void boundaryValues(const double* const, const double, const double, const int, const int normal,
                      const double* const, const double* const stateIn, const double* const,
                      double* const fluxOut, double* const stateOut) {
    if (g_bc_mode == 3)
      std::copy_n(stateIn, NumberOfVariables, stateOut);
    else
      PDE::wall(stateIn, normal, stateOut);
    for (int m = NumberOfVariables; m < NumberOfVariables + NPAR; m++) stateOut[m] = stateIn[m];
    double buf[3][NumberOfVariables];
    double* F[3] = {buf[0], buf[1], buf[2]};
    PDE::flux(stateOut, F);
    std::copy_n(F[normal], NumberOfVariables, fluxOut);
  }
};
template <class P, int O, int N, bool X> double** RefSolver<P, O, N, X>::weights = kernels::legendre::weights;
template <class P, int O, int N, bool X> double** RefSolver<P, O, N, X>::nodes = kernels::legendre::nodes;
template <class P, int O, int N, bool X> double*** RefSolver<P, O, N, X>::Kxi = kernels::legendre::Kxi;
template <class P, int O, int N, bool X> double*** RefSolver<P, O, N, X>::dudx = kernels::legendre::dudx;
template <class P, int O, int N, bool X> double*** RefSolver<P, O, N, X>::iK1 = kernels::legendre::iK1;
template <class P, int O, int N, bool X> double*** RefSolver<P, O, N, X>::FCoeff = kernels::legendre::FCoeff;

// The solver of a PDE with its own algebraic source (useSource = true): hides the base's point source.
template <class PDE, int ORDER>
struct RefSrcSolver : RefSolver<PDE, ORDER, 0> {
  void algebraicSource(const tarch::la::Vector<DIMENSIONS, double>& x, double t, const double* const Q, double* S) {
    double xs[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < DIMENSIONS; d++) xs[d] = x[d];
    PDE::algebraicSource(xs, t, Q, S);
  }
};

// The solver of a PDE with a viscous flux: the kernels call these members when instantiated with
// useViscousFlux = true (they hide the base's empty ones).
template <class PDE, int ORDER>
struct RefViscSolver : RefSolver<PDE, ORDER, 0> {
  void viscousFlux(const double* const Q, const double* const gradQ, double** const F) {
    PDE::viscousFlux(Q, gradQ, F);
  }
  void viscousEigenvalues(const double* const Q, const int d, double* const l) { PDE::viscousEigenvalues(Q, d, l); }
};

template <class S>
struct Sizes {
  static constexpr int n = S::Order + 1;
  static constexpr int v = S::NumberOfVariables;
  static constexpr int D = v + S::NumberOfParameters;
  static constexpr int nd = DIMENSIONS == 3 ? n * n * n : n * n;
  static constexpr int nf = DIMENSIONS == 3 ? n * n : n;  // nodes per face
  static constexpr int lQi = D * nd * n;
  static constexpr int lFi = (DIMENSIONS + 1) * v * nd * n;
  static constexpr int gradQ = DIMENSIONS * v * nd;
  static constexpr int lQhi = D * nd;
  static constexpr int lFhi = (DIMENSIONS + 1) * v * nd;
  static constexpr int luh = D * nd;
  static constexpr int lduh = v * nd;
  static constexpr int lQhbnd = 2 * DIMENSIONS * nf * D;
  static constexpr int lFhbnd = 2 * DIMENSIONS * nf * v;
};

inline tarch::la::Vector<DIMENSIONS, double> vec(const double* x) {
  tarch::la::Vector<DIMENSIONS, double> r;
  for (int d = 0; d < DIMENSIONS; d++) r[d] = x[d];
  return r;
}

// One whole cell predictor exactly as the generated glue does it
// (AbstractGenericADERDGSolverImplementation.template:168-211).
// VISC: useViscousFlux (the extrapolator then also writes the time-averaged gradient's face values).
template <class S, bool useNCP, bool useSource, bool VISC = false>
int predictor(S& s, const double* luh, const double* centre, const double* dx, double t, double dt,
              double* lQi, double* rhs, double* lFi, double* gradQ, double* lQhi, double* lFhi,
              double* lQhbnd, double* lFhbnd) {
  auto invDx = tarch::la::invertEntries(vec(dx));
  tl_src_on = useSource && source_near(centre, dx);
  std::vector<double> lGradQhbnd(VISC ? 2 * DIMENSIONS * Sizes<S>::nf * Sizes<S>::v * DIMENSIONS : 1);
  return kernels::aderdg::generic::c::spaceTimePredictorNonlinear<useSource, true, VISC, useNCP, false, S>(
      s, lQhbnd, VISC ? lGradQhbnd.data() : nullptr, lFhbnd, lQi, rhs, lFi, gradQ, lQhi, lFhi, luh, vec(centre),
      invDx, t, dt);
}

// Uniform patch driver in the global non-fused order: dt = min_cells stableTimeStepSize(luh)
// -> predictor + volume integral (all cells) -> Rusanov on all faces -> surface integral +
// solution update. Periodic in every direction unless `walls` is set (then every domain face goes
// through boundaryConditions: 1 reflective walls, 3 outflow, 3d/boundaryConditions.cpph:29-122 and glue
// :307-350). Cell c = (iz*ny + iy)*nx + ix. The reference's TBB/Peano scheduler is absent from
// the checkout; an OpenMP loop over cells and faces stands in for it.
template <class S, bool useNCP, bool useSource, bool VISC = false>
int run_patch(const int* ncell, const double* offset, const double* size, int walls, double* luh_all,
              int nsteps, double t0, double fixed_dt, double* t_out, double* dts, int* picard,
              int nthreads) {
  using Z = Sizes<S>;
  const int nx = ncell[0], ny = ncell[1], nz = DIMENSIONS == 3 ? ncell[2] : 1;
  const long nc = (long)nx * ny * nz;
  double dx[3] = {size[0] / nx, size[1] / ny, DIMENSIONS == 3 ? size[2] / nz : 1.0};
  std::vector<double> lduh(nc * Z::lduh), lQhbnd(nc * Z::lQhbnd), lFhbnd(nc * Z::lFhbnd);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  g_bc_mode = walls;
  double t = t0;
  auto cellIndex = [&](int ix, int iy, int iz) -> long { return ((long)iz * ny + iy) * nx + ix; };
  for (int step = 0; step < nsteps; step++) {
    double dt = std::numeric_limits<double>::max();
    if (fixed_dt > 0) {
      dt = fixed_dt;
    } else {
#pragma omp parallel for reduction(min : dt) schedule(static)
      for (long c = 0; c < nc; c++) {
        S s;
        dt = std::min(dt, kernels::aderdg::generic::c::stableTimeStepSize<S, VISC>(
                              s, luh_all + c * Z::luh, vec(dx)));
      }
    }
    long iters = 0;
#pragma omp parallel reduction(+ : iters)
    {
      std::vector<double> lQi(Z::lQi), rhs(Z::lQi), lFi(Z::lFi), gradQ(Z::gradQ), lQhi(Z::lQhi),
          lFhi(Z::lFhi);
      S s;
#pragma omp for schedule(static)
      for (long c = 0; c < nc; c++) {
        const int ix = c % nx, iy = (c / nx) % ny, iz = (int)(c / ((long)nx * ny));
        double centre[3] = {offset[0] + (ix + 0.5) * dx[0], offset[1] + (iy + 0.5) * dx[1],
                            DIMENSIONS == 3 ? offset[2] + (iz + 0.5) * dx[2] : 0.0};
        int it = predictor<S, useNCP, useSource, VISC>(s, luh_all + c * Z::luh, centre, dx, t, dt, lQi.data(),
                                      rhs.data(), lFi.data(), gradQ.data(), lQhi.data(), lFhi.data(),
                                      lQhbnd.data() + c * Z::lQhbnd, lFhbnd.data() + c * Z::lFhbnd);
        iters += it;
        if (picard) picard[(long)step * nc + c] = it;
        kernels::aderdg::generic::c::volumeIntegralNonlinear<S, useNCP || useSource, true, false, Z::v, Z::n>(
            lduh.data() + c * Z::lduh, lFhi.data(), vec(dx));
      }
    }
    // Riemann problems, one direction at a time so that no two faces touch the same cell face.
    for (int d = 0; d < DIMENSIONS; d++) {
#pragma omp parallel for schedule(static)
      for (long c = 0; c < nc; c++) {
        S s;
        const int ix = c % nx, iy = (c / nx) % ny, iz = (int)(c / ((long)nx * ny));
        int jx = ix, jy = iy, jz = iz;
        int lim = d == 0 ? nx : (d == 1 ? ny : nz);
        int& j = d == 0 ? jx : (d == 1 ? jy : jz);
        j += 1;
        double* FL = lFhbnd.data() + c * Z::lFhbnd + (2 * d + 1) * Z::nf * Z::v;
        const double* QL = lQhbnd.data() + c * Z::lQhbnd + (2 * d + 1) * Z::nf * Z::D;
        if (j == lim) {
          if (walls) {
            // right domain boundary of this cell
            std::vector<double> QOut(Z::nf * Z::D), FOut(Z::nf * Z::v);
            double centre[3] = {offset[0] + (ix + 0.5) * dx[0], offset[1] + (iy + 0.5) * dx[1],
                                DIMENSIONS == 3 ? offset[2] + (iz + 0.5) * dx[2] : 0.0};
            kernels::aderdg::generic::c::boundaryConditions<false, S>(
                s, FOut.data(), QOut.data(), FL, QL, nullptr, vec(centre), vec(dx), t, dt, 2 * d + 1, d);
            kernels::aderdg::generic::c::riemannSolverNonlinear<useNCP, VISC, S>(
                s, FL, FOut.data(), QL, QOut.data(), t, dt, vec(dx), d);
          } else {
            j = 0;
          }
        }
        if (j < lim) {
          long c2 = cellIndex(jx, jy, jz);
          double* FR = lFhbnd.data() + c2 * Z::lFhbnd + (2 * d) * Z::nf * Z::v;
          const double* QR = lQhbnd.data() + c2 * Z::lQhbnd + (2 * d) * Z::nf * Z::D;
          kernels::aderdg::generic::c::riemannSolverNonlinear<useNCP, VISC, S>(s, FL, FR, QL, QR, t, dt,
                                                                               vec(dx), d);
        }
        // left domain boundary of this cell
        int k = d == 0 ? ix : (d == 1 ? iy : iz);
        if (walls && k == 0) {
          double* FRb = lFhbnd.data() + c * Z::lFhbnd + (2 * d) * Z::nf * Z::v;
          const double* QRb = lQhbnd.data() + c * Z::lQhbnd + (2 * d) * Z::nf * Z::D;
          std::vector<double> QOut(Z::nf * Z::D), FOut(Z::nf * Z::v);
          double centre[3] = {offset[0] + (ix + 0.5) * dx[0], offset[1] + (iy + 0.5) * dx[1],
                              DIMENSIONS == 3 ? offset[2] + (iz + 0.5) * dx[2] : 0.0};
          kernels::aderdg::generic::c::boundaryConditions<false, S>(
              s, FOut.data(), QOut.data(), FRb, QRb, nullptr, vec(centre), vec(dx), t, dt, 2 * d, d);
          kernels::aderdg::generic::c::riemannSolverNonlinear<useNCP, VISC, S>(
              s, FOut.data(), FRb, QOut.data(), QRb, t, dt, vec(dx), d);
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
      S s;
      kernels::aderdg::generic::c::surfaceIntegralNonlinear<S, Z::v, Z::n>(
          lduh.data() + c * Z::lduh, lFhbnd.data() + c * Z::lFhbnd, vec(dx));
      kernels::aderdg::generic::c::solutionUpdate<S>(s, luh_all + c * Z::luh, luh_all + c * Z::luh,
                                                     lduh.data() + c * Z::lduh, dt);
    }
    if (dts) dts[step] = dt;
    t += dt;
    (void)iters;
  }
  if (t_out) *t_out = t;
  return 0;
}

#if DIMENSIONS == 3
// ---------------------------------------------------------------------------------------------
// Linear ADER-DG: the reference's linear generic kernels (3d/spaceTimePredictorLinear.cpph:30-647,
// Cauchy-Kowalewski; 3d/riemannSolverLinear.cpph:22-160; 3d/volumeIntegralLinear.cpph,
// 3d/surfaceIntegralLinear.cpph; 3d/deltaDistribution.cpph for point sources) with the PDE terms of
// the reference's own linear applications, in the pointer-array form the linear kernels call
// (AbstractGenericADERDGSolverImplementation.template:473-480). A second, independent scheme for the
// acoustic and elastic systems: the nonlinear path here integrates the same physics with a Picard
// predictor, Rusanov fluxes and flux-form functors.
//
// LinElastic: ApplicationExamples/Linear/ElasticWave3D/MyElasticWaveSolver.cpp, eigenvalues
// :190-208, flux :211-252, nonConservativeProduct :255-297, multiplyMaterialParameterMatrix
// :331-381 (variables v1 v2 v3 s11 s22 s33 s12 s13 s23, parameters rho cp cs). That file does not
// compile against its own header (riemannSolver is declared with a lengthScale argument in
// MyElasticWaveSolver.h and defined without one at :383), so its PDE terms are restated here.
// LinAcoustic: ApplicationExamples/AcousticWave/acousticwaveCPP/MyAcousticWaveSolver.cpp,
// eigenvalues :35-44, flux :46-61 (zero), nonConservativeProduct :97-156 (unit density and sound
// speed, no parameters; its velocity is minus the flux-form velocity).
struct LinElastic {
  static constexpr int NumberOfVariables = 9;
  static constexpr int NumberOfParameters = 3;
  static constexpr bool kFlux = true, kNCP = true, kMM = true;
  static void eigenvalues(const double* const Q, const int, double* const l) {
    const double cp = Q[10], cs = Q[11];
    const double e[9] = {cp, cs, cs, -cp, -cs, -cs, 0.0, 0.0, 0.0};
    std::copy_n(e, 9, l);
  }
  static void flux(const double* const Q, double** const F) {
    const double sxx = Q[3], syy = Q[4], szz = Q[5], sxy = Q[6], sxz = Q[7], syz = Q[8];
    const double f[3][3] = {{-sxx, -sxy, -sxz}, {-sxy, -syy, -syz}, {-sxz, -syz, -szz}};
    for (int d = 0; d < 3; d++) {
      std::fill_n(F[d], 9, 0.0);
      for (int k = 0; k < 3; k++) F[d][k] = f[d][k];
    }
  }
  static void ncp(const double* const, const double* const* const G, double** const B) {
    const double ux = G[0][0], vx = G[0][1], wx = G[0][2];
    const double uy = G[1][0], vy = G[1][1], wy = G[1][2];
    const double uz = G[2][0], vz = G[2][1], wz = G[2][2];
    for (int d = 0; d < 3; d++) std::fill_n(B[d], 9, 0.0);
    B[0][3] = -ux; B[0][6] = -vx; B[0][7] = -wx;
    B[1][4] = -vy; B[1][6] = -uy; B[1][8] = -wy;
    B[2][5] = -wz; B[2][7] = -uz; B[2][8] = -vz;
  }
  static void mm(const double* const Q, double** const rhs) {
    const double rho = Q[9], cp = Q[10], cs = Q[11];
    const double mu = rho * cs * cs;
    const double lambda = rho * cp * cp - 2 * mu;
    const double rho_inv = 1.0 / rho;
    for (int d = 0; d < 3; d++) {
      double* r = rhs[d];
      r[0] = rho_inv * r[0];
      r[1] = rho_inv * r[1];
      r[2] = rho_inv * r[2];
      const double lam_temp = lambda * (r[3] + r[4] + r[5]);
      r[3] = (2 * mu) * r[3] + lam_temp;
      r[4] = (2 * mu) * r[4] + lam_temp;
      r[5] = (2 * mu) * r[5] + lam_temp;
      r[6] = mu * r[6];
      r[7] = mu * r[7];
      r[8] = mu * r[8];
    }
  }
};

struct LinAcoustic {
  static constexpr int NumberOfVariables = 4;
  static constexpr int NumberOfParameters = 0;
  static constexpr bool kFlux = false, kNCP = true, kMM = false;
  static void eigenvalues(const double* const, const int, double* const l) {
    l[0] = 1.0;
    l[1] = -1.0;
    l[2] = 0.0;
    l[3] = 0.0;
  }
  static void flux(const double* const, double** const F) {
    for (int d = 0; d < 3; d++) std::fill_n(F[d], 4, 0.0);
  }
  static void ncp(const double* const, const double* const* const G, double** const B) {
    for (int d = 0; d < 3; d++) std::fill_n(B[d], 4, 0.0);
    B[0][0] = -G[0][1];
    B[0][1] = -G[0][0];
    B[1][0] = -G[1][2];
    B[1][2] = -G[1][0];
    B[2][0] = -G[2][3];
    B[2][3] = -G[2][0];
  }
  static void mm(const double* const, double** const) {}
};

// One point source at (g_src[0..2]) on variable g_src[7]: amplitude g_src[5] times the Ricker
// wavelet of peak frequency g_src[3] delayed by g_src[4] -- the time function of the
// regularised source of the nonlinear path, here as an exact delta distribution in space.
inline double ricker(double t) {
  const double pi = 3.14159265358979323846;
  const double a = pi * g_src[3] * (t - g_src[4]);
  return (1.0 - 2.0 * a * a) * std::exp(-a * a);
}

template <class PDE, int ORDER>
struct LinSolver {
  static constexpr int Order = ORDER;
  static constexpr int NumberOfVariables = PDE::NumberOfVariables;
  static constexpr int NumberOfParameters = PDE::NumberOfParameters;
  static constexpr int NumberOfPointSources = 1;
  static constexpr bool UseLobattoBasis = false;
  static constexpr double CFL = 0.9;
  static constexpr double PNPM = kPNPM[ORDER];
  static double** weights;
  static double** nodes;
  static double*** dudx;
  static double*** FCoeff;
  static kernels::UnivariateFunction** basisFunction;
  double pointSourceLocation[1][3];

  LinSolver() {
    for (int d = 0; d < 3; d++) pointSourceLocation[0][d] = g_src[d];
  }
  void eigenvalues(const double* const Q, const int d, double* const l) { PDE::eigenvalues(Q, d, l); }
  void viscousEigenvalues(const double* const, const int, double* const l) { std::fill_n(l, NumberOfVariables, 0.0); }
  void flux(const double* const Q, double** const F) { PDE::flux(Q, F); }
  void nonConservativeProduct(const double* const Q, const double* const* const G, double** const B) {
    PDE::ncp(Q, G, B);
  }
  void multiplyMaterialParameterMatrix(const double* const Q, double** const rhs) { PDE::mm(Q, rhs); }
  void algebraicSource(const tarch::la::Vector<DIMENSIONS, double>&, double, const double* const, double* S) {
    std::fill_n(S, NumberOfVariables, 0.0);
  }
  void pointSource(const double* const, const double* const, const double t, const double, double* const f, int) {
    std::fill_n(f, NumberOfVariables, 0.0);
    f[(int)g_src[7]] = g_src[5] * ricker(t);
  }
};
template <class P, int O> double** LinSolver<P, O>::weights = kernels::legendre::weights;
template <class P, int O> double** LinSolver<P, O>::nodes = kernels::legendre::nodes;
template <class P, int O> double*** LinSolver<P, O>::dudx = kernels::legendre::dudx;
template <class P, int O> double*** LinSolver<P, O>::FCoeff = kernels::legendre::FCoeff;
template <class P, int O> kernels::UnivariateFunction** LinSolver<P, O>::basisFunction = kernels::legendre::basisFunction;

// Periodic uniform patch in the order of the generated glue for linear solvers
// (AbstractGenericADERDGSolverImplementation.template:114-165 and :296-297): dt = min over cells
// of stableTimeStepSize (or fixed) -> per cell getPointSources / deltaDistribution, the
// Cauchy-Kowalewski predictor and the volume integral -> linear Riemann solver on every face ->
// surface integral + solution update. Cell c = (iz*ny + iy)*nx + ix; an OpenMP loop over cells
// stands in for the absent Peano scheduler.
template <class S>
int run_patch_linear(const int* ncell, const double* offset, const double* size, double* luh_all, int nsteps,
                     double t0, double fixed_dt, double* t_out, double* dts, int nthreads) {
  using PDE = typename std::conditional<S::NumberOfVariables == 9, LinElastic, LinAcoustic>::type;
  constexpr int n = S::Order + 1, v = S::NumberOfVariables, D = v + S::NumberOfParameters;
  constexpr int nd = n * n * n, nf = n * n;
  constexpr int sLQi = D * nd * (n + 1), sLFi = 4 * v * nd * n, sGradQ = 3 * v * nd;
  constexpr int sPSi = v * nd * (n + 1), sPSd = v * nd * n, sLQhi = D * nd, sLFhi = 4 * v * nd;
  constexpr int sLuh = D * nd, sLduh = v * nd, sQb = 6 * nf * D, sFb = 6 * nf * v;
  const int nx = ncell[0], ny = ncell[1], nz = ncell[2];
  const long nc = (long)nx * ny * nz;
  const double dx[3] = {size[0] / nx, size[1] / ny, size[2] / nz};
  std::vector<double> lduh(nc * sLduh), lQhbnd(nc * sQb), lFhbnd(nc * sFb);
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  auto cellIndex = [&](int ix, int iy, int iz) -> long { return ((long)iz * ny + iy) * nx + ix; };
  double t = t0;
  for (int step = 0; step < nsteps; step++) {
    double dt = std::numeric_limits<double>::max();
    if (fixed_dt > 0) {
      dt = fixed_dt;
    } else {
#pragma omp parallel for reduction(min : dt) schedule(static)
      for (long c = 0; c < nc; c++) {
        S s;
        dt = std::min(dt, kernels::aderdg::generic::c::stableTimeStepSize<S, false>(s, luh_all + c * sLuh, vec(dx)));
      }
    }
#pragma omp parallel
    {
      std::vector<double> lQi(sLQi), lFi(sLFi), gradQ(sGradQ), PSi(sPSi), PSd(sPSd), tmpPSd(sPSd), lQhi(sLQhi),
          lFhi(sLFhi);
      S s;
#pragma omp for schedule(static)
      for (long c = 0; c < nc; c++) {
        const int ix = c % nx, iy = (c / nx) % ny, iz = (int)(c / ((long)nx * ny));
        const double centre[3] = {offset[0] + (ix + 0.5) * dx[0], offset[1] + (iy + 0.5) * dx[1],
                                  offset[2] + (iz + 0.5) * dx[2]};
        const double* luh = luh_all + c * sLuh;
        const auto ctr = vec(centre), cdx = vec(dx);
        const auto invDx = tarch::la::invertEntries(cdx);
        std::vector<int>* ps = g_src_active ? kernels::aderdg::generic::c::getPointSources<S>(s, ctr, cdx) : nullptr;
        if (ps != nullptr) {
          kernels::aderdg::generic::c::deltaDistribution<S>(s, luh, t, dt, ctr, cdx, ps, PSi.data());
          kernels::aderdg::generic::c::spaceTimePredictorLinear<true, false, PDE::kFlux, PDE::kNCP, PDE::kMM, S>(
              s, lQhbnd.data() + c * sQb, lFhbnd.data() + c * sFb, lQi.data(), lFi.data(), gradQ.data(), PSi.data(),
              PSd.data(), tmpPSd.data(), lQhi.data(), lFhi.data(), luh, ctr, invDx, t, dt);
        } else {
          kernels::aderdg::generic::c::spaceTimePredictorLinear<false, false, PDE::kFlux, PDE::kNCP, PDE::kMM, S>(
              s, lQhbnd.data() + c * sQb, lFhbnd.data() + c * sFb, lQi.data(), lFi.data(), gradQ.data(), PSi.data(),
              PSd.data(), tmpPSd.data(), lQhi.data(), lFhi.data(), luh, ctr, invDx, t, dt);
        }
        kernels::aderdg::generic::c::volumeIntegralLinear<S, false, PDE::kFlux, v, n>(lduh.data() + c * sLduh,
                                                                                      lFhi.data(), cdx);
      }
    }
    // one direction at a time, so that no two faces write the same cell face
    for (int d = 0; d < 3; d++) {
#pragma omp parallel for schedule(static)
      for (long c = 0; c < nc; c++) {
        S s;
        const int ix = c % nx, iy = (c / nx) % ny, iz = (int)(c / ((long)nx * ny));
        int j[3] = {ix, iy, iz};
        const int lim = d == 0 ? nx : (d == 1 ? ny : nz);
        j[d] = (j[d] + 1) % lim;
        const long c2 = cellIndex(j[0], j[1], j[2]);
        kernels::aderdg::generic::c::riemannSolverLinear<PDE::kFlux, PDE::kNCP, PDE::kMM, S>(
            s, lFhbnd.data() + c * sFb + (2 * d + 1) * nf * v, lFhbnd.data() + c2 * sFb + (2 * d) * nf * v,
            lQhbnd.data() + c * sQb + (2 * d + 1) * nf * D, lQhbnd.data() + c2 * sQb + (2 * d) * nf * D, t, dt, d);
      }
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
      S s;
      kernels::aderdg::generic::c::surfaceIntegralLinear<S, v, n>(lduh.data() + c * sLduh, lFhbnd.data() + c * sFb,
                                                                  vec(dx));
      kernels::aderdg::generic::c::solutionUpdate<S>(s, luh_all + c * sLuh, luh_all + c * sLuh,
                                                     lduh.data() + c * sLduh, dt);
    }
    if (dts) dts[step] = dt;
    t += dt;
  }
  if (t_out) *t_out = t;
  return 0;
}
#endif

}  // namespace exaref

#if DIMENSIONS == 3
// The reference applications' PDE terms applied to a linear field (state Q with its material
// parameters, per-direction gradients G[d][0..v)): out[d] = M(Q) (F_d(G_d) + B_d(G)), the d-th
// term of -dQ/dt in the linear kernels' convention (3d/spaceTimePredictorLinear.cpph:183-345).
#define EXALIN_DEFINE(NAME, PDE, O)                                                                          \
  extern "C" int NAME##_run(const int* ncell, const double* offset, const double* size, double* luh,       \
                            int nsteps, double t0, double fixed_dt, double* t_out, double* dts, int nthreads) { \
    return exaref::run_patch_linear<exaref::LinSolver<exaref::PDE, O>>(ncell, offset, size, luh, nsteps, t0,  \
                                                                       fixed_dt, t_out, dts, nthreads);     \
  }
EXALIN_DEFINE(exalin_elastic_o3, LinElastic, 3)
EXALIN_DEFINE(exalin_elastic_o4, LinElastic, 4)
EXALIN_DEFINE(exalin_acoustic_o3, LinAcoustic, 3)
EXALIN_DEFINE(exalin_acoustic_o4, LinAcoustic, 4)

template <class PDE>
static void exalin_terms_impl(const double* Q, const double* G, double* out) {
  constexpr int v = PDE::NumberOfVariables;
  double fbuf[3][v], nbuf[3][v];
  double* F[3] = {fbuf[0], fbuf[1], fbuf[2]};
  double* B[3] = {nbuf[0], nbuf[1], nbuf[2]};
  const double* Gp[3] = {G, G + v, G + 2 * v};
  for (int d = 0; d < 3; d++) {
    // the flux of the d-th gradient (the flux terms are linear in the variables)
    double q[v + PDE::NumberOfParameters + 1];
    for (int m = 0; m < v; m++) q[m] = G[d * v + m];
    for (int m = v; m < v + PDE::NumberOfParameters; m++) q[m] = Q[m];
    double tb[3][v];
    double* T[3] = {tb[0], tb[1], tb[2]};
    PDE::flux(q, T);
    std::copy_n(tb[d], v, fbuf[d]);
  }
  PDE::ncp(Q, Gp, B);
  double rbuf[3][v];
  double* R[3] = {rbuf[0], rbuf[1], rbuf[2]};
  for (int d = 0; d < 3; d++)
    for (int m = 0; m < v; m++) rbuf[d][m] = (PDE::kFlux ? fbuf[d][m] : 0.0) + (PDE::kNCP ? nbuf[d][m] : 0.0);
  if (PDE::kMM) PDE::mm(Q, R);
  for (int d = 0; d < 3; d++) std::copy_n(rbuf[d], v, out + d * v);
}
extern "C" void exalin_elastic_terms(const double* Q, const double* G, double* out) {
  exalin_terms_impl<exaref::LinElastic>(Q, G, out);
}
extern "C" void exalin_acoustic_terms(const double* Q, const double* G, double* out) {
  exalin_terms_impl<exaref::LinAcoustic>(Q, G, out);
}
extern "C" void exalin_eigenvalues(int elastic, const double* Q, double* l) {
  if (elastic)
    exaref::LinElastic::eigenvalues(Q, 0, l);
  else
    exaref::LinAcoustic::eigenvalues(Q, 0, l);
}
#endif

#define EXAREF_S(PDE, O, P, X) exaref::RefSolver<exaref::PDE, O, P, X>
#define EXAREF_DEFINE(NAME, PDE, O, P, NCP) EXAREF_DEFINE_S(NAME, PDE, O, P, NCP, false, false)
#define EXAREF_DEFINE_S(NAME, PDE, O, P, NCP, SRC, FIXED) \
  EXAREF_DEFINE_G(NAME, EXAREF_S(PDE, O, P, FIXED), exaref::PDE::NumberOfVariables, O, NCP, SRC, false)
// a PDE with its own algebraic source (useSource = true), no parameters
#define EXAREF_DEFINE_A(NAME, PDE, O) \
  EXAREF_DEFINE_G(NAME, exaref::RefSrcSolver<exaref::PDE COMMA O>, exaref::PDE::NumberOfVariables, O, false, true, false)
// a PDE with a viscous flux (useViscousFlux = true), no parameters
#define EXAREF_DEFINE_V(NAME, PDE, O) \
  EXAREF_DEFINE_G(NAME, exaref::RefViscSolver<exaref::PDE COMMA O>, exaref::PDE::NumberOfVariables, O, false, false, true)
#define COMMA ,
// ST: the SolverType; NV: its NumberOfVariables
#define EXAREF_DEFINE_G(NAME, ST, NV, O, NCP, SRC, VISC)                                                    \
  extern "C" int NAME##_predictor(const double* luh, const double* centre, const double* dx, double t,     \
                                  double dt, double* lQi, double* rhs, double* lFi, double* gradQ,          \
                                  double* lQhi, double* lFhi, double* lQhbnd, double* lFhbnd) {             \
    ST s;                                                                                                   \
    return exaref::predictor<ST, NCP, SRC, VISC>(s, luh, centre, dx, t, dt, lQi, rhs, lFi, gradQ, lQhi,    \
                                                 lFhi, lQhbnd, lFhbnd);                                     \
  }                                                                                                         \
  extern "C" void NAME##_volume(double* lduh, const double* lFhi, const double* dx) {                        \
    kernels::aderdg::generic::c::volumeIntegralNonlinear<ST, NCP || SRC, true, false, NV, O + 1>(           \
        lduh, lFhi, exaref::vec(dx));                                                                       \
  }                                                                                                         \
  extern "C" void NAME##_riemann(double* FL, double* FR, const double* QL, const double* QR, double t,      \
                                 double dt, const double* dx, int direction) {                              \
    ST s;                                                                                                   \
    kernels::aderdg::generic::c::riemannSolverNonlinear<NCP, VISC, ST>(s, FL, FR, QL, QR, t, dt,           \
                                                                       exaref::vec(dx), direction);         \
  }                                                                                                         \
  extern "C" void NAME##_surface(double* lduh, const double* lFhbnd, const double* dx) {                    \
    kernels::aderdg::generic::c::surfaceIntegralNonlinear<ST, NV, O + 1>(lduh, lFhbnd, exaref::vec(dx));   \
  }                                                                                                         \
  extern "C" void NAME##_face(double* lduh, const double* lFhbnd, int direction, int orientation,           \
                              const double* dx) {                                                           \
    kernels::aderdg::generic::c::faceIntegralNonlinear<ST, NV, O + 1>(lduh, lFhbnd, direction, orientation, \
                                                                      exaref::vec(dx));                     \
  }                                                                                                         \
  extern "C" void NAME##_update(double* luh, const double* luhOld, const double* lduh, double dt) {        \
    ST s;                                                                                                   \
    kernels::aderdg::generic::c::solutionUpdate<ST>(s, luh, luhOld, lduh, dt);                              \
  }                                                                                                         \
  extern "C" double NAME##_dt(const double* luh, const double* dx) {                                        \
    ST s;                                                                                                   \
    return kernels::aderdg::generic::c::stableTimeStepSize<ST, VISC>(s, luh, exaref::vec(dx));            \
  }                                                                                                         \
  extern "C" void NAME##_boundary(double* FOut, double* QOut, const double* FIn, const double* QIn,        \
                                  const double* centre, const double* dx, double t, double dt,              \
                                  int faceIndex, int normal) {                                              \
    ST s;                                                                                                   \
    kernels::aderdg::generic::c::boundaryConditions<false, ST>(s, FOut, QOut, FIn, QIn, nullptr,            \
                                                               exaref::vec(centre), exaref::vec(dx), t, dt, \
                                                               faceIndex, normal);                          \
  }                                                                                                         \
  extern "C" int NAME##_run(const int* ncell, const double* offset, const double* size, int walls,         \
                            double* luh, int nsteps, double t0, double fixed_dt, double* t_out,             \
                            double* dts, int* picard, int nthreads) {                                       \
    return exaref::run_patch<ST, NCP, SRC, VISC>(ncell, offset, size, walls, luh, nsteps, t0, fixed_dt,    \
                                                 t_out, dts, picard, nthreads);                             \
  }

extern "C" void exaref_set_source(const double* src, int active) {
  for (int k = 0; k < 8; k++) exaref::g_src[k] = src[k];
  exaref::g_src_active = active;
}
extern "C" void exaref_set_boundary(int mode) { exaref::g_bc_mode = mode; }

#if DIMENSIONS == 3
EXAREF_DEFINE_S(exaref3d_acoustic_o4_p2, AcousticPDE, 4, 2, false, true, false)
EXAREF_DEFINE_S(exaref3d_elastic_o3_p3, ElasticPDE, 3, 3, false, true, false)
EXAREF_DEFINE_S(exaref3d_acousticfixed_o4_p2, AcousticPDE, 4, 2, false, true, true)
EXAREF_DEFINE_S(exaref3d_elasticfixed_o3_p3, ElasticPDE, 3, 3, false, true, true)
EXAREF_DEFINE_S(exaref3d_elastic_o7_p3, ElasticPDE, 7, 3, false, true, false)
EXAREF_DEFINE(exaref3d_euler_o3_p0, EulerPDE, 3, 0, false)
EXAREF_DEFINE(exaref3d_euler_o3_p1, EulerPDE, 3, 1, false)
EXAREF_DEFINE(exaref3d_euler_o5_p0, EulerPDE, 5, 0, false)
EXAREF_DEFINE(exaref3d_euler_o2_p0, EulerPDE, 2, 0, false)
EXAREF_DEFINE_V(exaref3d_advdiff_o3_p0, AdvDiffPDE, 3)
EXAREF_DEFINE_A(exaref3d_advreact_o3_p0, AdvReactPDE, 3)
#else
EXAREF_DEFINE(exaref2d_euler_o3_p0, EulerPDE, 3, 0, false)
EXAREF_DEFINE(exaref2d_euler_o3_p1, EulerPDE, 3, 1, false)
EXAREF_DEFINE(exaref2d_euler_o5_p0, EulerPDE, 5, 0, false)
EXAREF_DEFINE(exaref2d_swe_o4_p0, SWEPDE, 4, 0, true)
EXAREF_DEFINE(exaref2d_swe_o2_p0, SWEPDE, 2, 0, true)
EXAREF_DEFINE_V(exaref2d_advdiff_o3_p0, AdvDiffPDE, 3)
EXAREF_DEFINE_A(exaref2d_advreact_o3_p0, AdvReactPDE, 3)
#endif
