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
template <class S, bool useNCP, bool useSource>
int predictor(S& s, const double* luh, const double* centre, const double* dx, double t, double dt,
              double* lQi, double* rhs, double* lFi, double* gradQ, double* lQhi, double* lFhi,
              double* lQhbnd, double* lFhbnd) {
  auto invDx = tarch::la::invertEntries(vec(dx));
  tl_src_on = useSource && source_near(centre, dx);
  return kernels::aderdg::generic::c::spaceTimePredictorNonlinear<useSource, true, false, useNCP, false, S>(
      s, lQhbnd, nullptr, lFhbnd, lQi, rhs, lFi, gradQ, lQhi, lFhi, luh, vec(centre), invDx, t, dt);
}

// Uniform patch driver in the global non-fused order: dt = min_cells stableTimeStepSize(luh)
// -> predictor + volume integral (all cells) -> Rusanov on all faces -> surface integral +
// solution update. Periodic in every direction unless `walls` is set (then every domain face goes
// through boundaryConditions: 1 reflective walls, 3 outflow, 3d/boundaryConditions.cpph:29-122 and glue
// :307-350). Cell c = (iz*ny + iy)*nx + ix. The reference's TBB/Peano scheduler is absent from
// the checkout; an OpenMP loop over cells and faces stands in for it.
template <class S, bool useNCP, bool useSource>
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
        dt = std::min(dt, kernels::aderdg::generic::c::stableTimeStepSize<S, false>(
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
        int it = predictor<S, useNCP, useSource>(s, luh_all + c * Z::luh, centre, dx, t, dt, lQi.data(),
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
            kernels::aderdg::generic::c::riemannSolverNonlinear<useNCP, false, S>(
                s, FL, FOut.data(), QL, QOut.data(), t, dt, vec(dx), d);
          } else {
            j = 0;
          }
        }
        if (j < lim) {
          long c2 = cellIndex(jx, jy, jz);
          double* FR = lFhbnd.data() + c2 * Z::lFhbnd + (2 * d) * Z::nf * Z::v;
          const double* QR = lQhbnd.data() + c2 * Z::lQhbnd + (2 * d) * Z::nf * Z::D;
          kernels::aderdg::generic::c::riemannSolverNonlinear<useNCP, false, S>(s, FL, FR, QL, QR, t, dt,
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
          kernels::aderdg::generic::c::riemannSolverNonlinear<useNCP, false, S>(
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

}  // namespace exaref

#define EXAREF_S(PDE, O, P, X) exaref::RefSolver<exaref::PDE, O, P, X>
#define EXAREF_DEFINE(NAME, PDE, O, P, NCP) EXAREF_DEFINE_S(NAME, PDE, O, P, NCP, false, false)
#define EXAREF_DEFINE_S(NAME, PDE, O, P, NCP, SRC, FIXED)                                               \
  extern "C" int NAME##_predictor(const double* luh, const double* centre, const double* dx, double t,     \
                                  double dt, double* lQi, double* rhs, double* lFi, double* gradQ,          \
                                  double* lQhi, double* lFhi, double* lQhbnd, double* lFhbnd) {             \
    EXAREF_S(PDE, O, P, FIXED) s;                                                                                  \
    return exaref::predictor<EXAREF_S(PDE, O, P, FIXED), NCP, SRC>(s, luh, centre, dx, t, dt, lQi, rhs, lFi, gradQ,     \
                                                       lQhi, lFhi, lQhbnd, lFhbnd);                         \
  }                                                                                                         \
  extern "C" void NAME##_volume(double* lduh, const double* lFhi, const double* dx) {                        \
    kernels::aderdg::generic::c::volumeIntegralNonlinear<EXAREF_S(PDE, O, P, FIXED), NCP || SRC, true, false,      \
                                                         exaref::PDE::NumberOfVariables, O + 1>(            \
        lduh, lFhi, exaref::vec(dx));                                                                       \
  }                                                                                                         \
  extern "C" void NAME##_riemann(double* FL, double* FR, const double* QL, const double* QR, double t,      \
                                 double dt, const double* dx, int direction) {                              \
    EXAREF_S(PDE, O, P, FIXED) s;                                                                                  \
    kernels::aderdg::generic::c::riemannSolverNonlinear<NCP, false, EXAREF_S(PDE, O, P, FIXED)>(                   \
        s, FL, FR, QL, QR, t, dt, exaref::vec(dx), direction);                                              \
  }                                                                                                         \
  extern "C" void NAME##_surface(double* lduh, const double* lFhbnd, const double* dx) {                    \
    kernels::aderdg::generic::c::surfaceIntegralNonlinear<EXAREF_S(PDE, O, P, FIXED),                              \
                                                          exaref::PDE::NumberOfVariables, O + 1>(           \
        lduh, lFhbnd, exaref::vec(dx));                                                                     \
  }                                                                                                         \
  extern "C" void NAME##_face(double* lduh, const double* lFhbnd, int direction, int orientation,           \
                              const double* dx) {                                                           \
    kernels::aderdg::generic::c::faceIntegralNonlinear<EXAREF_S(PDE, O, P, FIXED), exaref::PDE::NumberOfVariables, \
                                                       O + 1>(lduh, lFhbnd, direction, orientation,         \
                                                              exaref::vec(dx));                             \
  }                                                                                                         \
  extern "C" void NAME##_update(double* luh, const double* luhOld, const double* lduh, double dt) {        \
    EXAREF_S(PDE, O, P, FIXED) s;                                                                                  \
    kernels::aderdg::generic::c::solutionUpdate<EXAREF_S(PDE, O, P, FIXED)>(s, luh, luhOld, lduh, dt);             \
  }                                                                                                         \
  extern "C" double NAME##_dt(const double* luh, const double* dx) {                                        \
    EXAREF_S(PDE, O, P, FIXED) s;                                                                                  \
    return kernels::aderdg::generic::c::stableTimeStepSize<EXAREF_S(PDE, O, P, FIXED), false>(s, luh,              \
                                                                                       exaref::vec(dx));    \
  }                                                                                                         \
  extern "C" void NAME##_boundary(double* FOut, double* QOut, const double* FIn, const double* QIn,        \
                                  const double* centre, const double* dx, double t, double dt,              \
                                  int faceIndex, int normal) {                                              \
    EXAREF_S(PDE, O, P, FIXED) s;                                                                                  \
    kernels::aderdg::generic::c::boundaryConditions<false, EXAREF_S(PDE, O, P, FIXED)>(                            \
        s, FOut, QOut, FIn, QIn, nullptr, exaref::vec(centre), exaref::vec(dx), t, dt, faceIndex, normal);  \
  }                                                                                                         \
  extern "C" int NAME##_run(const int* ncell, const double* offset, const double* size, int walls,         \
                            double* luh, int nsteps, double t0, double fixed_dt, double* t_out,             \
                            double* dts, int* picard, int nthreads) {                                       \
    return exaref::run_patch<EXAREF_S(PDE, O, P, FIXED), NCP, SRC>(ncell, offset, size, walls, luh, nsteps, t0,         \
                                                       fixed_dt, t_out, dts, picard, nthreads);             \
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
#else
EXAREF_DEFINE(exaref2d_euler_o3_p0, EulerPDE, 3, 0, false)
EXAREF_DEFINE(exaref2d_euler_o3_p1, EulerPDE, 3, 1, false)
EXAREF_DEFINE(exaref2d_euler_o5_p0, EulerPDE, 5, 0, false)
EXAREF_DEFINE(exaref2d_swe_o4_p0, SWEPDE, 4, 0, true)
EXAREF_DEFINE(exaref2d_swe_o2_p0, SWEPDE, 2, 0, true)
#endif
