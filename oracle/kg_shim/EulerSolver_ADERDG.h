// The user-solver class the reference's generated optimised kernels are written against
// (KernelGenerator output includes "EulerSolver_ADERDG.h" and calls its hooks), for the Euler
// application's PDE (ApplicationExamples/Euler/Euler_ADERDG/EulerSolver_ADERDG.cpp:61-146,
// gamma 1.4) with an outflow boundary: the outer state is the inner one, its flux the normal flux
// of that state (as the generic-kernel checker's glue does). CHECKER / BASELINE ONLY.
// KG_PNPM is the PNPM of the generated order (Toolkit/exahype/toolkit/solverController.py:17-23).
#pragma once
#include <algorithm>
#include <cmath>

namespace Euler {
class EulerSolver_ADERDG {
 public:
  static constexpr int NumberOfVariables = 5;
  static constexpr int NumberOfParameters = 0;
  static constexpr double CFL = 0.9;
  static constexpr double PNPM = KG_PNPM;

  void flux(const double* const Q, double** const F) {
    const double gamma = 1.4;
    const double irho = 1.0 / Q[0];
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]));
    for (int d = 0; d < 3; d++) {
      double* f = F[d];
      const double un = Q[1 + d];
      f[0] = un;
      f[1] = irho * Q[1] * un;
      f[2] = irho * Q[2] * un;
      f[3] = irho * Q[3] * un;
      f[1 + d] += p;
      f[4] = irho * (Q[4] + p) * un;
    }
  }
  void eigenvalues(const double* const Q, const int d, double* const lambda) {
    const double gamma = 1.4;
    const double irho = 1.0 / Q[0];
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]));
    const double u_n = Q[d + 1] * irho;
    const double c = std::sqrt(gamma * p * irho);
    std::fill_n(lambda, 5, u_n);
    lambda[0] -= c;
    lambda[4] += c;
  }
  void adjustPointSolution(const double* const, const double, const double, double* const) {}
  void boundaryValues(const double* const, const double, const double, const int, const int normal,
                      const double* const, const double* const stateIn, const double* const,
                      double* const fluxOut, double* const stateOut) {
    std::copy_n(stateIn, 5, stateOut);
    double buf[3][5];
    double* F[3] = {buf[0], buf[1], buf[2]};
    flux(stateOut, F);
    std::copy_n(F[normal], 5, fluxOut);
  }
};
}  // namespace Euler
