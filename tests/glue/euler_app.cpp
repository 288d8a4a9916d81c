// An application on the generated glue: the user's solver class derives from the generated
// Euler::AbstractEulerSolver_ADERDG (exahype-engine_b200/glue/generate_glue.py with
// euler_glue_spec.json) and supplies its host-side boundaryValues, a reflective wall as in the
// reference's Euler and SWE applications (SWE_ADERDG/MySWESolver.cpp:43-62), and its
// adjustPointSolution, a density wave at t = 0. The extern "C" functions let the tests drive the
// glue methods the way the reference's engine calls them.
#include <algorithm>
#include <cmath>

#include "AbstractEulerSolver_ADERDG.h"

namespace Euler {
class EulerSolver_ADERDG : public AbstractEulerSolver_ADERDG {
 public:
  static void flux(const double* const Q, double* const F, int d) {  // normal flux, gamma 1.4
    const double irho = 1.0 / Q[0];
    const double p = 0.4 * (Q[4] - 0.5 * irho * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]));
    const double un = Q[1 + d];
    F[0] = un;
    F[1] = irho * Q[1] * un;
    F[2] = irho * Q[2] * un;
    F[3] = irho * Q[3] * un;
    F[1 + d] += p;
    F[4] = irho * (Q[4] + p) * un;
  }
  void boundaryValues(const double* const, const double, const double, const int, const int normalNonZero,
                      const double* const, const double* const stateIn, const double* const,
                      double* const fluxOut, double* const stateOut) override {
    std::copy_n(stateIn, NumberOfVariables, stateOut);
    stateOut[1 + normalNonZero] = -stateOut[1 + normalNonZero];
    flux(stateOut, fluxOut, normalNonZero);
  }
  // rho = 1 + 0.1 sin(2 pi (x + 2y + 3z)), u = (0.3, 0.2, 0.1), p = 1
  void adjustPointSolution(const double* const x, const double t, const double, double* const Q) override {
    if (t != 0.0) return;
    const double rho = 1.0 + 0.1 * std::sin(2.0 * 3.14159265358979323846 * (x[0] + 2.0 * x[1] + 3.0 * x[2]));
    const double u[3] = {0.3, 0.2, 0.1};
    Q[0] = rho;
    for (int d = 0; d < 3; d++) Q[1 + d] = rho * u[d];
    Q[4] = 1.0 / 0.4 + 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  }
};
}  // namespace Euler

extern "C" {
void* glue_create() { return new Euler::EulerSolver_ADERDG(); }
void glue_destroy(void* h) { delete static_cast<Euler::EulerSolver_ADERDG*>(h); }
int glue_predictor(void* h, double* lduh, double* lQhbnd, double* lFhbnd, double* luh, const double* centre,
                   const double* dx, double t, double dt, int add) {
  return static_cast<Euler::EulerSolver_ADERDG*>(h)->fusedSpaceTimePredictorVolumeIntegral(
      lduh, lQhbnd, nullptr, lFhbnd, luh, centre, dx, t, dt, add != 0);
}
void glue_riemann(void* h, double* FL, double* FR, const double* QL, const double* QR, double t, double dt,
                  const double* dx, int d) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->riemannSolver(FL, FR, QL, QR, t, dt, dx, d, false, 0);
}
void glue_boundary(void* h, double* fluxIn, const double* stateIn, const double* centre, const double* size, double t,
                   double dt, int d, int o) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->boundaryConditions(fluxIn, stateIn, nullptr, nullptr, centre, size, t,
                                                                 dt, d, o);
}
void glue_face(void* h, double* out, const double* lFhbnd, int d, int o, const int* subface, int levelDelta,
               const double* dx, double dt, int addToUpdate) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->faceIntegral(out, lFhbnd, d, o, subface, levelDelta, dx, dt,
                                                           addToUpdate != 0);
}
void glue_adjust(void* h, double* luh, const double* centre, const double* size, double t, double dt) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->adjustSolution(luh, centre, size, t, dt);
}
void glue_volume_prolong(void* h, double* fine, const double* coarse, int lc, int lf, const int* sub) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->volumeUnknownsProlongation(fine, coarse, lc, lf, sub);
}
void glue_volume_restrict(void* h, double* coarse, const double* fine, int lc, int lf, const int* sub) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->volumeUnknownsRestriction(coarse, fine, lc, lf, sub);
}
void glue_face_prolong(void* h, double* qf, double* ff, const double* qc, const double* fc, int lc, int lf,
                       const int* sub) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->faceUnknownsProlongation(qf, ff, qc, fc, lc, lf, sub);
}
void glue_update(void* h, double* luh, const double* luhOld, const double* lduh, double dt) {
  static_cast<Euler::EulerSolver_ADERDG*>(h)->addUpdateToSolution(luh, luhOld, lduh, dt);
}
double glue_dt(void* h, const double* luh, const double* dx) {
  return static_cast<Euler::EulerSolver_ADERDG*>(h)->stableTimeStepSize(luh, dx);
}
int glue_grid(void* h, double* luh_all, const int* ncell, const double* offset, const double* size, int nsteps,
              double* t) {
  return static_cast<Euler::EulerSolver_ADERDG*>(h)->updateUniformGrid(luh_all, ncell, offset, size, nsteps, t);
}
}
