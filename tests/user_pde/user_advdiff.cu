// An application's PDE with a viscous flux, compiled against include/exa_aderdg_user.cuh: three
// scalars advected with their own velocities a_m and diffused with their own diffusivities nu_m.
// It exercises the useViscousFlux branch of the reference's generic kernels
// (3d/spaceTimePredictorNonlinear.cpph:99-212 viscousFlux with the iterate's gradient,
// 3d/riemannSolverNonlinear.cpph:73-87 and 3d/stableTimeStepSize.cpph:44-51 viscousEigenvalues).
// The same system is the viscous test solver of the checker's reference instantiation. Registered
// as pde EXA_PDE_USER_BASE + 1 for 3D and 2D order 3 (no parameters); used only by the tests.
#include "exa_aderdg_user.cuh"

struct UserAdvDiff {
  static constexpr int V = 3;
  static constexpr bool kNCP = false;
  static constexpr bool kSource = false;
  static constexpr bool kAdjoint = false;
  static constexpr bool kViscous = true;

  static __device__ double a(int m, int d) {
    constexpr double A[3][3] = {{0.3, -0.2, 0.1}, {-0.5, 0.25, 0.4}, {0.0, 0.6, -0.3}};
    return A[m][d];
  }
  static __device__ double nu(int m) { return m == 0 ? 0.01 : (m == 1 ? 0.005 : 0.02); }

  template <int DIM>
  static __device__ void flux(const double* Q, double* F) {
    for (int d = 0; d < DIM; d++)
      for (int m = 0; m < 3; m++) F[d * 3 + m] = a(m, d) * Q[m];
  }
  template <int DIM>
  static __device__ void viscous_flux(const double* Q, const double* gradQ, double* F) {
    for (int d = 0; d < DIM; d++)
      for (int m = 0; m < 3; m++) F[d * 3 + m] = a(m, d) * Q[m] - nu(m) * gradQ[d * 3 + m];
  }
  template <int DIM>
  static __device__ void eigenvalues(const double*, int d, double* lambda) {
    for (int m = 0; m < 3; m++) lambda[m] = a(m, d);
  }
  template <int DIM>
  static __device__ void viscous_eigenvalues(const double*, int, double* lambda) {
    for (int m = 0; m < 3; m++) lambda[m] = nu(m);
  }
  template <int DIM>
  static __device__ void ncp(const double*, const double*, double* B) {
    for (int m = 0; m < 3; m++) B[m] = 0.0;
  }
  template <int DIM>
  static __device__ void wall(const double* Qin, int, double* Qout) {
    for (int m = 0; m < 3; m++) Qout[m] = Qin[m];
  }
};

EXA_REGISTER_PDE(EXA_PDE_USER_BASE + 1, UserAdvDiff, 3, 3, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE + 1, UserAdvDiff, 2, 3, 0)
