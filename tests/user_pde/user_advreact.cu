// An application's PDE with its own algebraic source, compiled against include/exa_aderdg_user.cuh:
// three advected scalars with a source that depends on the position, the time and the state
// (linear coupling and a quadratic reaction). It exercises the useSource branch of the reference's
// generic kernels (algebraicSource at x = centre + dx (node - 0.5) and t + node_i dt,
// 3d/spaceTimePredictorNonlinear.cpph:323-367, and the time-averaged source in the volume
// integral). The same system is the source test solver of the checker's reference instantiation.
// Registered as pde EXA_PDE_USER_BASE + 2 for 3D and 2D order 3 (no parameters); used only by the
// tests.
#include "exa_aderdg_user.cuh"

struct UserAdvReact {
  static constexpr int V = 3;
  static constexpr bool kNCP = false;
  static constexpr bool kSource = false;
  static constexpr bool kAdjoint = false;

  static __device__ double a(int m, int d) {
    constexpr double A[3][3] = {{0.3, -0.2, 0.1}, {-0.5, 0.25, 0.4}, {0.0, 0.6, -0.3}};
    return A[m][d];
  }
  template <int DIM>
  static __device__ void flux(const double* Q, double* F) {
    for (int d = 0; d < DIM; d++)
      for (int m = 0; m < 3; m++) F[d * 3 + m] = a(m, d) * Q[m];
  }
  template <int DIM>
  static __device__ void eigenvalues(const double*, int d, double* lambda) {
    for (int m = 0; m < 3; m++) lambda[m] = a(m, d);
  }
  // x: 3 coordinates (z = 0 in 2D)
  template <int DIM>
  static __device__ void algebraic_source(const double* x, double t, const double* Q, double* S) {
    const double pi = 3.14159265358979323846;
    S[0] = -0.5 * Q[0] + 0.2 * Q[1] + 0.1 * sin(2.0 * pi * (x[0] + 2.0 * x[1] + 3.0 * x[2]) - t);
    S[1] = -0.3 * Q[1] * Q[2];
    S[2] = 0.05 * cos(2.0 * pi * x[0]) - 0.4 * Q[2];
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

EXA_REGISTER_PDE(EXA_PDE_USER_BASE + 2, UserAdvReact, 3, 3, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE + 2, UserAdvReact, 2, 3, 0)
