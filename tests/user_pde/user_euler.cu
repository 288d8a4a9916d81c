// An application's PDE system compiled against include/exa_aderdg_user.cuh, the way a user of the
// library binds its own solver: compressible Euler (gamma 1.4) written from the hooks of the
// reference's Euler application (ApplicationExamples/Euler/Euler_ADERDG/EulerSolver_ADERDG.cpp:
// flux, eigenvalues, boundaryValues, adjustPointSolution), with
//   - adjust_point_solution: at t = 0 a smooth density wave advected by a uniform velocity,
//     rho = 1 + 0.1 sin(2 pi (x + 2y + 3z)), u = (0.3, 0.2, 0.1), p = 1 (2D: z = 0, w = 0);
//   - boundary_values: a reflective wall (mirrored normal momentum, the normal flux of that state).
// Registered as pde EXA_PDE_USER_BASE for order 3 in 2D and 3D, and for the extreme orders of the
// reference's tables: 1 and 9 in 2D, 1, 8 and 9 in 3D (no parameters). Used only by the tests, which
// check it against the oracle's Euler system.
#include "exa_aderdg_user.cuh"

struct UserEuler {
  static constexpr int V = 5;
  static constexpr bool kNCP = false;
  static constexpr bool kSource = false;
  static constexpr bool kAdjoint = false;

  template <int DIM>
  static __device__ void flux(const double* Q, double* F) {
    const double gamma = 1.4;
    const double irho = 1.0 / Q[0];
    const double j2 = DIM == 3 ? Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3] : Q[1] * Q[1] + Q[2] * Q[2];
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
    for (int d = 0; d < DIM; d++) {
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
  template <int DIM>
  static __device__ void eigenvalues(const double* Q, int d, double* lambda) {
    const double gamma = 1.4;
    const double irho = 1.0 / Q[0];
    const double j2 = DIM == 3 ? Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3] : Q[1] * Q[1] + Q[2] * Q[2];
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
    const double u_n = (d == 0 ? Q[1] : (d == 1 ? Q[2] : Q[3])) * irho;
    const double c = sqrt(gamma * p * irho);
    for (int m = 0; m < 5; m++) lambda[m] = u_n;
    lambda[0] -= c;
    lambda[4] += c;
  }
  template <int DIM>
  static __device__ void ncp(const double*, const double*, double* B) {
    for (int m = 0; m < 5; m++) B[m] = 0.0;
  }
  template <int DIM>
  static __device__ void wall(const double* Qin, int normal, double* Qout) {
    for (int m = 0; m < 5; m++) Qout[m] = Qin[m];
    Qout[1 + normal] = -Qout[1 + normal];
  }
  template <int DIM>
  static __device__ void adjust_point_solution(const double* x, double t, double, double* Q) {
    if (t != 0.0) return;
    const double pi = 3.14159265358979323846;
    const double z = DIM == 3 ? x[2] : 0.0;
    const double rho = 1.0 + 0.1 * sin(2.0 * pi * (x[0] + 2.0 * x[1] + 3.0 * z));
    const double u[3] = {0.3, 0.2, DIM == 3 ? 0.1 : 0.0};
    Q[0] = rho;
    Q[1] = rho * u[0];
    Q[2] = rho * u[1];
    Q[3] = rho * u[2];
    Q[4] = 1.0 / 0.4 + 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  }
  template <int DIM>
  static __device__ void boundary_values(const double*, double, double, int, int normal, const double*,
                                         const double* Qin, double* Fout, double* Qout) {
    wall<DIM>(Qin, normal, Qout);
    double F[DIM * 5];
    flux<DIM>(Qout, F);
    for (int m = 0; m < 5; m++) Fout[m] = F[normal * 5 + m];
  }
};

EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 3, 3, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 2, 3, 0)
// the smallest cells (2D order 1: 4 nodes, 32 cells per CTA) and the largest (3D order 8 and 9: 729
// and 1000 nodes, the streamed predictor with tail threads that own no node)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 2, 1, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 2, 9, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 3, 1, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 3, 8, 0)
EXA_REGISTER_PDE(EXA_PDE_USER_BASE, UserEuler, 3, 9, 0)
