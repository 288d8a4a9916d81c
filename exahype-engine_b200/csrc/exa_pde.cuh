// User PDE terms as compile-time device functors (the L0 hooks of the reference's solver API:
// flux, eigenvalues, nonConservativeProduct, boundaryValues; AbstractGenericADERDGSolverHeader
// .template:220-338). A functor provides:
//
//   static constexpr int V;          number of evolved variables (NumberOfVariables)
//   static constexpr bool kNCP;      non-conservative product present (useNCP)
//   flux<DIM>(Q, F)                  F[d*V + m], d < DIM
//   eigenvalues<DIM>(Q, d, lambda)   lambda[V]
//   ncp<DIM>(Q, gradQ, BgradQ)       gradQ[d*V + m]  (only when kNCP)
//   wall<DIM>(QIn, normal, QOut)     ghost state of a reflective wall (boundaryValues)
//
// The bodies restate the reference applications' formulas in the same operation order so that
// the FP64 path agrees with the reference to rounding.
#pragma once

namespace exa {

// Compressible Euler, gamma = 1.4 (ApplicationExamples/Euler/Euler_ADERDG/EulerSolver_ADERDG.cpp
// :61-146). nVar = 5 in 2D and 3D; the 2D system carries the unused z-momentum Q[3].
struct EulerPDE {
  static constexpr int V = 5;
  static constexpr bool kNCP = false;
  static constexpr int id = 0;

  template <int DIM, class T>
  static __device__ __forceinline__ void flux(const T* Q, T* F) {
    const T gamma = T(1.4);
    const T irho = T(1) / Q[0];
    const T j2 = DIM == 3 ? Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3] : Q[1] * Q[1] + Q[2] * Q[2];
    const T p = (gamma - T(1)) * (Q[4] - T(0.5) * irho * j2);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      T* f = F + 5 * d;
      const T un = Q[1 + d];
      f[0] = un;
      f[1] = irho * Q[1] * un;
      f[2] = irho * Q[2] * un;
      f[3] = irho * Q[3] * un;
      f[1 + d] += p;
      f[4] = irho * (Q[4] + p) * un;
    }
  }
  template <int DIM>
  static __device__ __forceinline__ void eigenvalues(const double* Q, int d, double* lambda) {
    const double gamma = 1.4;
    const double irho = 1. / Q[0];
    const double j2 = DIM == 3 ? Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3] : Q[1] * Q[1] + Q[2] * Q[2];
    const double p = (gamma - 1) * (Q[4] - 0.5 * irho * j2);
    const double u_n = Q[d + 1] * irho;
    const double c = sqrt(gamma * p * irho);
#pragma unroll
    for (int m = 0; m < 5; m++) lambda[m] = u_n;
    lambda[0] -= c;
    lambda[4] += c;
  }
  template <int DIM, class T>
  static __device__ __forceinline__ void ncp(const T*, const T*, T* B) {
#pragma unroll
    for (int m = 0; m < 5; m++) B[m] = T(0);
  }
  template <int DIM>
  static __device__ __forceinline__ void wall(const double* Qin, int normal, double* Qout) {
#pragma unroll
    for (int m = 0; m < 5; m++) Qout[m] = Qin[m];
    Qout[1 + normal] = -Qout[1 + normal];
  }
};

// Shallow water with bathymetry b as 4th variable (ApplicationExamples/SWE/SWE_ADERDG/
// MySWESolver.cpp:103-152): flux, eigenvalues, NCP g*h*grad(b); reflective wall (:43-62).
struct SWEPDE {
  static constexpr int V = 4;
  static constexpr bool kNCP = true;
  static constexpr int id = 1;
  static constexpr double grav = 9.81;

  template <int DIM, class T>
  static __device__ __forceinline__ void flux(const T* Q, T* F) {
    const T g = T(grav);
    const T ih = T(1) / Q[0];
    F[0] = Q[1];
    F[1] = Q[1] * Q[1] * ih + T(0.5) * g * Q[0] * Q[0];
    F[2] = Q[1] * Q[2] * ih;
    F[3] = T(0);
    F[4] = Q[2];
    F[5] = Q[1] * Q[2] * ih;
    F[6] = Q[2] * Q[2] * ih + T(0.5) * g * Q[0] * Q[0];
    F[7] = T(0);
    if (DIM == 3) {
#pragma unroll
      for (int m = 8; m < 12; m++) F[m] = T(0);
    }
  }
  template <int DIM>
  static __device__ __forceinline__ void eigenvalues(const double* Q, int d, double* lambda) {
    const double c = sqrt(grav * Q[0]);
    const double ih = 1. / Q[0];
    const double u_n = Q[d + 1] * ih;
    lambda[0] = u_n + c;
    lambda[1] = u_n - c;
    lambda[2] = u_n;
    lambda[3] = 0.0;
  }
  template <int DIM, class T>
  static __device__ __forceinline__ void ncp(const T* Q, const T* gradQ, T* B) {
    B[0] = T(0);
    B[1] = T(grav) * Q[0] * gradQ[0 * 4 + 3];
    B[2] = T(grav) * Q[0] * gradQ[1 * 4 + 3];
    B[3] = T(0);
  }
  template <int DIM>
  static __device__ __forceinline__ void wall(const double* Qin, int normal, double* Qout) {
#pragma unroll
    for (int m = 0; m < 4; m++) Qout[m] = Qin[m];
    Qout[1 + normal] = -Qout[1 + normal];
  }
};

}  // namespace exa
