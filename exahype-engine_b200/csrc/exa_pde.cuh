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
//   static constexpr bool kSource;   the patch's point source (algebraicSource) may act on it
//   static constexpr bool kAdjoint;  the discrete adjoint is built for it (linear systems), with
//   flux_vjp<DIM>(Q, lF, lQ)         lQ[k] += sum_{d,m} lF[d*V + m] dF_d[m]/dQ[k], k < V + P
//   max_speed_grad<DIM>(Q, d, g)     returns max_m |lambda_m(Q)| and sets g[k] = its dQ[k] gradient
//
// Optional hooks (detected at compile time; functors without them keep the built-in behaviour):
//   adjust_point_solution<DIM>(x, t, dt, Q)      adjustPointSolution: sets / modifies the D values
//                                                of the node at position x (initial conditions)
//   boundary_values<DIM>(x, t, dt, faceIndex, normal, Fin, Qin, Fout, Qout)
//                                                boundaryValues for faces of type EXA_BC_USER:
//                                                Qout (D values, pre-filled with Qin) and Fout (V,
//                                                the normal flux of the outer state) at face node x
//   algebraic_source<DIM>(x, t, Q, S)            algebraicSource: S[V] at the space-time node (x, t)
//                                                (useSource), in the predictor's rhs and the volume
//                                                integral's time-averaged source, minus the NCP
//   static constexpr bool kViscous = true        the flux depends on the gradient (useViscousFlux):
//   viscous_flux<DIM>(Q, gradQ, F)               viscousFlux, gradQ[d*V + m], replacing flux in
//                                                the predictor
//   viscous_eigenvalues<DIM>(Q, d, lambda)       viscousEigenvalues: the Rusanov speed adds
//                                                2 (2N+1) / (dx_d sqrt(pi/2)) max|lambda| and the
//                                                CFL denominator max|lambda| 2 / (PNPM dx_d)
//
// The bodies restate the reference applications' formulas in the same operation order so that
// the FP64 path agrees with the reference to rounding.
#pragma once
#include <type_traits>

namespace exa {

template <class PDE, int DIM, class = void>
struct has_adjust_point_solution : std::false_type {};
template <class PDE, int DIM>
struct has_adjust_point_solution<PDE, DIM,
                                 std::void_t<decltype(PDE::template adjust_point_solution<DIM>(
                                     (const double*)nullptr, 0.0, 0.0, (double*)nullptr))>> : std::true_type {};

template <class PDE, int DIM, class = void>
struct has_boundary_values : std::false_type {};
template <class PDE, int DIM>
struct has_boundary_values<PDE, DIM,
                           std::void_t<decltype(PDE::template boundary_values<DIM>(
                               (const double*)nullptr, 0.0, 0.0, 0, 0, (const double*)nullptr, (const double*)nullptr,
                               (double*)nullptr, (double*)nullptr))>> : std::true_type {};

template <class PDE, int DIM, class = void>
struct has_algebraic_source : std::false_type {};
template <class PDE, int DIM>
struct has_algebraic_source<PDE, DIM,
                            std::void_t<decltype(PDE::template algebraic_source<DIM>(
                                (const double*)nullptr, 0.0, (const double*)nullptr, (double*)nullptr))>>
    : std::true_type {};

template <class PDE, class = void>
struct is_viscous : std::false_type {};
template <class PDE>
struct is_viscous<PDE, std::void_t<decltype(PDE::kViscous)>> : std::integral_constant<bool, PDE::kViscous> {};

// correctly rounded reciprocal: the same value as 1 / x (IEEE round to nearest), fewer instructions
__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float recip(float x) { return 1.0f / x; }

// Compressible Euler, gamma = 1.4 (ApplicationExamples/Euler/Euler_ADERDG/EulerSolver_ADERDG.cpp
// :61-146). nVar = 5 in 2D and 3D; the 2D system carries the unused z-momentum Q[3].
struct EulerPDE {
  static constexpr int V = 5;
  static constexpr bool kNCP = false;
  static constexpr bool kSource = false;  // no algebraicSource
  static constexpr bool kAdjoint = false;
  static constexpr int id = 0;

  template <int DIM, class T>
  static __device__ __forceinline__ void flux(const T* Q, T* F) {
    const T gamma = T(1.4);
    const T irho = recip(Q[0]);
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
    // Q[d + 1] written as a select so that register-resident Q is never indexed at run time
    const double u_n = (d == 0 ? Q[1] : (d == 1 ? Q[2] : Q[3])) * irho;
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
#pragma unroll
    for (int k = 0; k < 3; k++)
      if (k == normal) Qout[1 + k] = -Qout[1 + k];
  }
};

// Shallow water with bathymetry b as 4th variable (ApplicationExamples/SWE/SWE_ADERDG/
// MySWESolver.cpp:103-152): flux, eigenvalues, NCP g*h*grad(b); reflective wall (:43-62).
struct SWEPDE {
  static constexpr int V = 4;
  static constexpr bool kNCP = true;
  static constexpr bool kSource = false;
  static constexpr bool kAdjoint = false;
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
    const double u_n = (d == 0 ? Q[1] : Q[2]) * ih;
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
#pragma unroll
    for (int k = 0; k < 2; k++)
      if (k == normal) Qout[1 + k] = -Qout[1 + k];
  }
};

}  // namespace exa

namespace exa {

// Linear acoustics with material parameters carried per node (V = 4: p, u, v, w; P = 2: rho, c),
// written in flux form for the nonlinear ADER-DG path (the reference's acoustic and elastic apps
// use the linear kernels; these functors are new):
//   dp/dt + div(rho c^2 u) = 0,   du_d/dt + d(p / rho)/dx_d = 0.
// Inside a cell the parameters are constant, so the flux form equals the usual non-conservative
// form; across cells the Rusanov flux couples them. Eigenvalues -c, 0, 0, +c.
struct AcousticPDE {
  static constexpr int V = 4;
  static constexpr int P = 2;
  static constexpr bool kNCP = false;
  static constexpr bool kSource = true;  // regularised point source (Ricker)
  static constexpr bool kAdjoint = true;
  static constexpr int id = 2;

  template <int DIM, class T>
  static __device__ __forceinline__ void flux(const T* Q, T* F) {
    const T rho = Q[4], c = Q[5];
    const T K = rho * c * c;
    const T pr = Q[0] / rho;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      T* f = F + 4 * d;
      f[0] = K * Q[1 + d];
      f[1] = d == 0 ? pr : T(0);
      f[2] = d == 1 ? pr : T(0);
      f[3] = d == 2 ? pr : T(0);
    }
  }
  template <int DIM>
  static __device__ __forceinline__ void eigenvalues(const double* Q, int, double* lambda) {
    const double c = Q[5];
    lambda[0] = -c;
    lambda[1] = 0.0;
    lambda[2] = 0.0;
    lambda[3] = c;
  }
  template <int DIM, class T>
  static __device__ __forceinline__ void ncp(const T*, const T*, T* B) {
#pragma unroll
    for (int m = 0; m < 4; m++) B[m] = T(0);
  }
  template <int DIM>
  static __device__ __forceinline__ void wall(const double* Qin, int normal, double* Qout) {
#pragma unroll
    for (int m = 0; m < 6; m++) Qout[m] = Qin[m];
#pragma unroll
    for (int k = 0; k < 3; k++)
      if (k == normal) Qout[1 + k] = -Qout[1 + k];
  }
  // transposed flux Jacobian with respect to (p, u, v, w, rho, c)
  template <int DIM>
  static __device__ __forceinline__ void flux_vjp(const double* Q, const double* lF, double* lQ) {
    const double rho = Q[4], c = Q[5];
    const double K = rho * c * c;
    const double ir = 1.0 / rho;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const double a = lF[4 * d];          // against F_d[0] = K u_d
      const double b = lF[4 * d + 1 + d];  // against F_d[1 + d] = p / rho
      const double ud = d == 0 ? Q[1] : (d == 1 ? Q[2] : Q[3]);
      if (d == 0) lQ[1] += K * a;
      if (d == 1) lQ[2] += K * a;
      if (d == 2) lQ[3] += K * a;
      lQ[0] += b * ir;
      lQ[4] += a * c * c * ud - b * Q[0] * ir * ir;
      lQ[5] += a * 2.0 * rho * c * ud;
    }
  }
  template <int DIM>
  static __device__ __forceinline__ double max_speed_grad(const double* Q, int, double* g) {
#pragma unroll
    for (int k = 0; k < 6; k++) g[k] = 0.0;
    g[5] = Q[5] >= 0.0 ? 1.0 : -1.0;
    return fabs(Q[5]);
  }
};

// Linear elasticity, velocity-stress form with per-node parameters (V = 9: v1 v2 v3 s11 s22 s33
// s12 s13 s23; P = 3: rho, cp, cs; lambda = rho (cp^2 - 2 cs^2), mu = rho cs^2), in flux form:
//   dv_i/dt - d(s_ij / rho)/dx_j = 0,
//   ds_ij/dt - d(lambda delta_ij v_k + mu (delta_ik v_j + delta_jk v_i))/dx_k = 0.
// Eigenvalues -cp, -cs, -cs, 0, 0, 0, cs, cs, cp.
struct ElasticPDE {
  static constexpr int V = 9;
  static constexpr int P = 3;
  static constexpr bool kNCP = false;
  static constexpr bool kSource = true;  // regularised point source (Ricker)
  static constexpr bool kAdjoint = true;
  static constexpr int id = 3;

  template <int DIM, class T>
  static __device__ __forceinline__ void flux(const T* Q, T* F) {
    const T rho = Q[9], cp = Q[10], cs = Q[11];
    const T mu = rho * cs * cs;
    const T lam = rho * cp * cp - T(2) * mu;
    const T ir = T(1) / rho;
    // stress tensor entries by (i, j)
    const T s[3][3] = {{Q[3], Q[6], Q[7]}, {Q[6], Q[4], Q[8]}, {Q[7], Q[8], Q[5]}};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      T* f = F + 9 * d;
      f[0] = -s[0][d] * ir;
      f[1] = -s[1][d] * ir;
      f[2] = -s[2][d] * ir;
      const T vd = Q[d];
      // diagonal stresses: -(lambda v_d + 2 mu v_d delta_id)
      f[3] = -(lam * vd + (d == 0 ? T(2) * mu * vd : T(0)));
      f[4] = -(lam * vd + (d == 1 ? T(2) * mu * vd : T(0)));
      f[5] = -(lam * vd + (d == 2 ? T(2) * mu * vd : T(0)));
      // shear stresses s12, s13, s23: -mu (delta_1d v_2 + delta_2d v_1), ...
      f[6] = -mu * ((d == 0 ? Q[1] : T(0)) + (d == 1 ? Q[0] : T(0)));
      f[7] = -mu * ((d == 0 ? Q[2] : T(0)) + (d == 2 ? Q[0] : T(0)));
      f[8] = -mu * ((d == 1 ? Q[2] : T(0)) + (d == 2 ? Q[1] : T(0)));
    }
  }
  template <int DIM>
  static __device__ __forceinline__ void eigenvalues(const double* Q, int, double* lambda) {
    const double cp = Q[10], cs = Q[11];
    lambda[0] = -cp;
    lambda[1] = -cs;
    lambda[2] = -cs;
    lambda[3] = 0.0;
    lambda[4] = 0.0;
    lambda[5] = 0.0;
    lambda[6] = cs;
    lambda[7] = cs;
    lambda[8] = cp;
  }
  template <int DIM, class T>
  static __device__ __forceinline__ void ncp(const T*, const T*, T* B) {
#pragma unroll
    for (int m = 0; m < 9; m++) B[m] = T(0);
  }
  template <int DIM>
  static __device__ __forceinline__ void wall(const double* Qin, int normal, double* Qout) {
    // rigid wall: mirrored velocity
#pragma unroll
    for (int m = 0; m < 12; m++) Qout[m] = Qin[m];
#pragma unroll
    for (int k = 0; k < 3; k++) Qout[k] = -Qout[k];
    (void)normal;
  }
  // transposed flux Jacobian with respect to (v1 v2 v3 s11 s22 s33 s12 s13 s23, rho, cp, cs)
  template <int DIM>
  static __device__ __forceinline__ void flux_vjp(const double* Q, const double* lF, double* lQ) {
    const double rho = Q[9], cp = Q[10], cs = Q[11];
    const double mu = rho * cs * cs;
    const double lam = rho * cp * cp - 2.0 * mu;
    const double ir = 1.0 / rho;
    const double sg[3][3] = {{Q[3], Q[6], Q[7]}, {Q[6], Q[4], Q[8]}, {Q[7], Q[8], Q[5]}};
    // slot of stress s_ij in Q
    constexpr int sidx[3][3] = {{3, 6, 7}, {6, 4, 8}, {7, 8, 5}};
    double g_lam = 0.0, g_mu = 0.0, g_ir = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const double* f = lF + 9 * d;
      // f_i = -s_id / rho
#pragma unroll
      for (int i = 0; i < 3; i++) {
        lQ[sidx[i][d]] -= f[i] * ir;
        g_ir -= f[i] * sg[i][d];
      }
      const double vd = Q[d];
      // f_{3+k} = -(lambda v_d + 2 mu v_d delta_kd)
      const double fsum = f[3] + f[4] + f[5];
      lQ[d] -= lam * fsum + 2.0 * mu * f[3 + d];
      g_lam -= vd * fsum;
      g_mu -= 2.0 * vd * f[3 + d];
      // shear: f6 = -mu (d0 v1 + d1 v0), f7 = -mu (d0 v2 + d2 v0), f8 = -mu (d1 v2 + d2 v1)
      if (d == 0) {
        lQ[1] -= mu * f[6];
        lQ[2] -= mu * f[7];
        g_mu -= Q[1] * f[6] + Q[2] * f[7];
      } else if (d == 1) {
        lQ[0] -= mu * f[6];
        lQ[2] -= mu * f[8];
        g_mu -= Q[0] * f[6] + Q[2] * f[8];
      } else {
        lQ[0] -= mu * f[7];
        lQ[1] -= mu * f[8];
        g_mu -= Q[0] * f[7] + Q[1] * f[8];
      }
    }
    // lambda = rho cp^2 - 2 rho cs^2, mu = rho cs^2, 1/rho
    lQ[9] += g_lam * (cp * cp - 2.0 * cs * cs) + g_mu * cs * cs - g_ir * ir * ir;
    lQ[10] += g_lam * 2.0 * rho * cp;
    lQ[11] += -g_lam * 4.0 * rho * cs + g_mu * 2.0 * rho * cs;
  }
  template <int DIM>
  static __device__ __forceinline__ double max_speed_grad(const double* Q, int, double* g) {
#pragma unroll
    for (int k = 0; k < 12; k++) g[k] = 0.0;
    if (fabs(Q[10]) >= fabs(Q[11])) {
      g[10] = Q[10] >= 0.0 ? 1.0 : -1.0;
      return fabs(Q[10]);
    }
    g[11] = Q[11] >= 0.0 ? 1.0 : -1.0;
    return fabs(Q[11]);
  }
};

}  // namespace exa
