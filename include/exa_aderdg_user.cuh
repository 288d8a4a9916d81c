/* exa_aderdg_user.cuh -- compile an application's PDE system into the B200 ADER-DG kernels.
 *
 * The reference binds an application's solver class into the generic kernels by static
 * polymorphism: the toolkit generates Abstract<App>Solver_ADERDG, whose kernel calls are templated
 * on the user's class with its hooks flux, eigenvalues, nonConservativeProduct, boundaryValues and
 * adjustPointSolution (Toolkit/exahype/toolkit/templates/solvers/AbstractGenericADERDGSolverHeader
 * .template:34-68, 220-338). Here the application writes the same hooks as a struct of static
 * __device__ functions, compiles it with this header into its own shared library, and registers
 * the (dimension, order, parameters) instantiations it needs:
 *
 *   #include "exa_aderdg_user.cuh"
 *   struct MyEuler {
 *     static constexpr int V = 5;              // NumberOfVariables
 *     static constexpr bool kNCP = false;      // the system has a non-conservative product
 *     static constexpr bool kSource = false;   // the patch's point source acts on it
 *     static constexpr bool kAdjoint = false;  // discrete adjoint hooks (flux_vjp, max_speed_grad)
 *     template <int DIM> static __device__ void flux(const double* Q, double* F);   // F[d * V + m]
 *     template <int DIM> static __device__ void eigenvalues(const double* Q, int d, double* lambda);
 *     template <int DIM> static __device__ void ncp(const double* Q, const double* gradQ, double* BgradQ);
 *     template <int DIM> static __device__ void wall(const double* Qin, int normal, double* Qout);
 *     // optional:
 *     template <int DIM> static __device__ void adjust_point_solution(const double* x, double t,
 *                                                                     double dt, double* Q);
 *     template <int DIM> static __device__ void boundary_values(const double* x, double t, double dt,
 *         int faceIndex, int normal, const double* Fin, const double* Qin, double* Fout, double* Qout);
 *     // the reference's algebraicSource (useSource): S[V] at the space-time node (x[3], t)
 *     template <int DIM> static __device__ void algebraic_source(const double* x, double t,
 *                                                                const double* Q, double* S);
 *     // a flux that depends on the gradient (the reference's useViscousFlux, viscousFlux and
 *     // viscousEigenvalues): gradQ[d * V + m]
 *     static constexpr bool kViscous = true;
 *     template <int DIM> static __device__ void viscous_flux(const double* Q, const double* gradQ, double* F);
 *     template <int DIM> static __device__ void viscous_eigenvalues(const double* Q, int d, double* lambda);
 *   };
 *   EXA_REGISTER_PDE(EXA_PDE_USER_BASE, MyEuler, 3, 5, 0)  // id, functor, DIM, Order, NumberOfParameters
 *
 * Q holds the D = V + NumberOfParameters values of a node; flux fills DIM * V values; wall is the
 * ghost state of a reflective wall (EXA_BC_WALL faces; the outflow type copies the inner state);
 * boundary_values is the user's boundaryValues for EXA_BC_USER faces: Qout arrives pre-filled with
 * Qin, Fout receives the normal flux of the outer state; adjust_point_solution sets or modifies a
 * node's values at position x (exa_patch_adjust_solution). Every kernel -- FP64 and mixed
 * predictors, Riemann, boundary, update and CFL -- is instantiated for the functor.
 *
 * ORDER runs over 1..9 in 2D and 3D, the orders of the reference's generated quadrature tables.
 * A cell whose space-time Picard state (n^(DIM+1) * D doubles, n = ORDER + 1) does not fit one
 * CTA's shared memory runs the streamed predictor, which keeps that state in an L2-resident
 * scratch. That predictor takes systems without an NCP, and one time node's fluxes
 * (DIM * V * n^DIM doubles) must still fit the CTA. A static_assert names an instantiation that
 * fits neither form.
 *
 * With algebraic_source the predictor adds S(x, t + node_i dt, Q) - NCP at every space-time node
 * and the volume integral its time average, as the reference does; x = cell centre + dx (node -
 * 0.5), with z = 0 in 2D. The cell positions come from the patch, from the per-cell shim's
 * cellCenter, or from exa_fused_predictor_volume_integral_x (the batched call without centres
 * refuses such a PDE). No mixed-precision form, streamed predictor or adjoint for it.
 *
 * With kViscous the predictor evaluates viscous_flux at every node and time node with the gradient
 * of the Picard iterate there; the Rusanov speed and the CFL step add the viscous eigenvalues' terms
 * of the reference. flux is still required: the built-in wall and outflow faces take the inviscid
 * flux of their ghost state. Systems with a viscous flux have no mixed-precision form, no
 * streamed predictor and no adjoint. The batched face entry points need the cell size for them
 * (exa_riemann_solver_nonlinear_dx). The time-averaged gradient's face values (lGradQhbnd, which the
 * reference passes to boundaryValues) are not produced.
 *
 * Build with the same flags as the library (exahype-engine_b200/build.py: build_user_pde does it),
 * linking libexa_aderdg.so. Loading the application's library registers its instantiations; from
 * then on exa_solver_create accepts cfg.pde = the registered id through the unchanged C ABI, and
 * exa_pde_available reports them.
 */
#ifndef EXA_ADERDG_USER_CUH
#define EXA_ADERDG_USER_CUH

#include <cstdio>

#include "exa_aderdg.h"
#include "../exahype-engine_b200/csrc/exa_ops.cuh"

#define EXA_USER_CAT2(a, b) a##b
#define EXA_USER_CAT(a, b) EXA_USER_CAT2(a, b)

/* Registers exa::OpsImpl<FUNCTOR, DIM, ORDER, NPAR> under pde id ID when the library is loaded.
 * The launcher object is a function-local static of the application's library. */
#define EXA_REGISTER_PDE(ID, FUNCTOR, DIM, ORDER, NPAR)                                              \
  namespace {                                                                                        \
  struct EXA_USER_CAT(exa_user_registrar_, __LINE__) {                                               \
    EXA_USER_CAT(exa_user_registrar_, __LINE__)() {                                                  \
      static exa::OpsImpl<FUNCTOR, DIM, ORDER, NPAR> ops;                                            \
      if (exa_register_pde((ID), (DIM), (ORDER), (NPAR), &ops) != EXA_OK)                            \
        std::fprintf(stderr, "exa_register_pde(%d, %d, %d, %d): %s\n", (ID), (DIM), (ORDER), (NPAR), \
                     exa_last_error());                                                              \
    }                                                                                                \
  } EXA_USER_CAT(exa_user_registrar_instance_, __LINE__);                                            \
  }

#endif /* EXA_ADERDG_USER_CUH */
