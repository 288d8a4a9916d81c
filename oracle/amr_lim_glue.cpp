// Checker glue around the reference's OWN mesh-level and limiter kernels (2D or 3D).
//
// Test infrastructure: compiled by oracle/Makefile, with the unmodified reference sources
// ExaHyPE/kernels/aderdg/generic/Kernels.h ({2d,3d}/amrRoutines.cpph), kernels/limiter/generic/Limiter.h
// (c/Limiter.cpph), kernels/LimiterProjectionMatrices.{h,cpp}, kernels/GaussLegendreBasis.cpp and
// kernels/GaussLobattoBasis.cpp read in place, into oracle/_ref/libexaref_amrlim{2,3}d.so. Only tests load
// it. The solver type plays the role of the generated glue: the static tables the kernels read
// (weights, fineGridProjector) and the default DMP hooks of
// AbstractGenericADERDGSolverHeader.template:176-198 (observables = the first NumberOfDMPObservables
// variables; the specified relaxation parameter), with the projectors set up as
// GenericLimiterSolverImplementation.template:36-38 does (PatchSize = 2N+1).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "kernels/GaussLegendreBasis.h"
#include "kernels/KernelUtils.h"
#include "kernels/aderdg/generic/Kernels.h"
#include "kernels/limiter/generic/Limiter.h"

namespace exaamr {

template <int ORDER, int NVAR, int NPAR, int NOBS>
struct Solver {
  static constexpr int Order = ORDER;
  static constexpr int NumberOfVariables = NVAR;
  static constexpr int NumberOfParameters = NPAR;
  static constexpr int NumberOfDMPObservables = NOBS;
  static double** weights;
  static double**** fineGridProjector;
  void mapDiscreteMaximumPrincipleObservables(double* const observables, const double* const Q) const {
    std::copy_n(Q, NOBS, observables);
  }
  double getDiscreteMaximumPrincipleRelaxationParameter(const double& specified, const int&, const double&,
                                                        const double&, const double&, const double&) const {
    return specified;
  }
};
template <int O, int V, int P, int B> double** Solver<O, V, P, B>::weights = kernels::legendre::weights;
template <int O, int V, int P, int B> double**** Solver<O, V, P, B>::fineGridProjector = kernels::legendre::fineGridProjector;

template <class S>
void volume(int mode, double* out, const double* in, int coarseLevel, int fineLevel, const int* idx) {
  tarch::la::Vector<DIMENSIONS, int> sub;
  for (int d = 0; d < DIMENSIONS; d++) sub[d] = idx[d];
  constexpr int n = S::Order + 1;
  if (mode == 0)
    kernels::aderdg::generic::c::volumeUnknownsProlongation<S, S::NumberOfVariables, S::NumberOfParameters, n>(
        out, in, coarseLevel, fineLevel, sub);
  else
    kernels::aderdg::generic::c::volumeUnknownsRestriction<S, S::NumberOfVariables, S::NumberOfParameters, n>(
        out, in, coarseLevel, fineLevel, sub);
}

template <class S>
void face(int mode, double* outQ, double* outF, const double* inQ, const double* inF, int coarseLevel,
          int fineLevel, const int* idx) {
  tarch::la::Vector<DIMENSIONS - 1, int> sub;
  for (int d = 0; d < DIMENSIONS - 1; d++) sub[d] = idx[d];
  constexpr int n = S::Order + 1;
  if (mode == 0)
    kernels::aderdg::generic::c::faceUnknownsProlongation<S, S::NumberOfVariables, S::NumberOfParameters, n>(
        outQ, outF, inQ, inF, coarseLevel, fineLevel, sub);
  else if (mode == 1)
    kernels::aderdg::generic::c::faceUnknownsRestriction<S, S::NumberOfVariables, S::NumberOfParameters, n>(
        outQ, outF, inQ, inF, coarseLevel, fineLevel, sub);
  else
    kernels::aderdg::generic::c::faceUnknownsRestriction<S, S::NumberOfVariables, n>(outF, inF, sub,
                                                                                    fineLevel - coarseLevel);
}

template <int ORDER>
struct Proj {
  static constexpr int n = ORDER + 1, P = 2 * ORDER + 1;
  double dg2fv[n * P] = {0.0};
  double fv2dg[n * P] = {0.0};
  double leg2lob[n * n] = {0.0};
  Proj() {
    kernels::computeDG2FVProjector<ORDER, P>(dg2fv);
    kernels::computeFV2DGProjector<ORDER, P>(fv2dg, dg2fv);
    kernels::computeLegendre2LobattoProjector<ORDER>(leg2lob);
  }
};

// op: 0 projectOnFVLimiterSpace (a -> b), 1 projectOnDGSpace (a -> b), 2 findCellLocalMinAndMax
// (a -> mn, mx), 3 findCellLocalLimiterMinAndMax (a -> mn, mx), 4 discreteMaximumPrincipleAndMinAndMaxSearch
// (a, relax, scale; mn, mx in/out [2*DIM][NOBS]) returning the verdict
template <class S, int G>
int limiter(int op, const double* a, double* b, double* mn, double* mx, double relax, double scale) {
  constexpr int n = S::Order + 1, P = 2 * S::Order + 1, D = S::NumberOfVariables + S::NumberOfParameters;
  constexpr int B = S::NumberOfDMPObservables;
  static const Proj<S::Order> pr;
  S s;
  namespace L = kernels::limiter::generic::c;
  switch (op) {
    case 0: L::projectOnFVLimiterSpace<D, n, P, G>(a, pr.dg2fv, b); return 1;
    case 1: L::projectOnDGSpace<D, n, P, G>(a, pr.fv2dg, b); return 1;
    case 2: L::findCellLocalMinAndMax<S, B, n, P>(a, s, pr.dg2fv, pr.fv2dg, pr.leg2lob, mn, mx); return 1;
    case 3: L::findCellLocalLimiterMinAndMax<S, B, n, P, G>(a, s, mn, mx); return 1;
    case 4:
      return L::discreteMaximumPrincipleAndMinAndMaxSearch<S, B, n, P, G>(a, s, pr.dg2fv, pr.fv2dg, pr.leg2lob,
                                                                             relax, scale, mn, mx) ? 1 : 0;
  }
  return -1;
}

}  // namespace exaamr

using exaamr::Solver;

// configurations (order, nVar, nPar) of the GPU library's instantiations: 3D (3, 5, 0), (3, 5, 1),
// (5, 5, 0) [Euler], (4, 4, 2) [acoustics], (4, 9, 3) [elasticity with material parameters]; 2D
// (3, 5, 0), (3, 5, 1) [Euler], (4, 4, 0) [shallow water]
#if DIMENSIONS == 3
#define EXAAMR_DISPATCH(FN, ...)                                                                   \
  if (order == 3 && nvar == 5 && npar == 0) return FN<Solver<3, 5, 0, 5>>(__VA_ARGS__), 0;           \
  if (order == 3 && nvar == 5 && npar == 1) return FN<Solver<3, 5, 1, 5>>(__VA_ARGS__), 0;           \
  if (order == 4 && nvar == 4 && npar == 2) return FN<Solver<4, 4, 2, 4>>(__VA_ARGS__), 0;           \
  if (order == 5 && nvar == 5 && npar == 0) return FN<Solver<5, 5, 0, 5>>(__VA_ARGS__), 0;           \
  if (order == 4 && nvar == 9 && npar == 3) return FN<Solver<4, 9, 3, 9>>(__VA_ARGS__), 0;           \
  return -1;
#else
#define EXAAMR_DISPATCH(FN, ...)                                                                   \
  if (order == 3 && nvar == 5 && npar == 0) return FN<Solver<3, 5, 0, 5>>(__VA_ARGS__), 0;           \
  if (order == 3 && nvar == 5 && npar == 1) return FN<Solver<3, 5, 1, 5>>(__VA_ARGS__), 0;           \
  if (order == 4 && nvar == 4 && npar == 0) return FN<Solver<4, 4, 0, 4>>(__VA_ARGS__), 0;           \
  return -1;
#endif

extern "C" int exaamr_volume(int order, int nvar, int npar, int mode, double* out, const double* in,
                             int coarseLevel, int fineLevel, const int* idx) {
  EXAAMR_DISPATCH(exaamr::volume, mode, out, in, coarseLevel, fineLevel, idx)
}

extern "C" int exaamr_face(int order, int nvar, int npar, int mode, double* outQ, double* outF, const double* inQ,
                           const double* inF, int coarseLevel, int fineLevel, const int* idx) {
  EXAAMR_DISPATCH(exaamr::face, mode, outQ, outF, inQ, inF, coarseLevel, fineLevel, idx)
}

// fine[j][k][m] of order `order` (3 n n doubles)
extern "C" void exaamr_fine_grid_projector(int order, double* out) {
  const int n = order + 1;
  for (int j = 0; j < 3; j++)
    for (int k = 0; k < n; k++)
      for (int m = 0; m < n; m++) out[(j * n + k) * n + m] = kernels::legendre::fineGridProjector[order][j][k][m];
}

template <int O>
static void proj_copy(double* dg2fv, double* fv2dg, double* leg2lob) {
  exaamr::Proj<O> p;
  std::copy_n(p.dg2fv, sizeof(p.dg2fv) / sizeof(double), dg2fv);
  std::copy_n(p.fv2dg, sizeof(p.fv2dg) / sizeof(double), fv2dg);
  std::copy_n(p.leg2lob, sizeof(p.leg2lob) / sizeof(double), leg2lob);
}
// dg2fv [n][P], fv2dg [P][n], leg2lob [n][n] as the limiter solver computes them
extern "C" int exaamr_limiter_projectors(int order, double* dg2fv, double* fv2dg, double* leg2lob) {
  switch (order) {
    case 1: proj_copy<1>(dg2fv, fv2dg, leg2lob); return 0;
    case 2: proj_copy<2>(dg2fv, fv2dg, leg2lob); return 0;
    case 3: proj_copy<3>(dg2fv, fv2dg, leg2lob); return 0;
    case 4: proj_copy<4>(dg2fv, fv2dg, leg2lob); return 0;
    case 5: proj_copy<5>(dg2fv, fv2dg, leg2lob); return 0;
    case 6: proj_copy<6>(dg2fv, fv2dg, leg2lob); return 0;
    case 7: proj_copy<7>(dg2fv, fv2dg, leg2lob); return 0;
    case 8: proj_copy<8>(dg2fv, fv2dg, leg2lob); return 0;
    case 9: proj_copy<9>(dg2fv, fv2dg, leg2lob); return 0;
  }
  return -1;
}

// the limiter kernels, ghost layer width 0, 1 or 2; returns the op's result or -1
extern "C" int exaamr_limiter(int order, int nvar, int npar, int ghost, int op, const double* a, double* b,
                              double* mn, double* mx, double relax, double scale) {
#define EXAAMR_LIM(O, V, P)                                                                            \
  if (order == O && nvar == V && npar == P) {                                                       \
    if (ghost == 0) return exaamr::limiter<Solver<O, V, P, V>, 0>(op, a, b, mn, mx, relax, scale);    \
    if (ghost == 1) return exaamr::limiter<Solver<O, V, P, V>, 1>(op, a, b, mn, mx, relax, scale);    \
    if (ghost == 2) return exaamr::limiter<Solver<O, V, P, V>, 2>(op, a, b, mn, mx, relax, scale);    \
  }
  EXAAMR_LIM(3, 5, 0)
  EXAAMR_LIM(3, 5, 1)
#if DIMENSIONS == 3
  EXAAMR_LIM(5, 5, 0)
  EXAAMR_LIM(4, 9, 3)
#else
  EXAAMR_LIM(4, 4, 0)
#endif
#undef EXAAMR_LIM
  return -1;
}
