// Uniform-patch driver over the reference's generated optimised kernels (KernelGenerator plain-loop
// output in oracle/_ref/kg/<name>/kernels, namespace KG_NS). CHECKER / BASELINE ONLY.
//
// Same step as ref_glue.cpp's run_patch (global non-fused order): dt = min over cells of
// stableTimeStepSize -> fusedSpaceTimePredictorVolumeIntegral per cell -> riemannSolver on every
// face (outflow domain faces through boundaryConditions, as the generic glue wires it,
// AbstractGenericADERDGSolverImplementation.template:307-350) -> surfaceIntegral + solutionUpdate.
// The generated kernels assume cubic cells (one inverse dx), pad the variables to 8 doubles in
// lduh, lQhbnd and lFhbnd, and keep luh unpadded ([node][5]), the generic layout. OpenMP over cells
// and faces stands in for the absent TBB/Peano scheduler.
#include <omp.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

#include "EulerSolver_ADERDG.h"
#include "kernels/DGMatrices.h"
#include "kernels/Kernels.h"
#include "kernels/Quadrature.h"

namespace {
using namespace KG_NS;
constexpr int N1 = getBasisSize();            // nodes per axis
constexpr int V = getNumberOfVariable();
constexpr int ND = N1 * N1 * N1;

// aligned scratch (the generated code assumes ALIGNMENT-aligned arrays)
struct Buf {
  double* p = nullptr;
  explicit Buf(size_t n) { p = static_cast<double*>(::aligned_alloc(ALIGNMENT, ((n * 8 + ALIGNMENT - 1) / ALIGNMENT) * ALIGNMENT)); }
  ~Buf() { std::free(p); }
  Buf(const Buf&) = delete;
};
// the generated kernels read their operator and quadrature tables from globals that the
// application initialises once (kernels/DGMatrices.h, kernels/Quadrature.h)
struct Tables {
  Tables() {
    initDGMatrices();
    initQuadratureNodesAndWeights();
  }
};
Tables& tables() {
  static Tables t;
  return t;
}
}  // namespace

extern "C" int kgref_run(const int* ncell, const double* size, int walls, double* luh_all, int nsteps,
                         double fixed_dt, double* t_out, double* dts, int* picard, int nthreads) {
  (void)tables();
  const int nx = ncell[0], ny = ncell[1], nz = ncell[2];
  const long nc = (long)nx * ny * nz;
  const double dx = size[0] / nx;
  const double idx = 1.0 / dx;
  const double cs[3] = {dx, dx, dx};
  constexpr int QB = getBndFaceSize(), FB = getBndFluxSize();
  Buf lduh(nc * getUpdateSize()), lQhbnd(nc * getBndFaceTotalSize()), lFhbnd(nc * 6 * FB);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double t = 0.0;
  auto cellIndex = [&](int ix, int iy, int iz) -> long { return ((long)iz * ny + iy) * nx + ix; };
  for (int step = 0; step < nsteps; step++) {
    double dt = std::numeric_limits<double>::max();
    if (fixed_dt > 0) {
      dt = fixed_dt;
    } else {
#pragma omp parallel for reduction(min : dt) schedule(static)
      for (long c = 0; c < nc; c++) {
        Euler::EulerSolver_ADERDG s;
        dt = std::min(dt, stableTimeStepSize(s, luh_all + c * ND * V, idx));
      }
    }
#pragma omp parallel
    {
      Buf lQi(getlQiSize()), rhs(getlQiSize()), lFi(getlFiSize()), lQhi(getlQhiSize()), lFhi(getlFhiSize());
      Euler::EulerSolver_ADERDG s;
#pragma omp for schedule(static)
      for (long c = 0; c < nc; c++) {
        const int it = fusedSpaceTimePredictorVolumeIntegral(
            s, lduh.p + c * getUpdateSize(), lQhbnd.p + c * getBndFaceTotalSize(), nullptr, lFhbnd.p + c * 6 * FB,
            lQi.p, rhs.p, lFi.p, nullptr, lQhi.p, lFhi.p, nullptr, nullptr, nullptr, luh_all + c * ND * V, idx, dt);
        if (picard) picard[(long)step * nc + c] = it;
      }
    }
    for (int d = 0; d < 3; d++) {
#pragma omp parallel
      {
        Buf qo(QB), fo(FB);
        Euler::EulerSolver_ADERDG s;
#pragma omp for schedule(static)
        for (long c = 0; c < nc; c++) {
          const int ix = c % nx, iy = (c / nx) % ny, iz = (int)(c / ((long)nx * ny));
          int j[3] = {ix, iy, iz};
          const int lim = d == 0 ? nx : (d == 1 ? ny : nz);
          j[d] += 1;
          double* FL = lFhbnd.p + c * 6 * FB + (2 * d + 1) * FB;
          const double* QL = lQhbnd.p + c * getBndFaceTotalSize() + (2 * d + 1) * QB;
          const double centre[3] = {(ix + 0.5) * dx, (iy + 0.5) * dx, (iz + 0.5) * dx};
          if (j[d] == lim) {
            if (walls) {
              boundaryConditions(s, fo.p, qo.p, FL, QL, nullptr, centre, cs, t, dt, 2 * d + 1, d);
              riemannSolver(s, FL, fo.p, QL, qo.p, t, dt, dx, d);
            } else {
              j[d] = 0;
            }
          }
          if (j[d] < lim) {
            const long c2 = cellIndex(j[0], j[1], j[2]);
            double* FR = lFhbnd.p + c2 * 6 * FB + (2 * d) * FB;
            const double* QR = lQhbnd.p + c2 * getBndFaceTotalSize() + (2 * d) * QB;
            riemannSolver(s, FL, FR, QL, QR, t, dt, dx, d);
          }
          const int k = d == 0 ? ix : (d == 1 ? iy : iz);
          if (walls && k == 0) {
            double* FRb = lFhbnd.p + c * 6 * FB + (2 * d) * FB;
            const double* QRb = lQhbnd.p + c * getBndFaceTotalSize() + (2 * d) * QB;
            boundaryConditions(s, fo.p, qo.p, FRb, QRb, nullptr, centre, cs, t, dt, 2 * d, d);
            riemannSolver(s, fo.p, FRb, qo.p, QRb, t, dt, dx, d);
          }
        }
      }
    }
#pragma omp parallel for schedule(static)
    for (long c = 0; c < nc; c++) {
      surfaceIntegral(lduh.p + c * getUpdateSize(), lFhbnd.p + c * 6 * FB, idx);
      solutionUpdate(luh_all + c * ND * V, luh_all + c * ND * V, lduh.p + c * getUpdateSize(), dt);
    }
    if (dts) dts[step] = dt;
    t += dt;
  }
  if (t_out) *t_out = t;
  return 0;
}
