// Discrete adjoint of one ADER-DG time step for the linear systems (acoustic, elastic) with a
// fixed Picard sweep count and a fixed time step.
//
// The forward step u_{k+1} = u_k + dt/w_p * (volume(lFhi) - surface(Rusanov(lQhbnd, lFhbnd)))
// is differentiated exactly as it is computed (predictor, time averaging, extrapolation, volume
// integral, Rusanov with its face-averaged max wave speed, surface integral, update). The
// material parameters sit in the luh entries V..D-1 of every node; they are constant in time,
// so their adjoints accumulate in the same entries of lambda from step to step. After the last
// (first in time) adjoint step, lambda[.., V + j] holds dJ/d(parameter j at that node) and
// lambda[.., m < V] holds dJ/du_0.
//
// Forward references: the Picard loop 3d/spaceTimePredictorNonlinear.cpph:39-433 with
// UseMaxPicardIterations (a fixed sweep count, no residual test), time averaging :441-515,
// extrapolation :517-687, 3d/volumeIntegralNonlinear.cpph:133-223, 3d/riemannSolverNonlinear.cpph
// :37-128, 3d/surfaceIntegralNonlinear.cpph:21-90, 3d/solutionUpdate.cpph:28-67.
//
// Kernels, in launch order (the forward predictor at u_k runs first and leaves lQhbnd):
//   adjoint_face_kernel       one warp per interior face: transposed surface integral of both
//                             cells' lambda, transposed Rusanov -> adjoints of the predictor's
//                             face traces (adjQ, adjF), both sides;
//   adjoint_boundary_kernel   one warp per domain face (reflective wall or outflow): the same for
//                             the cell's side of a boundary Rusanov flux whose outer state is a
//                             diagonal sign map B of the inner trace (boundary_kernel's ghost);
//   adjoint_predictor_kernel  one CTA per cell, one thread per node: takes the Picard iterates
//                             from a global scratch (written there by the forward predictor
//                             launch when have_iter is set, else recomputed first), then runs
//                             the transposed extrapolation, volume integral, time averaging and
//                             Picard sweeps in reverse, and adds the result to lambda in place.
#pragma once

namespace exa {

struct AdjArgs {
  CellArgs c;      // the patch's cell arguments at u_k (luh, geometry, grid dt, source)
  FaceArgs f;      // interior faces
  FaceArgs fb;     // domain faces (walls, outflow): bcell / bface / btype, fb.nfaces of them
  double* lam;     // in: dJ/du_{k+1}; out: dJ/du_k (luh layout, D entries per node)
  double* adjQ;    // [cell][2 DIM][nf][D]: adjoint of the predictor's lQhbnd
  double* adjF;    // [cell][2 DIM][nf][V]: adjoint of the predictor's lFhbnd (before Riemann)
  double* iter;    // [cell][S][n][V][nd]: Picard iterates 1..S-1 (node-fastest: coalesced)
  int sweeps;      // fixed Picard sweep count S >= 1
  int have_iter;   // iter already holds q^1 .. q^{S-1} (written by the forward predictor)
};

template <class PDE, int DIM, int N, int P>
struct AdjShape {
  using S = Shape<PDE, DIM, N, P>;
  static constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, NL = S::NL;
  static constexpr int TPB = (nd + 31) / 32 * 32;
  static constexpr int items = DIM * V * NL;  // line contractions per pass
  static constexpr int rounds = (items + TPB - 1) / TPB;
  // shared memory: iterate / lambda_q slices, rhs / lambda_rhs slices, line buffers
  static constexpr int smemQ = n * nd * V;
  static constexpr int smemR = n * nd * V;
  static constexpr int smemF = DIM * V * nd;
  static constexpr size_t smem = sizeof(double) * (smemQ + smemR + smemF);
  // four resident CTAs where the per-thread state (n*V adjoint accumulators) fits 128 registers
  // without spilling (acoustic N=4: 166 -> 128 registers, 3 -> 4 CTAs per SM)
  static constexpr int MinBlocks = (V <= 4 && TPB <= 128 && 4 * (smem + 2048) <= 228 * 1024) ? 4 : 1;
};

// ------------------------------------------------------------------------------------------
// faces
// ------------------------------------------------------------------------------------------
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) adjoint_face_kernel(AdjArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf;
  const int face = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (face >= a.f.nfaces) return;  // uniform per warp
  const int L = a.f.left[face], R = a.f.right[face], d = a.f.dir[face];
  const int g = a.c.cell_grid ? a.c.cell_grid[L] : 0;
  const double dx = a.c.grid_dx ? a.c.grid_dx[g * 3 + d] : a.c.u_dx[d];
  const double dt = a.c.grid_dt ? a.c.grid_dt[g] : a.c.u_dt;
  const double cdt = dt / dx;
  const double* QL = a.c.lQhbnd + (size_t)L * S::sizeQhb + (size_t)(2 * d + 1) * nf * D;
  const double* QR = a.c.lQhbnd + (size_t)R * S::sizeQhb + (size_t)(2 * d) * nf * D;
  const double* lamL = a.lam + (size_t)L * nd * D;
  const double* lamR = a.lam + (size_t)R * nd * D;
  const int st = line_stride<n>(d);

  // forward: face averages and the Rusanov max wave speed (RiemannSolverUtils.h:152-177)
  double aL[D], aR[D];
#pragma unroll
  for (int m = 0; m < D; m++) aL[m] = aR[m] = 0.0;
  for (int fn = lane; fn < nf; fn += 32) {
    const double w = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
#pragma unroll
    for (int m = 0; m < D; m++) {
      aL[m] += w * QL[fn * D + m];
      aR[m] += w * QR[fn * D + m];
    }
  }
#pragma unroll
  for (int m = 0; m < D; m++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      aL[m] += __shfl_xor_sync(0xffffffffu, aL[m], off);
      aR[m] += __shfl_xor_sync(0xffffffffu, aR[m], off);
    }
  }
  double gL[D], gR[D];
  const double sL = PDE::template max_speed_grad<DIM>(aL, d, gL);
  const double sR = PDE::template max_speed_grad<DIM>(aR, d, gR);
  const bool leftMax = sL >= sR;  // fmax(sL, sR) in the forward kernel
  const double smax = leftMax ? sL : sR;

  // adjoint of the Rusanov flux F* from both cells' surface integrals, then of F*
  double* aFL = a.adjF + (size_t)L * S::sizeFhb + (size_t)(2 * d + 1) * nf * V;
  double* aFR = a.adjF + (size_t)R * S::sizeFhb + (size_t)(2 * d) * nf * V;
  double* aQL = a.adjQ + (size_t)L * S::sizeQhb + (size_t)(2 * d + 1) * nf * D;
  double* aQR = a.adjQ + (size_t)R * S::sizeQhb + (size_t)(2 * d) * nf * D;
  double lsm = 0.0;  // adjoint of smax
  for (int fn = lane; fn < nf; fn += 32) {
    const int base = line_base<DIM, n>(d, fn);
    double lf[V];
#pragma unroll
    for (int m = 0; m < V; m++) lf[m] = 0.0;
    // surface integral: lduh[(fn,k)] -= F+ F1[k] w_ab/dx (left cell), += F- F0[k] w_ab/dx
    // (right cell); the update scales lduh by dt / (w_ab w_k)
#pragma unroll
    for (int k = 0; k < n; k++) {
      const double cl = -cdt * G::F1(k) / G::weights(k);
      const double cr = cdt * G::F0(k) / G::weights(k);
      const double* ll = lamL + (size_t)(base + k * st) * D;
      const double* lr = lamR + (size_t)(base + k * st) * D;
#pragma unroll
      for (int m = 0; m < V; m++) lf[m] += cl * ll[m] + cr * lr[m];
    }
    // F* = (FL + FR)/2 - smax (QR - QL)/2
#pragma unroll
    for (int m = 0; m < V; m++) {
      lsm -= 0.5 * lf[m] * (QR[fn * D + m] - QL[fn * D + m]);
      aFL[fn * V + m] = 0.5 * lf[m];
      aFR[fn * V + m] = 0.5 * lf[m];
    }
    // evolved entries; the max-wave-speed term is added below
#pragma unroll
    for (int m = 0; m < D; m++) {
      aQL[fn * D + m] = m < V ? 0.5 * smax * lf[m] : 0.0;
      aQR[fn * D + m] = m < V ? -0.5 * smax * lf[m] : 0.0;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) lsm += __shfl_xor_sync(0xffffffffu, lsm, off);
  __syncwarp();
  // smax = max|lambda(Qav)| of the larger side; Qav = sum_fn w_fn Q[fn]
  for (int fn = lane; fn < nf; fn += 32) {
    const double w = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
    double* aq = leftMax ? aQL : aQR;
#pragma unroll
    for (int m = 0; m < D; m++) aq[fn * D + m] += lsm * w * (leftMax ? gL[m] : gR[m]);
  }
}

// Domain faces (3d/boundaryConditions.cpph:29-122 with the built-in ghosts of boundary_kernel).
// The cell's trace q meets the ghost qg = B q (B: +-1 per entry; outflow the identity, a wall the
// functor's mirrored velocity; parameters copied) whose normal flux is F_d(qg). With the cell on
// side o of the face (o = 1: the cell is left, o = 0: right),
//   F* = (F_c + F_d(B q)) / 2 - smax (q_R - q_L) / 2,  q_L, q_R = (q, B q) or (B q, q),
// so lambda_F* reaches F_c with 1/2, q through B^T J_d(B q)^T / 2 and the dissipation term, and the
// parameters through smax = max|lambda| of the larger side's face average.
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) adjoint_boundary_kernel(AdjArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf;
  const int bf = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (bf >= a.fb.nfaces) return;  // uniform per warp
  const long c = a.fb.bcell[bf];
  const int face = a.fb.bface[bf];
  const int d = face >> 1, o = face & 1;
  const int type = a.fb.btype ? a.fb.btype[bf] : 1;
  const int normal = type == 3 ? -1 : d;  // boundary_kernel: outflow (3) or the functor's wall
  const int g = a.c.cell_grid ? a.c.cell_grid[c] : 0;
  const double dx = a.c.grid_dx ? a.c.grid_dx[g * 3 + d] : a.c.u_dx[d];
  const double dt = a.c.grid_dt ? a.c.grid_dt[g] : a.c.u_dt;
  const double cdt = dt / dx;
  const double* Q = a.c.lQhbnd + (size_t)c * S::sizeQhb + (size_t)face * nf * D;
  const double* lam = a.lam + (size_t)c * nd * D;
  const int st = line_stride<n>(d);
  // diag(B): the ghost map of a vector of ones
  double b[D];
  {
    double one[D];
#pragma unroll
    for (int m = 0; m < D; m++) one[m] = 1.0;
    ghost_state<PDE, DIM, D>(one, normal, b);
#pragma unroll
    for (int m = V; m < D; m++) b[m] = 1.0;
  }
  // forward: face averages of both sides and the Rusanov max wave speed
  double aI[D], aG[D];
#pragma unroll
  for (int m = 0; m < D; m++) aI[m] = aG[m] = 0.0;
  for (int fn = lane; fn < nf; fn += 32) {
    const double w = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
#pragma unroll
    for (int m = 0; m < D; m++) {
      aI[m] += w * Q[fn * D + m];
      aG[m] += w * b[m] * Q[fn * D + m];
    }
  }
#pragma unroll
  for (int m = 0; m < D; m++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      aI[m] += __shfl_xor_sync(0xffffffffu, aI[m], off);
      aG[m] += __shfl_xor_sync(0xffffffffu, aG[m], off);
    }
  }
  double gI[D], gG[D];
  const double sI = PDE::template max_speed_grad<DIM>(aI, d, gI);
  const double sG = PDE::template max_speed_grad<DIM>(aG, d, gG);
  const double sL = o == 0 ? sG : sI, sR = o == 0 ? sI : sG;
  const bool leftMax = sL >= sR;  // fmax(sL, sR) in the forward kernel
  const double smax = leftMax ? sL : sR;
  const bool ghostMax = (o == 0) == leftMax;
  double* aF = a.adjF + (size_t)c * S::sizeFhb + (size_t)face * nf * V;
  double* aQ = a.adjQ + (size_t)c * S::sizeQhb + (size_t)face * nf * D;
  double lsm = 0.0;  // adjoint of smax
  const double sgn = o == 1 ? 1.0 : -1.0;  // F* = ... - smax sgn (B q - q) / 2
  for (int fn = lane; fn < nf; fn += 32) {
    const int base = line_base<DIM, n>(d, fn);
    double lf[V];
#pragma unroll
    for (int m = 0; m < V; m++) lf[m] = 0.0;
    // the cell's surface integral (o = 1: its right face, F1; o = 0: its left face, F0)
#pragma unroll
    for (int k = 0; k < n; k++) {
      const double ck = o == 1 ? -cdt * G::F1(k) / G::weights(k) : cdt * G::F0(k) / G::weights(k);
      const double* ll = lam + (size_t)(base + k * st) * D;
#pragma unroll
      for (int m = 0; m < V; m++) lf[m] += ck * ll[m];
    }
    double q[D], qg[D];
#pragma unroll
    for (int m = 0; m < D; m++) {
      q[m] = Q[fn * D + m];
      qg[m] = b[m] * q[m];
    }
    // the ghost's normal flux F_d(B q)
    double lF[DIM * V], lqg[D];
#pragma unroll
    for (int k = 0; k < DIM * V; k++) lF[k] = 0.0;
#pragma unroll
    for (int m = 0; m < V; m++) lF[d * V + m] = 0.5 * lf[m];
#pragma unroll
    for (int m = 0; m < D; m++) lqg[m] = 0.0;
    PDE::template flux_vjp<DIM>(qg, lF, lqg);
#pragma unroll
    for (int m = 0; m < V; m++) {
      lsm -= 0.5 * sgn * lf[m] * (qg[m] - q[m]);
      aF[fn * V + m] = 0.5 * lf[m];
    }
#pragma unroll
    for (int m = 0; m < D; m++) {
      // dissipation: d/dq of -smax sgn (b q - q) / 2
      const double diss = m < V ? -0.5 * smax * sgn * (b[m] - 1.0) * lf[m] : 0.0;
      aQ[fn * D + m] = b[m] * lqg[m] + diss;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) lsm += __shfl_xor_sync(0xffffffffu, lsm, off);
  __syncwarp();
  // smax = max|lambda| of the larger side's face average (of q, or of B q)
  for (int fn = lane; fn < nf; fn += 32) {
    const double w = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
#pragma unroll
    for (int m = 0; m < D; m++) aQ[fn * D + m] += lsm * w * (ghostMax ? b[m] * gG[m] : gI[m]);
  }
}

// ------------------------------------------------------------------------------------------
// cells
// ------------------------------------------------------------------------------------------
// In-place line contractions over the shared line buffers [dir][var][line][node along line]:
// TRANS = false: out[l] = coef * sum_k x[k] Kxi[k][l]   (forward flux / volume form)
// TRANS = true:  out[k] = coef * sum_l Kxi[k][l] x[l]   (its transpose)
template <int DIM, int N, int V, int TPB, bool TRANS>
__device__ __forceinline__ void adj_contract(double* sF, const double* coef_line) {
  using G = GL<N>;
  constexpr int n = N + 1, nd = DIM == 3 ? n * n * n : n * n, NL = nd / n;
  constexpr int items = DIM * V * NL;
  for (int it = threadIdx.x; it < items; it += TPB) {
    double* f = sF + (size_t)it * n;
    const int d = it / (V * NL), L = it % NL;
    const double coef = coef_line[d * NL + L];
    double x[n];
#pragma unroll
    for (int k = 0; k < n; k++) x[k] = f[k];
#pragma unroll
    for (int l = 0; l < n; l++) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < n; k++) acc = TRANS ? fma(G::Kxi(l, k), x[k], acc) : fma(x[k], G::Kxi(k, l), acc);
      f[l] = coef * acc;
    }
  }
}

template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__((AdjShape<PDE, DIM, N, P>::TPB), (AdjShape<PDE, DIM, N, P>::MinBlocks))
adjoint_predictor_kernel(AdjArgs a) {
  using A = AdjShape<PDE, DIM, N, P>;
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = A::n, V = A::V, D = A::D, nd = A::nd, NL = A::NL, TPB = A::TPB;
  static_assert(PDE::kAdjoint && !PDE::kNCP, "the adjoint is built for the linear flux-form systems");
  extern __shared__ double smem[];
  double* sQ = smem;                // [t][node][V]: iterate (recomputation), then lambda_q
  double* sR = smem + A::smemQ;     // [t][node][V]: rhs slices, then lambda_rhs slices
  double* sF = sR + A::smemR;       // [dir][var][line][k]
  __shared__ double s_coef[DIM * NL];
  __shared__ double s_cvol[DIM * NL];

  const int p = threadIdx.x;
  const bool live = p < nd;
  const long cell = blockIdx.x;
  const int g = a.c.cell_grid ? a.c.cell_grid[cell] : 0;
  const double dt = a.c.grid_dt ? a.c.grid_dt[g] : a.c.u_dt;
  double invdx[3];
#pragma unroll
  for (int d = 0; d < 3; d++) invdx[d] = d < DIM ? 1.0 / (a.c.grid_dx ? a.c.grid_dx[g * 3 + d] : a.c.u_dx[d]) : 0.0;
  for (int j = p; j < DIM * NL; j += TPB) {
    const int d = j / NL, L = j % NL;
    const double wt = DIM == 3 ? G::weights(L / n) * G::weights(L % n) : G::weights(L);
    s_coef[j] = wt * dt * invdx[d];   // times w_i per time node
    s_cvol[j] = dt * invdx[d];
  }

  int co[3] = {0, 0, 0};
  node_coords<DIM, n>(live ? p : 0, co);
  const double w_sp = DIM == 3 ? G::weights(co[2]) * G::weights(co[1]) * G::weights(co[0])
                               : G::weights(co[1]) * G::weights(co[0]);
  const double iweight = 1.0 / w_sp;
  int slot[DIM];  // this node's slot in every direction's line buffer (without the var offset)
#pragma unroll
  for (int d = 0; d < DIM; d++) slot[d] = node_line<DIM, n>(live ? p : 0, d) * n + co[d];

  double u[D];
  {
    const double* luh = a.c.luh + (size_t)cell * nd * D + (size_t)(live ? p : 0) * D;
#pragma unroll
    for (int m = 0; m < D; m++) u[m] = live ? luh[m] : 1.0;
  }
  // point source of the forward step (only its iterates depend on it)
  bool srcOn = false;
  double tcell = 0.0;
  if (PDE::kSource && a.c.src) {
    const double dxv[3] = {1.0 / invdx[0], DIM > 1 ? 1.0 / invdx[1] : 1.0, DIM > 2 ? 1.0 / invdx[2] : 1.0};
    double cc[3];
    cell_centre(a.c, cell, g, dxv, cc);
    srcOn = source_near<DIM>(a.c.src, cc, dxv);
    tcell = a.c.grid_t ? a.c.grid_t[g] : a.c.u_t;
  }
  const int srcVar = (PDE::kSource && a.c.src) ? (int)a.c.src[7] : -1;
  auto src_at = [&](int i) -> double {
    const double dxv[3] = {1.0 / invdx[0], DIM > 1 ? 1.0 / invdx[1] : 1.0, DIM > 2 ? 1.0 / invdx[2] : 1.0};
    double cc[3], x[3];
    cell_centre(a.c, cell, g, dxv, cc);
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = cc[d] + dxv[d] * (G::nodes(co[d]) - 0.5);
    return point_source<DIM>(a.c.src, x, tcell + G::nodes(i) * dt);
  };
  const int S_ = a.sweeps;
  double* iter = a.iter + (size_t)cell * S_ * n * nd * V;
  __syncthreads();

  // ---------------- recomputation of the Picard iterates q^1 .. q^{S-1} ----------------
  // (skipped when the forward predictor at u_k has exported them)
  for (int s = 0; s + 1 < (a.have_iter ? 1 : S_); s++) {
#pragma unroll
    for (int i = 0; i < n; i++) {
      if (live) {
        double q[D], F[DIM * V];
#pragma unroll
        for (int m = 0; m < D; m++) q[m] = (s == 0 || m >= V) ? u[m] : sQ[(i * nd + p) * V + m];
        PDE::template flux<DIM>(q, F);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) sF[(d * V + m) * nd + slot[d]] = F[d * V + m];
      }
      __syncthreads();
      // coefficients w_i * w_a w_b dt/dx_d: scale the per-line table by w_i on the fly
      {
        const double wi = G::weights(i);
        for (int it = threadIdx.x; it < A::items; it += TPB) {
          double* f = sF + (size_t)it * n;
          const int d = it / (V * NL), L = it % NL;
          const double coef = wi * s_coef[d * NL + L];
          double x[n];
#pragma unroll
          for (int k = 0; k < n; k++) x[k] = f[k];
#pragma unroll
          for (int l = 0; l < n; l++) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < n; k++) acc = fma(x[k], G::Kxi(k, l), acc);
            f[l] = coef * acc;
          }
        }
      }
      __syncthreads();
      if (live) {
        const double wi = G::weights(i);
        const double si = (PDE::kSource && srcOn) ? src_at(i) : 0.0;
#pragma unroll
        for (int m = 0; m < V; m++) {
          double rhs = w_sp * G::F0(i) * u[m];
#pragma unroll
          for (int d = 0; d < DIM; d++) rhs -= sF[(d * V + m) * nd + slot[d]];
          if (PDE::kSource && srcOn && m == srcVar) rhs += wi * w_sp * dt * si;
          sR[(i * nd + p) * V + m] = iweight * rhs;
        }
      }
      __syncthreads();
    }
    if (live) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        double r[n];
#pragma unroll
        for (int i = 0; i < n; i++) r[i] = sR[(i * nd + p) * V + m];
#pragma unroll
        for (int t = 0; t < n; t++) {
          double qn = 0.0;
#pragma unroll
          for (int i = 0; i < n; i++) qn = fma(r[i], G::iK1(t, i), qn);
          sQ[(t * nd + p) * V + m] = qn;
          iter[(((size_t)(s + 1) * n + t) * V + m) * nd + p] = qn;
        }
      }
    }
    __syncthreads();
  }

  // the iterate q^s at time node i and this node (s = 0: luh)
  auto iterate = [&](int s, int i, double* q) {
#pragma unroll
    for (int m = 0; m < D; m++)
      q[m] = (s == 0 || m >= V) ? u[m] : iter[(((size_t)s * n + i) * V + m) * nd + p];
  };

  // ---------------- reverse ----------------
  const double* lam_in = a.lam + (size_t)cell * nd * D + (size_t)(live ? p : 0) * D;
  double lu[D];  // adjoint of this node's luh
#pragma unroll
  for (int m = 0; m < D; m++) lu[m] = 0.0;

  // extrapolation (lQhbnd, lFhbnd from lQhi, lFhi) transposed
  double lQhi[D], lFhi[DIM * V];
#pragma unroll
  for (int m = 0; m < D; m++) lQhi[m] = 0.0;
  if (live) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int fn = node_line<DIM, n>(p, d), k = co[d];
      const double f0 = G::F0(k), f1 = G::F1(k);
      const double* q0 = a.adjQ + (size_t)cell * S::sizeQhb + (size_t)((2 * d) * S::nf + fn) * D;
      const double* q1 = a.adjQ + (size_t)cell * S::sizeQhb + (size_t)((2 * d + 1) * S::nf + fn) * D;
      const double* f0p = a.adjF + (size_t)cell * S::sizeFhb + (size_t)((2 * d) * S::nf + fn) * V;
      const double* f1p = a.adjF + (size_t)cell * S::sizeFhb + (size_t)((2 * d + 1) * S::nf + fn) * V;
#pragma unroll
      for (int m = 0; m < D; m++) lQhi[m] += f0 * q0[m] + f1 * q1[m];
#pragma unroll
      for (int m = 0; m < V; m++) lFhi[d * V + m] = f0 * f0p[m] + f1 * f1p[m];
    }
    // volume integral transposed: lduh = lambda * dt / w_p; lduh[(L,k)] += sum_mm Kxi[k][mm]
    // lFhi_d[(L,mm)] w_ab / dx_d  ->  lFhi_d[(L,mm)] += dt/dx_d sum_k Kxi[k][mm] lambda[(L,k)] / w_k
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) sF[(d * V + m) * nd + slot[d]] = lam_in[m] / G::weights(co[d]);
  }
  __syncthreads();
  adj_contract<DIM, N, V, TPB, false>(sF, s_cvol);
  __syncthreads();
  if (live) {
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) lFhi[d * V + m] += sF[(d * V + m) * nd + slot[d]];
  }
  __syncthreads();

  // time averaging transposed: lQhi = sum_t w_t q^S_t (parameters: sum_t w_t luh);
  // lFhi = sum_t w_t F(q^{S-1}_t)
  double wsum = 0.0;
#pragma unroll
  for (int t = 0; t < n; t++) wsum += G::weights(t);
#pragma unroll
  for (int m = V; m < D; m++) lu[m] += wsum * lQhi[m];
  double lq[n][V];  // adjoint of the iterate q^s being reversed
  if (live) {
#pragma unroll
    for (int t = 0; t < n; t++)
#pragma unroll
      for (int m = 0; m < V; m++) sQ[(t * nd + p) * V + m] = G::weights(t) * lQhi[m];  // lambda_q^S
#pragma unroll
    for (int t = 0; t < n; t++) {
      double q[D], lF[DIM * V], gq[D];
      iterate(S_ - 1, t, q);
#pragma unroll
      for (int k = 0; k < DIM * V; k++) lF[k] = G::weights(t) * lFhi[k];
#pragma unroll
      for (int m = 0; m < D; m++) gq[m] = 0.0;
      PDE::template flux_vjp<DIM>(q, lF, gq);
#pragma unroll
      for (int m = 0; m < V; m++) lq[t][m] = gq[m];
#pragma unroll
      for (int m = V; m < D; m++) lu[m] += gq[m];
    }
  } else {
#pragma unroll
    for (int t = 0; t < n; t++)
#pragma unroll
      for (int m = 0; m < V; m++) lq[t][m] = 0.0;
  }

  // Picard sweeps in reverse: q^{s+1}_l = (1/w_p) sum_t iK1[l][t] rhs_t, with
  // rhs_t = w_p F0[t] luh - sum_d w_t w_ab dt/dx_d Kxi-contraction of F(q^s_t) (+ source)
  for (int s = S_ - 1; s >= 0; s--) {
    if (live) {
#pragma unroll
      for (int m = 0; m < V; m++) {
        double l1[n];
#pragma unroll
        for (int l = 0; l < n; l++) l1[l] = sQ[(l * nd + p) * V + m];
#pragma unroll
        for (int t = 0; t < n; t++) {
          double r = 0.0;
#pragma unroll
          for (int l = 0; l < n; l++) r = fma(G::iK1(l, t), l1[l], r);
          r *= iweight;
          sR[(t * nd + p) * V + m] = r;
          lu[m] = fma(w_sp * G::F0(t), r, lu[m]);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < n; i++) {
      if (live) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) sF[(d * V + m) * nd + slot[d]] = sR[(i * nd + p) * V + m];
      }
      __syncthreads();
      {
        const double wi = G::weights(i);
        for (int it = threadIdx.x; it < A::items; it += TPB) {
          double* f = sF + (size_t)it * n;
          const int d = it / (V * NL), L = it % NL;
          const double coef = -wi * s_coef[d * NL + L];
          double x[n];
#pragma unroll
          for (int k = 0; k < n; k++) x[k] = f[k];
#pragma unroll
          for (int k = 0; k < n; k++) {
            double acc = 0.0;
#pragma unroll
            for (int l = 0; l < n; l++) acc = fma(G::Kxi(k, l), x[l], acc);
            f[k] = coef * acc;
          }
        }
      }
      __syncthreads();
      if (live) {
        double q[D], lF[DIM * V], gq[D];
        iterate(s, i, q);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) lF[d * V + m] = sF[(d * V + m) * nd + slot[d]];
#pragma unroll
        for (int m = 0; m < D; m++) gq[m] = 0.0;
        PDE::template flux_vjp<DIM>(q, lF, gq);
#pragma unroll
        for (int m = 0; m < V; m++) lq[i][m] += gq[m];
#pragma unroll
        for (int m = V; m < D; m++) lu[m] += gq[m];
      }
      __syncthreads();
    }
    // lambda_q^s is complete: it becomes the input of the next (earlier) sweep
    if (live) {
#pragma unroll
      for (int t = 0; t < n; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          sQ[(t * nd + p) * V + m] = lq[t][m];
          lq[t][m] = 0.0;
        }
    }
  }
  if (live) {
    // q^0_t = luh for every t
#pragma unroll
    for (int t = 0; t < n; t++)
#pragma unroll
      for (int m = 0; m < V; m++) lu[m] += sQ[(t * nd + p) * V + m];
    double* lam_out = a.lam + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
    for (int m = 0; m < D; m++) lam_out[m] = lam_in[m] + lu[m];
  }
}

}  // namespace exa
