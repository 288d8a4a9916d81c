// sm_100a kernels of the ADER-DG cell update (nonlinear, generic-kernel semantics).
//
//   predictor_kernel   fused space-time predictor + time averaging + face extrapolation +
//                      volume integral, one CTA per cell (several for small cells).
//                      Reference: ExaHyPE/kernels/aderdg/generic/c/3d/spaceTimePredictorNonlinear
//                      .cpph:39-864 and 3d/volumeIntegralNonlinear.cpph:133-223 (2D: 2d/...).
//   riemann_kernel     Rusanov flux on interior faces, one warp per face, in place on the face
//                      traces (3d/riemannSolverNonlinear.cpph:37-128).
//   boundary_kernel    boundaryValues ghost state + Rusanov on domain faces
//                      (3d/boundaryConditions.cpph:29-122, glue ...Implementation.template:307-350).
//   update_kernel      surface integral + solution update + CFL time step of the new state,
//                      reduced to one dt per grid (3d/surfaceIntegralNonlinear.cpph:21-90,
//                      3d/solutionUpdate.cpph:28-67, 3d/stableTimeStepSize.cpph:14-62).
//   cfl_kernel         stableTimeStepSize alone (initial dt, batched API).
//
// Device layouts are the reference's per-cell layouts, cells contiguous one after another
// (cell-major): luh[c][node][D], lduh[c][node][V], lQhbnd[c][2*DIM][face node][D],
// lFhbnd[c][2*DIM][face node][V], node = (z*n + y)*n + x, face nodes (a,b) with the slower
// tangential axis first. A CTA reads or writes whole cells, so every access is a contiguous
// block (8.6 KB per cell for 3D Euler N=5).
#pragma once
#include <cstdint>

#include "exa_pde.cuh"
#include "exa_tables.cuh"

namespace exa {

enum : unsigned {
  ST_NONFINITE_PREDICTOR = 1u,
  ST_PICARD_CAP = 2u,
  ST_NONFINITE_UPDATE = 4u,
  ST_BAD_DT = 8u,
};

template <class PDE, int DIM, int N, int P>
struct Shape {
  static constexpr int n = N + 1;
  static constexpr int V = PDE::V;
  static constexpr int D = V + P;
  static constexpr int nd = DIM == 3 ? n * n * n : n * n;  // nodes per cell
  static constexpr int nf = DIM == 3 ? n * n : n;          // nodes per face
  static constexpr int NL = nd / n;                        // lines per direction
  static constexpr int CPB = nd >= 256 ? 1 : 256 / nd;     // cells per CTA
  static constexpr int TPB = (CPB * nd + 31) / 32 * 32;    // whole warps; the tail threads idle
  static constexpr int sizeQhb = 2 * DIM * nf * D;
  static constexpr int sizeFhb = 2 * DIM * nf * V;
  static constexpr int maxSweeps = 2 * n;
  // dynamic shared memory of the predictor: lQi [cell][t][node][D] + flux/partials [cell][dir][V][node]
  static constexpr int smemQ = CPB * n * nd * D;
  static constexpr int smemF = CPB * DIM * V * nd;
  static constexpr size_t predictor_smem = sizeof(double) * (smemQ + smemF);
};

// Arguments shared by the cell kernels (device pointers).
struct CellArgs {
  int ncells;
  const double* luh;
  double* luh_out;          // update kernel: new solution (may alias luh)
  double* lduh;
  double* lQhbnd;
  double* lFhbnd;
  int* picard;              // sweeps executed per cell (nullable)
  const int* cell_grid;     // grid of each cell (nullable: all grid 0)
  const double* grid_dx;    // [grid][3] (nullable: u_dx for every cell)
  const double* grid_dt;    // [grid] time step used by this step (nullable: u_dt)
  double u_dx[3];           // uniform cell size when grid_dx is null
  double u_dt;              // uniform time step when grid_dt is null
  double* grid_dt_next;     // [grid] CFL reduction target (nullable)
  double* cell_dt;          // [cell] per-cell CFL dt (nullable)
  unsigned* status;         // error bits (nullable)
  int max_picard;           // 0: residual test, 2(N+1) cap; > 0: fixed sweep count
  double cfl_pnpm;          // CFL * PNPM
  // optional export of the predictor's internals, reference layouts (per-cell shims, tests)
  double* ex_lQi;
  double* ex_lFi;
  double* ex_lQhi;
  double* ex_lFhi;
};

struct FaceArgs {
  int nfaces;
  const int* left;          // cell on the low side
  const int* right;         // cell on the high side
  const int8_t* dir;        // normal direction
  const double* lQhbnd;
  double* lFhbnd;
  // boundary faces
  const int* bcell;         // cell owning the boundary face
  const int8_t* bface;      // face index 2*dir + orientation
  const int8_t* btype;      // boundary type (EXA_BC_WALL, EXA_BC_OUTFLOW)
};

// ------------------------------------------------------------------------------------------
// geometry helpers (compile-time n)
// ------------------------------------------------------------------------------------------
template <int DIM, int n>
__device__ __forceinline__ int line_base(int dir, int L) {
  if (DIM == 3) {
    if (dir == 0) return L * n;                       // L = z*n + y
    if (dir == 1) return (L / n) * n * n + (L % n);   // L = z*n + x
    return L;                                         // L = y*n + x
  }
  return dir == 0 ? L * n : L;                        // L = y | L = x
}
template <int n>
__device__ __forceinline__ int line_stride(int dir) { return dir == 0 ? 1 : (dir == 1 ? n : n * n); }
template <int DIM, int n>
__device__ __forceinline__ void node_coords(int p, int* c) {
  c[0] = p % n;
  c[1] = (p / n) % n;
  c[2] = DIM == 3 ? p / (n * n) : 0;
}
// line of node p in direction dir, and its coordinate along the line
template <int DIM, int n>
__device__ __forceinline__ int node_line(int p, int dir) {
  int c[3];
  node_coords<DIM, n>(p, c);
  if (DIM == 3) return dir == 0 ? c[2] * n + c[1] : (dir == 1 ? c[2] * n + c[0] : c[1] * n + c[0]);
  return dir == 0 ? c[1] : c[0];
}

template <class T>
__device__ __forceinline__ bool finite(T x) { return isfinite(x); }

__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

// ------------------------------------------------------------------------------------------
// Fused predictor + volume integral
// ------------------------------------------------------------------------------------------
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(Shape<PDE, DIM, N, P>::TPB)
predictor_kernel(CellArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf, NL = S::NL, CPB = S::CPB;
  constexpr bool NCP = PDE::kNCP;
  extern __shared__ double smem[];
  double* sQ = smem;                 // [CPB][n][nd][D]   lQi of the current iterate (time-major)
  double* sF = smem + S::smemQ;      // [CPB][DIM][V][nd] fluxes, then contraction partials in place
  __shared__ double s_w[n], s_Kxi[n * n], s_dudx[n * n], s_F0[n], s_F1[n];
  __shared__ double s_dt[CPB], s_invdx[CPB][3], s_res[CPB];
  __shared__ int s_active[CPB];

  const int tid = threadIdx.x;
  const bool inr = tid < CPB * nd;   // threads past the last cell only help in item loops
  const int lc = inr ? tid / nd : 0; // cell within the CTA
  const int p = inr ? tid % nd : 0;  // node within the cell
  const long cell = (long)blockIdx.x * CPB + lc;
  const bool live = inr && cell < a.ncells;

  if (tid < n) {
    s_w[tid] = G::weights(tid);
    s_F0[tid] = G::F0(tid);
    s_F1[tid] = G::F1(tid);
  }
  if (tid < n * n) {
    s_Kxi[tid] = G::Kxi(tid / n, tid % n);
    s_dudx[tid] = G::dudx(tid / n, tid % n);
  }
  if (tid < CPB) {
    const long c = (long)blockIdx.x * CPB + tid;
    const int g = (c < a.ncells && a.cell_grid) ? a.cell_grid[c] : 0;
    s_dt[tid] = a.grid_dt ? a.grid_dt[g] : a.u_dt;
#pragma unroll
    for (int d = 0; d < 3; d++)
      s_invdx[tid][d] = d < DIM ? 1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 0.0;
    s_active[tid] = c < a.ncells;
  }
  __syncthreads();

  int co[3];
  node_coords<DIM, n>(p, co);
  const double w_sp = DIM == 3 ? s_w[co[2]] * s_w[co[1]] * s_w[co[0]] : s_w[co[1]] * s_w[co[0]];
  const double iweight = 1.0 / w_sp;
  const double dt = s_dt[lc];
  double invDx[3] = {s_invdx[lc][0], s_invdx[lc][1], s_invdx[lc][2]};

  // luh of this node; the trivial initial guess lQi[., t] = luh (:71-82)
  double u[D];
  const double* luh = a.luh + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
  for (int m = 0; m < D; m++) u[m] = live ? luh[m] : 1.0;
  double* q_s = sQ + (size_t)lc * n * nd * D;
  if (inr) {
#pragma unroll
    for (int t = 0; t < n; t++)
#pragma unroll
      for (int m = 0; m < D; m++) q_s[(t * nd + p) * D + m] = u[m];
  }
  double* f_s = sF + (size_t)lc * DIM * V * nd;

  double qn[n][V];      // new iterate lQi[p][t][m], m < V
  double fh[DIM][V];    // time-averaged flux of the current sweep (lFhi)
  double sh[V];         // time-averaged source (lShi), NCP only
  const int maxIter = a.max_picard > 0 ? a.max_picard : S::maxSweeps;
  int sweeps = 0;
  bool done = false;

  // Gradient of the iterate at time node ti and this node: gradQ[d][m] (:111-175), NCP only.
  auto gradient = [&](int ti, double* gq) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int L = node_line<DIM, n>(p, d);
      const int base = line_base<DIM, n>(d, L), st = line_stride<n>(d);
      const int l = co[d];
#pragma unroll
      for (int m = 0; m < V; m++) {
        double g = 0.0;
#pragma unroll
        for (int k = 0; k < n; k++)
          g += 1.0 * invDx[d] * q_s[(ti * nd + base + k * st) * D + m] * s_dudx[l * n + k];
        gq[d * V + m] = g;
      }
    }
  };

  // Phase 2: contractions along every line, in place on f_s. coef excludes/includes w_i.
  auto contract = [&](double wi) {
    for (int it = tid; it < CPB * DIM * V * NL; it += S::TPB) {
      const int L = it % NL;
      int r = it / NL;
      const int m = r % V;
      r /= V;
      const int d = r % DIM;
      const int c = r / DIM;
      double* f = sF + ((size_t)(c * DIM + d) * V + m) * nd;
      const int base = line_base<DIM, n>(d, L), st = line_stride<n>(d);
      const double wt = DIM == 3 ? s_w[L / n] * s_w[L % n] : s_w[L];
      const double coef = wi * wt * s_dt[c] * s_invdx[c][d];
      double x[n];
#pragma unroll
      for (int k = 0; k < n; k++) x[k] = f[base + k * st];
#pragma unroll
      for (int l = 0; l < n; l++) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < n; k++) acc = fma(x[k], G::Kxi(k, l), acc);
        f[base + l * st] = coef * acc;
      }
    }
  };

  for (int s = 0; s < maxIter; s++) {
    if (s_active[lc] == 0) done = true;  // phantom cells and converged cells idle
    const bool work = live && !done;
    // converged cells keep qn/fh/sh of their last sweep: only working cells reset and accumulate
    if (work) {
#pragma unroll
      for (int t = 0; t < n; t++)
#pragma unroll
        for (int m = 0; m < V; m++) qn[t][m] = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int m = 0; m < V; m++) fh[d][m] = 0.0;
#pragma unroll
      for (int m = 0; m < V; m++) sh[m] = 0.0;
    }

    if (s == 0) {
      // First sweep: the iterate is luh at every time node, so the flux, the gradient and the
      // contractions are time-independent; compute them once and weight by w_i per time node.
      double F[DIM * V];
      double S0[V];
      PDE::template flux<DIM>(u, F);
      if (inr) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) f_s[(d * V + m) * nd + p] = F[d * V + m];
      }
      if (NCP) {
        double gq[DIM * V], B[V];
        gradient(0, gq);
        PDE::template ncp<DIM>(u, gq, B);
#pragma unroll
        for (int m = 0; m < V; m++) S0[m] = -B[m];
      }
      __syncthreads();
      contract(1.0);
      __syncthreads();
      double o[V];
#pragma unroll
      for (int m = 0; m < V; m++) {
        double acc = f_s[(0 * V + m) * nd + p];
#pragma unroll
        for (int d = 1; d < DIM; d++) acc += f_s[(d * V + m) * nd + p];
        o[m] = acc;
      }
      if (a.ex_lFi && work) {
        for (int i = 0; i < n; i++) {
          double* e = a.ex_lFi + (size_t)cell * n * nd * (DIM + 1) * V + ((size_t)(i * nd + p) * (DIM + 1)) * V;
          for (int d = 0; d < DIM; d++)
            for (int m = 0; m < V; m++) e[d * V + m] = F[d * V + m];
          if (NCP)
            for (int m = 0; m < V; m++) e[DIM * V + m] = S0[m];
        }
      }
      for (int i = 0; i < n && work; i++) {
        const double wi = G::weights(i);
        const double f0 = G::F0(i);
#pragma unroll
        for (int m = 0; m < V; m++) {
          double rhs = w_sp * f0 * u[m] - wi * o[m];
          if (NCP) rhs += wi * w_sp * dt * S0[m];
          const double r = iweight * rhs;
#pragma unroll
          for (int t = 0; t < n; t++) qn[t][m] = fma(r, G::iK1(t, i), qn[t][m]);
#pragma unroll
          for (int d = 0; d < DIM; d++) fh[d][m] = fma(F[d * V + m], wi, fh[d][m]);
          if (NCP) sh[m] = fma(S0[m], wi, sh[m]);
        }
      }
      __syncthreads();
    } else {
      for (int i = 0; i < n; i++) {
        // Phase 1: flux (and NCP source) of the iterate at time node i (:196-227, :323-367)
        double q[D];
#pragma unroll
        for (int m = 0; m < D; m++) q[m] = q_s[(i * nd + p) * D + m];
        double F[DIM * V];
        double Si[V];
        PDE::template flux<DIM>(q, F);
        if (inr) {
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) f_s[(d * V + m) * nd + p] = F[d * V + m];
        }
        if (NCP) {
          double gq[DIM * V], B[V];
          gradient(i, gq);
          PDE::template ncp<DIM>(q, gq, B);
#pragma unroll
          for (int m = 0; m < V; m++) Si[m] = -B[m];
        }
        if (a.ex_lFi && work) {
          double* e = a.ex_lFi + (size_t)cell * n * nd * (DIM + 1) * V + ((size_t)(i * nd + p) * (DIM + 1)) * V;
          for (int d = 0; d < DIM; d++)
            for (int m = 0; m < V; m++) e[d * V + m] = F[d * V + m];
          if (NCP)
            for (int m = 0; m < V; m++) e[DIM * V + m] = Si[m];
        }
        const double wi = G::weights(i);
        __syncthreads();
        // Phase 2: flux contractions with Kxi along x, y, z (:248-321)
        contract(wi);
        __syncthreads();
        // Phase 3: rhs at time node i and the iK1 time solve (:231-246, :370-405)
        const double f0 = G::F0(i);
#pragma unroll
        for (int m = 0; m < V && work; m++) {
          double rhs = w_sp * f0 * u[m];
#pragma unroll
          for (int d = 0; d < DIM; d++) rhs -= f_s[(d * V + m) * nd + p];
          if (NCP) rhs += wi * w_sp * dt * Si[m];
          const double r = iweight * rhs;
#pragma unroll
          for (int t = 0; t < n; t++) qn[t][m] = fma(r, G::iK1(t, i), qn[t][m]);
#pragma unroll
          for (int d = 0; d < DIM; d++) fh[d][m] = fma(F[d * V + m], wi, fh[d][m]);
          if (NCP) sh[m] = fma(Si[m], wi, sh[m]);
        }
        __syncthreads();
      }
    }

    // residual of this sweep and commit of the new iterate (:370-405)
    double res = 0.0;
    if (work) {
#pragma unroll
      for (int t = 0; t < n; t++)
#pragma unroll
        for (int m = 0; m < V; m++) {
          double* o = &q_s[(t * nd + p) * D + m];
          const double dlt = qn[t][m] - *o;
          res = fma(dlt, dlt, res);
          *o = qn[t][m];
        }
    }
    // per-cell reduction: segmented warp tree, then one shared atomic per segment head
    if (tid < CPB) s_res[tid] = 0.0;
    __syncthreads();
    {
      const int lane = tid & 31;
      const int seg_end = (lc + 1) * nd - 1;  // last thread of this cell
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_down_sync(0xffffffffu, res, off);
        if (lane + off < 32 && tid + off <= seg_end) res += o;
      }
      const bool head = (p == 0) || (lane == 0);
      if (head && work) atomicAdd(&s_res[lc], res);
    }
    __syncthreads();
    const bool was_active = !done;
    if (work) {
      sweeps = s + 1;
      const double r = s_res[lc];
      if (!finite(r)) {
        if (a.status) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
      }
      // exit test (:407-412): |res|^2 < 1e-7^2, unless a fixed sweep count is requested
      if (a.max_picard <= 0 && r < 1e-7 * 1e-7) done = true;
    }
    (void)was_active;
    // keep the block looping until every cell of the CTA has converged
    __syncthreads();
    if (p == 0 && live && done) s_active[lc] = 0;
    __syncthreads();
    bool any = false;
#pragma unroll
    for (int c = 0; c < CPB; c++) any |= s_active[c] != 0;
    if (!any) break;
    __syncthreads();
  }
  if (live && a.picard && p == 0) a.picard[cell] = sweeps;
  if (live && p == 0 && a.max_picard <= 0 && !done && a.status) atomicOr(a.status, ST_PICARD_CAP);
  __syncthreads();

  // ---------------- time averaging (:441-515) ----------------
  // lQhi[p][m] = sum_t w_t lQi[p][t][m]; parameters are constant in time.
  double qh[D];
#pragma unroll
  for (int m = 0; m < D; m++) {
    double acc = 0.0;
#pragma unroll
    for (int t = 0; t < n; t++) acc = fma(m < V ? q_s[(t * nd + p) * D + m] : u[m], G::weights(t), acc);
    qh[m] = acc;
  }
  if (live && a.ex_lQi) {
    double* e = a.ex_lQi + (size_t)cell * nd * n * D + (size_t)p * n * D;
    for (int t = 0; t < n; t++)
      for (int m = 0; m < D; m++) e[t * D + m] = m < V ? q_s[(t * nd + p) * D + m] : u[m];
  }
  __syncthreads();
  // stage lQhi [node][D] and lShi [node][V] in the lQi region, lFhi [dir][V][node] in the flux region
  double* qh_s = q_s;
  double* sh_s = q_s + nd * D;
  if (inr) {
#pragma unroll
    for (int m = 0; m < D; m++) qh_s[p * D + m] = qh[m];
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) f_s[(d * V + m) * nd + p] = fh[d][m];
    if (NCP) {
#pragma unroll
      for (int m = 0; m < V; m++) sh_s[p * V + m] = sh[m];
    }
  }
  if (live && a.ex_lQhi) {
    for (int m = 0; m < D; m++) a.ex_lQhi[(size_t)cell * nd * D + p * D + m] = qh[m];
  }
  if (live && a.ex_lFhi) {
    // reference lFhi blocks: x [z][y][x], y [z][x][y], z [y][x][z], source [z][y][x]
    double* e = a.ex_lFhi + (size_t)cell * (DIM + 1) * nd * V;
    for (int d = 0; d < DIM; d++) {
      const int L = node_line<DIM, n>(p, d);
      const int idx = L * n + co[d];
      for (int m = 0; m < V; m++) e[(size_t)d * nd * V + idx * V + m] = fh[d][m];
    }
    for (int m = 0; m < V; m++) e[(size_t)DIM * nd * V + p * V + m] = NCP ? sh[m] : 0.0;
  }
  __syncthreads();

  // ---------------- volume integral (volumeIntegralNonlinear :133-223) ----------------
  if (live) {
    double* lduh = a.lduh + (size_t)cell * nd * V + (size_t)p * V;
    double acc[V];
#pragma unroll
    for (int m = 0; m < V; m++) acc[m] = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int L = node_line<DIM, n>(p, d);
      const int base = line_base<DIM, n>(d, L), st = line_stride<n>(d);
      const double wt = DIM == 3 ? s_w[L / n] * s_w[L % n] : s_w[L];
      const double us = wt * invDx[d];
      const int k = co[d];
#pragma unroll
      for (int m = 0; m < V; m++)
#pragma unroll
        for (int mm = 0; mm < n; mm++)
          acc[m] += s_Kxi[k * n + mm] * f_s[(d * V + m) * nd + base + mm * st] * us;
    }
    if (NCP) {
#pragma unroll
      for (int m = 0; m < V; m++) acc[m] += w_sp * sh_s[p * V + m];
    }
    bool ok = true;
#pragma unroll
    for (int m = 0; m < V; m++) {
      lduh[m] = acc[m];
      ok &= finite(acc[m]);
    }
    if (!ok && a.status) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
  }

  // ---------------- extrapolation to the faces (:517-687) ----------------
  // lQhbnd[c][face][fn][D] then lFhbnd[c][face][fn][V]; item index runs over the output block
  for (int j = tid; j < CPB * (S::sizeQhb + S::sizeFhb); j += S::TPB) {
    const int c = j / (S::sizeQhb + S::sizeFhb);
    const long gc = (long)blockIdx.x * CPB + c;
    if (gc >= a.ncells) continue;
    int r = j % (S::sizeQhb + S::sizeFhb);
    const bool isQ = r < S::sizeQhb;
    if (!isQ) r -= S::sizeQhb;
    const int W = isQ ? D : V;
    const int m = r % W;
    const int fn = (r / W) % nf;
    const int face = r / (W * nf);
    const int d = face >> 1, o = face & 1;
    const int base = line_base<DIM, n>(d, fn), st = line_stride<n>(d);
    double acc = 0.0;
    if (isQ) {
      // 2D x faces extrapolate only the evolved variables (2d/spaceTimePredictorNonlinear.cpph:436-445)
      if (!(DIM == 2 && d == 0 && m >= V)) {
        const double* src = smem + (size_t)c * n * nd * D;
#pragma unroll
        for (int l = 0; l < n; l++) acc = fma(src[(base + l * st) * D + m], o ? G::F1(l) : G::F0(l), acc);
      }
      a.lQhbnd[(size_t)gc * S::sizeQhb + r] = acc;
    } else {
      const double* src = sF + ((size_t)(c * DIM + d) * V + m) * nd;
#pragma unroll
      for (int l = 0; l < n; l++) acc = fma(src[base + l * st], o ? G::F1(l) : G::F0(l), acc);
      a.lFhbnd[(size_t)gc * S::sizeFhb + r] = acc;
    }
  }
}

// ------------------------------------------------------------------------------------------
// Rusanov on interior faces: one warp per face, in place on lFhbnd
// ------------------------------------------------------------------------------------------
template <class PDE, int DIM, int N, int P>
__device__ __forceinline__ void rusanov_face(const double* QL, const double* QR, double* FL, double* FR, int d,
                                             int lane, bool ghostL, bool ghostR, int ghost_normal) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nf = S::nf;
  // face averages (averageRiemannInputs, RiemannSolverUtils.h:152-177)
  double aL[D], aR[D];
#pragma unroll
  for (int m = 0; m < D; m++) aL[m] = aR[m] = 0.0;
  for (int fn = lane; fn < nf; fn += 32) {
    const double w = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
    double ql[D], qr[D];
#pragma unroll
    for (int m = 0; m < D; m++) {
      ql[m] = QL[fn * D + m];
      qr[m] = QR[fn * D + m];
    }
    if (ghostL) PDE::template wall<DIM>(qr, ghost_normal, ql);
    if (ghostR) PDE::template wall<DIM>(ql, ghost_normal, qr);
    if (ghostL || ghostR) {
#pragma unroll
      for (int m = V; m < D; m++) {
        ql[m] = ghostL ? qr[m] : ql[m];
        qr[m] = ghostR ? ql[m] : qr[m];
      }
    }
#pragma unroll
    for (int m = 0; m < D; m++) {
      aL[m] += w * ql[m];
      aR[m] += w * qr[m];
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
  double lL[V], lR[V];
  PDE::template eigenvalues<DIM>(aL, d, lL);
  PDE::template eigenvalues<DIM>(aR, d, lR);
  double sL = fabs(lL[0]), sR = fabs(lR[0]);
#pragma unroll
  for (int m = 1; m < V; m++) {
    sL = fmax(sL, fabs(lL[m]));
    sR = fmax(sR, fabs(lR[m]));
  }
  const double smax = fmax(sL, sR);
  for (int fn = lane; fn < nf; fn += 32) {
    double ql[D], qr[D], fl[V], fr[V];
#pragma unroll
    for (int m = 0; m < D; m++) {
      ql[m] = QL[fn * D + m];
      qr[m] = QR[fn * D + m];
    }
    if (ghostL) PDE::template wall<DIM>(qr, ghost_normal, ql);
    if (ghostR) PDE::template wall<DIM>(ql, ghost_normal, qr);
    if (ghostL || ghostR) {
#pragma unroll
      for (int m = V; m < D; m++) {
        ql[m] = ghostL ? qr[m] : ql[m];
        qr[m] = ghostR ? ql[m] : qr[m];
      }
      // boundaryValues returns the flux of the ghost state in the normal direction
      double Fg[DIM * V];
      PDE::template flux<DIM>(ghostL ? ql : qr, Fg);
#pragma unroll
      for (int m = 0; m < V; m++) {
        fl[m] = ghostL ? Fg[d * V + m] : FL[fn * V + m];
        fr[m] = ghostR ? Fg[d * V + m] : FR[fn * V + m];
      }
    } else {
#pragma unroll
      for (int m = 0; m < V; m++) {
        fl[m] = FL[fn * V + m];
        fr[m] = FR[fn * V + m];
      }
    }
    double ncp[V];
    if (PDE::kNCP) {
      double gq[DIM * V], qa[D];
#pragma unroll
      for (int k = 0; k < DIM * V; k++) gq[k] = 0.0;
#pragma unroll
      for (int m = 0; m < V; m++) gq[d * V + m] = qr[m] - ql[m];
#pragma unroll
      for (int m = 0; m < D; m++) qa[m] = 0.5 * (qr[m] + ql[m]);
      PDE::template ncp<DIM>(qa, gq, ncp);
    }
#pragma unroll
    for (int m = 0; m < V; m++) {
      const double F = 0.5 * (fr[m] + fl[m]) - 0.5 * smax * (qr[m] - ql[m]);
      double oL = F, oR = F;
      if (PDE::kNCP) {
        oR = F - 0.5 * ncp[m];
        oL = F + 0.5 * ncp[m];
      }
      if (!ghostL) FL[fn * V + m] = oL;
      if (!ghostR) FR[fn * V + m] = oR;
    }
  }
}

template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) riemann_kernel(FaceArgs f) {
  using S = Shape<PDE, DIM, N, P>;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= f.nfaces) return;
  const int d = f.dir[warp];
  const long cl = f.left[warp], cr = f.right[warp];
  const double* QL = f.lQhbnd + cl * S::sizeQhb + (2 * d + 1) * S::nf * S::D;
  const double* QR = f.lQhbnd + cr * S::sizeQhb + (2 * d) * S::nf * S::D;
  double* FL = f.lFhbnd + cl * S::sizeFhb + (2 * d + 1) * S::nf * S::V;
  double* FR = f.lFhbnd + cr * S::sizeFhb + (2 * d) * S::nf * S::V;
  rusanov_face<PDE, DIM, N, P>(QL, QR, FL, FR, d, lane, false, false, d);
}

// Domain-boundary faces with a reflective wall: the ghost state is the mirrored inner state,
// its flux the flux of the ghost state; the Riemann solver sees it on the outer side.
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) boundary_kernel(FaceArgs f) {
  using S = Shape<PDE, DIM, N, P>;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= f.nfaces) return;
  const long c = f.bcell[warp];
  const int face = f.bface[warp];
  const int d = face >> 1, o = face & 1;
  const double* Q = f.lQhbnd + c * S::sizeQhb + face * S::nf * S::D;
  double* F = f.lFhbnd + c * S::sizeFhb + face * S::nf * S::V;
  // orientation 0: the cell is on the right of the face (ghost left); 1: ghost right
  if (o == 0)
    rusanov_face<PDE, DIM, N, P>(Q, Q, F, F, d, lane, true, false, d);
  else
    rusanov_face<PDE, DIM, N, P>(Q, Q, F, F, d, lane, false, true, d);
}

// ------------------------------------------------------------------------------------------
// Surface integral + solution update + CFL of the new state
// ------------------------------------------------------------------------------------------
template <class PDE, int DIM, int N, int P, bool SURFACE, bool UPDATE>
__global__ void __launch_bounds__(Shape<PDE, DIM, N, P>::TPB) update_kernel(CellArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf, CPB = S::CPB;
  __shared__ double sFb[CPB * S::sizeFhb];
  __shared__ double s_w[n], s_F0[n], s_F1[n], s_min[CPB];
  const int tid = threadIdx.x;
  const bool inr = tid < CPB * nd;
  const int lc = inr ? tid / nd : 0, p = inr ? tid % nd : 0;
  const long cell = (long)blockIdx.x * CPB + lc;
  const bool live = inr && cell < a.ncells;
  if (tid < n) {
    s_w[tid] = G::weights(tid);
    s_F0[tid] = G::F0(tid);
    s_F1[tid] = G::F1(tid);
  }
  if (tid < CPB) s_min[tid] = __longlong_as_double(0x7ff0000000000000ll);
  if (SURFACE) {
    for (int j = tid; j < CPB * S::sizeFhb; j += S::TPB) {
      const long gc = (long)blockIdx.x * CPB + j / S::sizeFhb;
      sFb[j] = gc < a.ncells ? a.lFhbnd[(size_t)blockIdx.x * CPB * S::sizeFhb + j] : 0.0;
    }
  }
  __syncthreads();
  const int g = (live && a.cell_grid) ? a.cell_grid[cell] : 0;
  double invDx[3];
#pragma unroll
  for (int d = 0; d < 3; d++) invDx[d] = d < DIM ? 1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 0.0;
  int co[3];
  node_coords<DIM, n>(p, co);
  double q[D];
  bool ok = true;
  if (live) {
    const double* luh = a.luh + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
    for (int m = 0; m < D; m++) q[m] = luh[m];
    if (UPDATE) {
      double du[V];
      const double* lduh = a.lduh + (size_t)cell * nd * V + (size_t)p * V;
#pragma unroll
      for (int m = 0; m < V; m++) du[m] = lduh[m];
      if (SURFACE) {
        const double* Fb = sFb + lc * S::sizeFhb;
#pragma unroll
        for (int d = 0; d < DIM; d++) {
          const int fn = node_line<DIM, n>(p, d);
          const double wt = DIM == 3 ? s_w[fn / n] * s_w[fn % n] : s_w[fn];
          const double us = wt * invDx[d];
          const int k = co[d];
#pragma unroll
          for (int m = 0; m < V; m++)
            du[m] -= (Fb[((2 * d + 1) * nf + fn) * V + m] * s_F1[k] - Fb[((2 * d) * nf + fn) * V + m] * s_F0[k]) * us;
        }
      }
      const double w_sp = DIM == 3 ? s_w[co[2]] * s_w[co[1]] * s_w[co[0]] : s_w[co[1]] * s_w[co[0]];
      const double updateSize = (a.grid_dt ? a.grid_dt[g] : a.u_dt) / w_sp;
      double* out = a.luh_out + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
      for (int m = 0; m < V; m++) {
        q[m] = q[m] + du[m] * updateSize;
        ok &= finite(q[m]);
        out[m] = q[m];
      }
      if (a.luh_out != a.luh) {
#pragma unroll
        for (int m = V; m < D; m++) out[m] = q[m];
      }
    }
  }
  // CFL of the (new) state (stableTimeStepSize :14-62)
  double dtp = __longlong_as_double(0x7ff0000000000000ll);
  if (live && (a.grid_dt_next || a.cell_dt)) {
    double den = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      double lam[V];
      PDE::template eigenvalues<DIM>(q, d, lam);
      double mx = 0.0;
#pragma unroll
      for (int m = 0; m < V; m++) mx = fmax(fabs(lam[m]), mx);
      den += mx * invDx[d];
    }
    dtp = a.cfl_pnpm / den;
    if (!(dtp > 0.0)) {  // NaN or non-positive
      if (a.status) atomicOr(a.status, ST_BAD_DT);
      dtp = __longlong_as_double(0x7ff0000000000000ll);
    }
  }
  if (!ok && a.status) atomicOr(a.status, ST_NONFINITE_UPDATE);
  // per-cell min: warp tree min restricted to the cell's lanes, shared atomic per segment head
  {
    const int lane = tid & 31;
    const int seg_end = (lc + 1) * nd - 1;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, dtp, off);
      if (lane + off < 32 && tid + off <= seg_end) dtp = fmin(dtp, o);
    }
    if ((p == 0 || lane == 0) && live) atomic_min_pos(&s_min[lc], dtp);
  }
  __syncthreads();
  if (p == 0 && live) {
    if (a.cell_dt) a.cell_dt[cell] = s_min[lc];
    if (a.grid_dt_next) atomic_min_pos(&a.grid_dt_next[g], s_min[lc]);
  }
}

// t += dt, dt = dt_next, dt_next = +inf for every grid (one thread per grid).
__global__ void advance_kernel(int ngrids, double* t, double* dt, double* dt_next, long long* steps) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrids) return;
  t[g] += dt[g];
  dt[g] = dt_next[g];
  dt_next[g] = __longlong_as_double(0x7ff0000000000000ll);
  if (g == 0 && steps) steps[0] += 1;
}

__global__ void fill_kernel(int count, double* x, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) x[i] = v;
}

}  // namespace exa
