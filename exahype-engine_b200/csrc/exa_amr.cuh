// Mesh-level projections and the a-posteriori subcell limiter's cell kernels, batched.
//
// Mesh levels (reference 3d/amrRoutines.cpph, 2d/amrRoutines.cpph): a fine cell of a 3:1 refined
// mesh lies in the third j of its parent along each axis; over levelDelta levels its subcell index
// along an axis has levelDelta base-3 digits. Every single-level operator is a tensor product of 1D
// matrices, so the multi-level one is too:
//   prolongation  fine = coarse x_axis T,  T = P_{j1} P_{j2} ... P_{jL}  (j1 the most significant
//                 digit), P_j[k][m] = phi_k((j + x_m) / 3) (AmrT<N>::fine);
//   restriction   coarse += fine x_axis T, T = R_{j1} R_{j2} ... R_{jL}  (j1 the least significant
//                 digit), R_j[k][m] = w_k P_j[m][k] / (3 w_m) -- the L2 projection onto the coarse
//                 basis over the subcell, the reference's w_n P / (w_m 3^DIM) per dimension.
// Each job's composed 1D operators are built in shared memory and applied by sum factorisation
// (one 1D contraction per axis), variable by variable. The reference applies the single levels one
// after another with the full DIM-fold sums; the results agree to rounding.
//
// Limiter (limiter/generic/c/Limiter.cpph) with a finite-volume patch of P = 2N+1 subcells per axis
// and ghost layers of width g (the generated limiting solver's PatchSize and GhostLayerWidth):
//   projectOnFVLimiterSpace  lim = luh x_axis dg2fv (interior subcells only; ghosts untouched),
//   projectOnDGSpace         luh = lim x_axis fv2dg (interior subcells),
//   findCellLocalMinAndMax   min / max of each observable over the nodes, the Gauss-Lobatto nodes
//                            (luh x_axis leg2lob) and the subcell means (luh x_axis dg2fv),
//   findCellLocalLimiterMinAndMax  over the interior subcells,
//   discreteMaximumPrincipleAndMinAndMaxSearch  the local min / max against the min / max of the
//                            2 DIM neighbour blocks, relaxed by max((max - min) * scale, relax).
// Observables are the first nobs variables (the generated solver's default
// mapDiscreteMaximumPrincipleObservables); the relaxation parameter is the specified one (its default
// getDiscreteMaximumPrincipleRelaxationParameter).
#pragma once
#include "exa_amr_tables.cuh"

namespace exa {

constexpr int kAmrMaxLevelDelta = 12;  // 3^12 subintervals per axis fit an int
constexpr unsigned ST_BAD_JOB = 32;     // EXA_ST_BAD_JOB

struct AmrArgs {
  int mode;              // 0 prolongation (overwrite), 1 restriction (accumulate), 2 flux-only restriction (overwrite)
  double* outQ;          // volume: luh blocks; face: lQhbnd blocks (unused in mode 2)
  const double* inQ;
  double* outF;          // face only: lFhbnd blocks
  const double* inF;
  long long nfine, ncoarse;  // blocks in the fine and coarse arrays (index bounds)
  int ngroups;           // CTAs; group g = jobs [ptr[g], ptr[g+1]), or job g alone when ptr is null
  const int* ptr;
  int njobs;             // entries of jobs (bounds of ptr)
  const int* jobs;       // [job][6]: fine block, coarse block, levelDelta, subcell index (DIM or DIM-1 digits)
  unsigned* status;
};

constexpr int kAmrThreads = 256;

// 1D contraction along one axis of a row-major block, extents known at compile time:
// out[b][m][a] = sum_k in[b][k][a] M(k, m) for b < BEFORE (slower axes), a < AFTER (faster axes and
// the variables of a chunk), k < KIN, m < KOUT. One thread per line (b, a): the line's KIN inputs
// are loaded once and its KOUT outputs formed in registers, so shared memory sees one load per
// input and one store per output rather than one load per multiply-add. M(k, m) is a uniform
// operand (a constant-bank table or a shared-memory broadcast). sink(o, value) receives output
// o = (b KOUT + m) AFTER + a; thread t takes lines t, t + STEP, ... (with STEP and AFTER multiples of
// the chunk width, a thread stays on one variable).
template <int BEFORE, int KIN, int KOUT, int AFTER, int STEP = kAmrThreads, class Mat, class Sink>
__device__ __forceinline__ void sweep(const double* __restrict__ in, Mat&& M, Sink&& sink) {
  constexpr int lines = BEFORE * AFTER;
  if ((int)threadIdx.x >= STEP) return;
  for (int l = threadIdx.x; l < lines; l += STEP) {
    const int a = l % AFTER, b = l / AFTER;
    const double* src = in + b * KIN * AFTER + a;
    double x[KIN];
#pragma unroll
    for (int k = 0; k < KIN; k++) x[k] = src[k * AFTER];
#pragma unroll
    for (int m = 0; m < KOUT; m++) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < KIN; k++) acc = fma(x[k], M(k, m), acc);
      sink((b * KOUT + m) * AFTER + a, acc);
    }
  }
}
template <int BEFORE, int KIN, int KOUT, int AFTER, class Mat>
__device__ __forceinline__ void sweep_to(const double* __restrict__ in, double* __restrict__ out, Mat&& M) {
  sweep<BEFORE, KIN, KOUT, AFTER>(in, M, [&](int o, double v) { out[o] = v; });
}

// the composed 1D operators of one job along R axes into T[R][n][n] (W: scratch of the same size);
// false when the job's level difference or a digit string is out of range
template <int N>
__device__ bool amr_operators(int mode, int R, const int* job, double* T, double* W) {
  using A = AmrT<N>;
  using G = GL<N>;
  constexpr int n = N + 1;
  const int L = job[2];
  bool ok = L >= 1 && L <= kAmrMaxLevelDelta;
  int span = 1;
  for (int l = 0; l < (ok ? L : 0); l++) span *= 3;
  for (int r = 0; r < R; r++) ok = ok && job[3 + r] >= 0 && job[3 + r] < span;
  if (!ok) return false;
  // digit of level step l (0-based) along axis r
  auto digit = [&](int r, int l) -> int {
    int p = 1;
    const int e = mode == 0 ? L - 1 - l : l;  // prolongation: most significant first
    for (int q = 0; q < e; q++) p *= 3;
    return (job[3 + r] / p) % 3;
  };
  auto single = [&](int j, int k, int m) -> double {
    return mode == 0 ? A::fine(j, k, m) : G::weights(k) * A::fine(j, m, k) / (3.0 * G::weights(m));
  };
  for (int e = threadIdx.x; e < R * n * n; e += blockDim.x) {
    const int r = e / (n * n), k = (e / n) % n, m = e % n;
    T[e] = single(digit(r, 0), k, m);
  }
  __syncthreads();
  for (int l = 1; l < L; l++) {
    for (int e = threadIdx.x; e < R * n * n; e += blockDim.x) {
      const int r = e / (n * n), k = (e / n) % n, m = e % n;
      const int j = digit(r, l);
      double acc = 0.0;
      for (int q = 0; q < n; q++) acc = fma(T[r * n * n + k * n + q], single(j, q, m), acc);
      W[e] = acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < R * n * n; e += blockDim.x) T[e] = W[e];
    __syncthreads();
  }
  return true;
}

// Shared-memory plan of the mesh-level kernel: the variables of a block are processed in chunks of
// VC (all of them where two chunk buffers fit `budget`), so that a block is staged with contiguous
// loads and every sweep contracts all variables of the chunk at once.
template <int N, int R, int NV>
struct AmrShape {
  static constexpr int n = N + 1;
  static constexpr int nb = R == 3 ? n * n * n : (R == 2 ? n * n : n);
  static constexpr int budget = 64 * 1024;
  static constexpr int fit = budget / (2 * nb * 8);
  static constexpr int VC = fit >= NV ? NV : (fit < 1 ? 1 : fit);
  static constexpr size_t smem = sizeof(double) * (2 * (size_t)nb * VC + 6 * n * n);
};

// the R sweeps of one chunk: X (input) -> Y -> X (-> Y), the last one into `sink`
template <int n, int R, int VC, class Sink>
__device__ __forceinline__ void amr_sweeps(double* X, double* Y, const double* T, Sink&& sink) {
  auto axis = [&](int r) { return [T, r](int k, int m) { return T[(r * n + k) * n + m]; }; };
  if constexpr (R == 3) {
    sweep_to<n * n, n, n, VC>(X, Y, axis(0));
    __syncthreads();
    sweep_to<n, n, n, n * VC>(Y, X, axis(1));
    __syncthreads();
    sweep<1, n, n, n * n * VC>(X, axis(2), sink);
  } else if constexpr (R == 2) {
    sweep_to<n, n, n, VC>(X, Y, axis(0));
    __syncthreads();
    sweep<1, n, n, n * VC>(Y, axis(1), sink);
  } else {
    sweep<1, n, n, VC>(X, axis(0), sink);
  }
}

// One group of jobs per CTA. R = axes of a block (DIM for cells, DIM - 1 for faces); the Q blocks
// have DQ doubles per node, the F blocks (faces) V. Dynamic shared memory: AmrShape<N, R, DQ>::smem.
template <int N, int R, int DQ, int V, bool FACE>
__global__ void __launch_bounds__(kAmrThreads) amr_kernel(AmrArgs a) {
  using Sh = AmrShape<N, R, DQ>;
  constexpr int n = N + 1, nb = Sh::nb, VC = Sh::VC;
  extern __shared__ __align__(16) double sm[];
  double* X = sm;                 // [nb][VC] each
  double* Y = X + nb * VC;
  double* T = Y + nb * VC;        // [R][n][n]
  double* W = T + 3 * n * n;
  const int g = blockIdx.x;
  const int j0 = a.ptr ? a.ptr[g] : g, j1 = a.ptr ? a.ptr[g + 1] : g + 1;
  if (j0 < 0 || j1 > a.njobs || j1 < j0) {
    if (threadIdx.x == 0 && a.status) atomicOr(a.status, ST_BAD_JOB);
    return;
  }
  if (j1 == j0) return;
  const long long coarse0 = a.jobs[6 * j0 + 1];
  const int first_arr = (FACE && a.mode == 2) ? 1 : 0;
  for (int j = j0; j < j1; j++) {
    const int* job = a.jobs + 6 * j;
    const long long fine = job[0], coarse = job[1];
    // a restriction group accumulates into one coarse block; the test is uniform over the CTA
    bool ok = fine >= 0 && fine < a.nfine && coarse >= 0 && coarse < a.ncoarse && (a.mode == 0 || coarse == coarse0);
    __syncthreads();  // T and the chunk buffers of the previous job are free
    ok = ok && amr_operators<N>(a.mode == 0 ? 0 : 1, R, job, T, W);
    if (!ok) {
      if (threadIdx.x == 0 && a.status) atomicOr(a.status, ST_BAD_JOB);
      continue;
    }
    const long long src_blk = a.mode == 0 ? coarse : fine;
    const long long dst_blk = a.mode == 0 ? fine : coarse;
    // restriction: the coarse values (mode 1; zero in mode 2) plus the children in job order,
    // read from and written back to the coarse block job by job (the jobs of a group run in order
    // in this CTA, a barrier apart)
    const bool add = a.mode == 1 || (a.mode == 2 && j > j0);
    for (int arr = first_arr; arr < (FACE ? 2 : 1); arr++) {
      const int nv = arr == 0 ? DQ : V;
      double* out = arr == 0 ? a.outQ : a.outF;
      const double* in = arr == 0 ? a.inQ : a.inF;
      for (int v0 = 0; v0 < nv; v0 += VC) {
        const int vc = nv - v0 < VC ? nv - v0 : VC;  // the last chunk is zero-padded to VC
        __syncthreads();
        for (int e = threadIdx.x; e < nb * VC; e += kAmrThreads) {
          const int p = e / VC, c = e % VC;
          X[e] = c < vc ? in[((size_t)src_blk * nb + p) * nv + v0 + c] : 0.0;
        }
        __syncthreads();
        double* o = out + (size_t)dst_blk * nb * nv + v0;
        amr_sweeps<n, R, VC>(X, Y, T, [&](int e, double x) {
          const int p = e / VC, c = e % VC;
          if (c < vc) {
            double* d = o + (size_t)p * nv + c;
            *d = add ? *d + x : x;
          }
        });
      }
    }
  }
}

struct LimArgs {
  int op;           // 0 luh -> lim, 1 lim -> luh, 2 min/max of luh, 3 min/max of lim, 4 discrete maximum principle
  int ncells, ghost, nobs;
  const double* luh;   // [cell][n^DIM][D]
  double* luh_out;
  const double* lim;   // [cell][(P + 2 ghost)^DIM][D]
  double* lim_out;
  double* mn;          // op 2, 3: [cell][nobs]; op 4: [cell][2 DIM][nobs], read and rewritten
  double* mx;
  unsigned char* ok;   // op 4: 1 where the principle holds
  double relax, scale;
};

// Shared-memory plan of the limiter kernel: the DG block of a chunk of VC variables and two sweep
// intermediates (at most n P^2 points each), all variables of the chunk contracted together.
template <int N, int DIM, int D>
struct LimShape {
  static constexpr int n = N + 1, P = 2 * N + 1;
  static constexpr int nb = DIM == 3 ? n * n * n : n * n;
  static constexpr int pb = DIM == 3 ? P * P * P : P * P;
  static constexpr int mid = DIM == 3 ? n * P * P : n * P;
  static constexpr int budget = 72 * 1024;
  static constexpr int fit = budget / (8 * (nb + 2 * mid));
  static constexpr int VC = fit >= D ? D : (fit < 1 ? 1 : fit);
  static constexpr int STEP = (kAmrThreads / VC) * VC;  // threads on one variable each
  static constexpr size_t smem = sizeof(double) * ((size_t)(nb + 2 * mid) * VC + 3 * n * P + 2 * kAmrThreads);
};

// one cell per CTA
template <int N, int DIM, int D>
__global__ void __launch_bounds__(kAmrThreads) limiter_kernel(LimArgs a) {
  using A = AmrT<N>;
  using Sh = LimShape<N, DIM, D>;
  constexpr int n = Sh::n, P = Sh::P, nb = Sh::nb, pb = Sh::pb, VC = Sh::VC, STEP = Sh::STEP;
  extern __shared__ __align__(16) double sm[];
  double* U = sm;                  // [nb][VC] DG values of the chunk
  double* M1 = U + nb * VC;        // sweep intermediates
  double* M2 = M1 + Sh::mid * VC;
  double* dg2fv = M2 + Sh::mid * VC;   // [n][P]
  double* fv2dg = dg2fv + n * P;       // [P][n]
  double* l2l = fv2dg + n * P;         // [n][n]
  double* red_lo = dg2fv + 3 * n * P;  // [threads] per-thread partial extrema
  double* red_hi = red_lo + kAmrThreads;
  __shared__ double s_lmin[32], s_lmax[32];
  const int c = blockIdx.x;
  const int g = a.ghost;
  const int E = P + 2 * g;
  const size_t ext = DIM == 3 ? (size_t)E * E * E : (size_t)E * E;
  for (int e = threadIdx.x; e < n * P; e += kAmrThreads) {
    dg2fv[e] = A::dg2fv(e / P, e % P);
    fv2dg[e] = A::fv2dg(e / n, e % n);
  }
  for (int e = threadIdx.x; e < n * n; e += kAmrThreads) l2l[e] = A::leg2lob(e / n, e % n);
  if (a.op == 4 && threadIdx.x == 0) a.ok[c] = 1;
  __syncthreads();
  // interior subcell s = (z P + y) P + x -> its offset in the patch with ghosts
  auto lim_at = [&](int s) -> size_t {
    const int x = s % P, y = (s / P) % P, z = DIM == 3 ? s / (P * P) : 0;
    return DIM == 3 ? ((size_t)(z + g) * E + (y + g)) * E + (x + g) : (size_t)(y + g) * E + (x + g);
  };
  const double* luh = a.luh ? a.luh + (size_t)c * nb * D : nullptr;
  const double* lim = a.lim ? a.lim + (size_t)c * ext * D : nullptr;
  const int nvar = (a.op <= 1) ? D : a.nobs;
  const int myv = (int)threadIdx.x < STEP ? (int)threadIdx.x % VC : -1;  // this thread's variable in extrema passes
  // the projectors as uniform operands of the unrolled sweeps (constant bank)
  auto d2f = [](int k, int m) { return A::dg2fv(k, m); };
  auto f2d = [](int i, int k) { return A::fv2dg(i, k); };
  auto l2b = [](int k, int i) { return A::leg2lob(k, i); };

  // the pass's per-variable extrema merged into s_lmin / s_lmax (fmin / fmax skip a NaN value,
  // as the reference's std::min(acc, x) / std::max(acc, x) do)
  auto extrema_end = [&](double lo, double hi, int vc) {
    red_lo[threadIdx.x] = lo;
    red_hi[threadIdx.x] = hi;
    __syncthreads();
    if ((int)threadIdx.x < vc) {
      double m0 = INFINITY, m1 = -INFINITY;
      for (int t = threadIdx.x; t < STEP; t += VC) {
        m0 = fmin(m0, red_lo[t]);
        m1 = fmax(m1, red_hi[t]);
      }
      s_lmin[threadIdx.x] = fmin(s_lmin[threadIdx.x], m0);
      s_lmax[threadIdx.x] = fmax(s_lmax[threadIdx.x], m1);
    }
    __syncthreads();
  };

  for (int v0 = 0; v0 < nvar; v0 += VC) {
    const int vc = nvar - v0 < VC ? nvar - v0 : VC;  // the last chunk is zero-padded to VC
    if (threadIdx.x < 32) {
      s_lmin[threadIdx.x] = INFINITY;
      s_lmax[threadIdx.x] = -INFINITY;
    }
    if (a.op == 0 || a.op == 2 || a.op == 4) {
      for (int e = threadIdx.x; e < nb * VC; e += kAmrThreads)
        U[e] = (e % VC) < vc ? luh[(size_t)(e / VC) * D + v0 + e % VC] : 0.0;
      __syncthreads();
    }
    if (a.op == 0) {
      // subcell means: x, y sweeps into M1, M2, the z sweep straight into the patch
      double* out = a.lim_out + (size_t)c * ext * D + v0;
      auto store = [&](int o, double x) {
        if (o % VC < vc) out[lim_at(o / VC) * D + o % VC] = x;
      };
      if constexpr (DIM == 3) {
        sweep_to<n * n, n, P, VC>(U, M1, d2f);
        __syncthreads();
        sweep_to<n, n, P, P * VC>(M1, M2, d2f);
        __syncthreads();
        sweep<1, n, P, P * P * VC>(M2, d2f, store);
      } else {
        sweep_to<n, n, P, VC>(U, M1, d2f);
        __syncthreads();
        sweep<1, n, P, P * VC>(M1, d2f, store);
      }
      __syncthreads();
    } else if (a.op == 1) {
      // the interior subcells of the chunk, read straight from the patch by the x sweep:
      // M1[row][k][cc] = sum_i lim[row][i][cc] fv2dg[i][k], row = (z, y)
      constexpr int rows = DIM == 3 ? P * P : P;
      for (int o = threadIdx.x; o < rows * n * VC; o += kAmrThreads) {
        const int cc = o % VC, k = (o / VC) % n, row = o / (VC * n);
        double acc = 0.0;
        if (cc < vc) {
          const double* src = lim + lim_at(row * P) * D + v0 + cc;  // x runs contiguously in the patch
#pragma unroll
          for (int i = 0; i < P; i++) acc = fma(src[(size_t)i * D], fv2dg[i * n + k], acc);  // k varies: shared table
        }
        M1[o] = acc;
      }
      __syncthreads();
      double* out = a.luh_out + (size_t)c * nb * D + v0;
      auto store = [&](int o, double x) {
        if (o % VC < vc) out[(size_t)(o / VC) * D + o % VC] = x;
      };
      if constexpr (DIM == 3) {
        sweep_to<P, P, n, n * VC>(M1, M2, f2d);
        __syncthreads();
        sweep<1, P, n, n * n * VC>(M2, f2d, store);
      } else {
        sweep<1, P, n, n * VC>(M1, f2d, store);
      }
      __syncthreads();
    } else if (a.op == 3) {
      double lo = INFINITY, hi = -INFINITY;
      if (myv >= 0 && myv < vc)
        for (int s = threadIdx.x / VC; s < pb; s += STEP / VC) {
          const double x = lim[lim_at(s) * D + v0 + myv];
          lo = fmin(lo, x);
          hi = fmax(hi, x);
        }
      extrema_end(lo, hi, vc);
    } else {  // op 2, 4: the nodes, the Gauss-Lobatto nodes, the subcell means
      double lo = INFINITY, hi = -INFINITY;
      if (myv >= 0 && myv < vc)
        for (int p = threadIdx.x / VC; p < nb; p += STEP / VC) {
          lo = fmin(lo, U[p * VC + myv]);
          hi = fmax(hi, U[p * VC + myv]);
        }
      auto take = [&](int, double x) {
        if (myv < vc) {
          lo = fmin(lo, x);
          hi = fmax(hi, x);
        }
      };
      if constexpr (DIM == 3) {
        sweep_to<n * n, n, n, VC>(U, M1, l2b);
        __syncthreads();
        sweep_to<n, n, n, n * VC>(M1, M2, l2b);
        __syncthreads();
        sweep<1, n, n, n * n * VC, STEP>(M2, l2b, take);
        __syncthreads();
        sweep_to<n * n, n, P, VC>(U, M1, d2f);
        __syncthreads();
        sweep_to<n, n, P, P * VC>(M1, M2, d2f);
        __syncthreads();
        sweep<1, n, P, P * P * VC, STEP>(M2, d2f, take);
      } else {
        sweep_to<n, n, n, VC>(U, M1, l2b);
        __syncthreads();
        sweep<1, n, n, n * VC, STEP>(M1, l2b, take);
        __syncthreads();
        sweep_to<n, n, P, VC>(U, M1, d2f);
        __syncthreads();
        sweep<1, n, P, P * VC, STEP>(M1, d2f, take);
      }
      __syncthreads();
      extrema_end(lo, hi, vc);
    }
    // op 2 / 4: per observable of the chunk (thread 0 of the CTA)
    if ((a.op == 2 || a.op == 4) && threadIdx.x == 0) {
      for (int cc = 0; cc < vc; cc++) {
        const int v = v0 + cc;
        const double lmin = s_lmin[cc], lmax = s_lmax[cc];
        if (a.op == 2) {
          a.mn[(size_t)c * a.nobs + v] = lmin;
          a.mx[(size_t)c * a.nobs + v] = lmax;
          continue;
        }
        double* bmn = a.mn + (size_t)c * 2 * DIM * a.nobs;
        double* bmx = a.mx + (size_t)c * 2 * DIM * a.nobs;
        double bmin = bmn[v], bmax = bmx[v];
        for (int f = 1; f < 2 * DIM; f++) {
          bmin = fmin(bmin, bmn[f * a.nobs + v]);
          bmax = fmax(bmax, bmx[f * a.nobs + v]);
        }
        double sd = (bmax - bmin) * a.scale;
        sd = fmax(sd, a.relax);
        bool ok = !((lmin < bmin - sd) || (lmax > bmax + sd));
        ok = ok && isfinite(lmin) && isfinite(lmax);
        if (!ok) a.ok[c] = 0;
        bmn[v] = lmin;
        bmx[v] = lmax;
        bmn[a.nobs + v] = bmin;
        bmx[a.nobs + v] = bmax;
      }
    } else if (a.op == 3 && threadIdx.x == 0) {
      for (int cc = 0; cc < vc; cc++) {
        a.mn[(size_t)c * a.nobs + v0 + cc] = s_lmin[cc];
        a.mx[(size_t)c * a.nobs + v0 + cc] = s_lmax[cc];
      }
    }
    __syncthreads();
  }
}

// Warp-level sweep: the lanes of one warp take the lines of a single-variable block (BEFORE x AFTER
// lines), synchronising with __syncwarp only. Same contraction as `sweep`.
template <int BEFORE, int KIN, int KOUT, int AFTER, class Mat, class Sink>
__device__ __forceinline__ void warp_sweep(const double* __restrict__ in, Mat&& M, Sink&& sink) {
  constexpr int lines = BEFORE * AFTER;
  const int lane = threadIdx.x & 31;
  for (int l = lane; l < lines; l += 32) {
    const int a = l % AFTER, b = l / AFTER;
    const double* src = in + b * KIN * AFTER + a;
    double x[KIN];
#pragma unroll
    for (int k = 0; k < KIN; k++) x[k] = src[k * AFTER];
#pragma unroll
    for (int m = 0; m < KOUT; m++) {
      double acc = 0.0;
#pragma unroll
      for (int k = 0; k < KIN; k++) acc = fma(x[k], M(k, m), acc);
      sink((b * KOUT + m) * AFTER + a, acc);
    }
  }
}

// Shared-memory plan of the min / max kernel: one warp per observable, WPC warps per CTA, each with
// its own DG block and two sweep intermediates.
template <int N, int DIM, int D>
struct LimMinMaxShape {
  static constexpr int n = N + 1, P = 2 * N + 1;
  static constexpr int nb = DIM == 3 ? n * n * n : n * n;
  static constexpr int m1 = DIM == 3 ? n * n * P : n * P;
  static constexpr int m2 = DIM == 3 ? n * P * P : 1;
  static constexpr int per_warp = nb + m1 + m2;
  // warps per CTA: one per observable up to 8, as many as fit one CTA's shared memory next to the
  // cell's DG block (staged once with contiguous loads for all warps)
  static constexpr int fitw = (int)((220 * 1024 - 8 * nb * D) / (8 * per_warp));
  static constexpr int WPC = (D < 8 ? D : 8) < fitw ? (D < 8 ? D : 8) : (fitw < 1 ? 1 : fitw);
  static constexpr int smem_words = nb * D + WPC * per_warp;
  static constexpr size_t smem = sizeof(double) * (size_t)smem_words;
  // resident CTAs the register budget is sized for (shared memory permitting)
  static constexpr int MinBlocks = 3 * (8 * smem_words + 2048) <= 220 * 1024 ? 3
                                   : (2 * (8 * smem_words + 2048) <= 220 * 1024 ? 2 : 1);
};

// Limiter ops 2 (findCellLocalMinAndMax), 3 (findCellLocalLimiterMinAndMax) and 4
// (discreteMaximumPrincipleAndMinAndMaxSearch): one cell per CTA, warp w on observables w, w + WPC,
// ...; each warp projects its observable onto the Gauss-Lobatto nodes and the subcell means with
// warp-synchronous sweeps, reduces its extrema by shuffles, and thread 0 applies the principle.
template <int N, int DIM, int D>
__global__ void __launch_bounds__(32 * LimMinMaxShape<N, DIM, D>::WPC, LimMinMaxShape<N, DIM, D>::MinBlocks)
limiter_minmax_kernel(LimArgs a) {
  using A = AmrT<N>;
  using Sh = LimMinMaxShape<N, DIM, D>;
  constexpr int n = Sh::n, P = Sh::P, nb = Sh::nb, WPC = Sh::WPC;
  extern __shared__ __align__(16) double sm[];
  __shared__ double s_lmin[32], s_lmax[32];
  const int c = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* blk = sm;                                          // [nb][D] the cell's DG block
  double* U = sm + (size_t)nb * D + (size_t)warp * Sh::per_warp;  // [nb]
  double* M1 = U + nb;
  double* M2 = M1 + Sh::m1;
  const int g = a.ghost;
  const int E = P + 2 * g;
  const size_t ext = DIM == 3 ? (size_t)E * E * E : (size_t)E * E;
  auto d2f = [](int k, int m) { return A::dg2fv(k, m); };
  auto l2b = [](int k, int i) { return A::leg2lob(k, i); };
  if (a.op == 4 && threadIdx.x == 0) a.ok[c] = 1;
  if (a.op != 3) {
    const double* src = a.luh + (size_t)c * nb * D;
    for (int e = threadIdx.x; e < nb * D; e += blockDim.x) blk[e] = src[e];
    __syncthreads();
  }
  for (int v = warp; v < a.nobs; v += WPC) {
    double lo = INFINITY, hi = -INFINITY;
    auto take = [&](int, double x) {
      lo = fmin(lo, x);
      hi = fmax(hi, x);
    };
    if (a.op == 3) {
      // the interior subcells of the patch
      const double* lim = a.lim + (size_t)c * ext * D + v;
      constexpr int pb = DIM == 3 ? P * P * P : P * P;
      for (int s = lane; s < pb; s += 32) {
        const int x = s % P, y = (s / P) % P, z = DIM == 3 ? s / (P * P) : 0;
        const size_t at = DIM == 3 ? ((size_t)(z + g) * E + (y + g)) * E + (x + g) : (size_t)(y + g) * E + (x + g);
        take(0, lim[at * D]);
      }
    } else {
      for (int p = lane; p < nb; p += 32) {
        U[p] = blk[p * D + v];
        take(0, U[p]);
      }
      __syncwarp();
      if constexpr (DIM == 3) {
        warp_sweep<n * n, n, n, 1>(U, l2b, [&](int o, double x) { M1[o] = x; });
        __syncwarp();
        warp_sweep<n, n, n, n>(M1, l2b, [&](int o, double x) { M2[o] = x; });
        __syncwarp();
        warp_sweep<1, n, n, n * n>(M2, l2b, take);
        __syncwarp();
        warp_sweep<n * n, n, P, 1>(U, d2f, [&](int o, double x) { M1[o] = x; });
        __syncwarp();
        warp_sweep<n, n, P, P>(M1, d2f, [&](int o, double x) { M2[o] = x; });
        __syncwarp();
        warp_sweep<1, n, P, P * P>(M2, d2f, take);
      } else {
        warp_sweep<n, n, n, 1>(U, l2b, [&](int o, double x) { M1[o] = x; });
        __syncwarp();
        warp_sweep<1, n, n, n>(M1, l2b, take);
        __syncwarp();
        warp_sweep<n, n, P, 1>(U, d2f, [&](int o, double x) { M1[o] = x; });
        __syncwarp();
        warp_sweep<1, n, P, P>(M1, d2f, take);
      }
      __syncwarp();
    }
    // fmin / fmax skip a NaN value, as the reference's std::min(acc, x) / std::max(acc, x) do
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
      if (a.op == 4) {
        s_lmin[v & 31] = lo;  // nobs <= 32
        s_lmax[v & 31] = hi;
      } else {
        a.mn[(size_t)c * a.nobs + v] = lo;
        a.mx[(size_t)c * a.nobs + v] = hi;
      }
    }
  }
  if (a.op != 4) return;
  __syncthreads();
  // limiter/generic/c/Limiter.cpph discreteMaximumPrincipleAndMinAndMaxSearch, observable v
  for (int v = threadIdx.x; v < a.nobs; v += blockDim.x) {
    double* bmn = a.mn + (size_t)c * 2 * DIM * a.nobs;
    double* bmx = a.mx + (size_t)c * 2 * DIM * a.nobs;
    const double lmin = s_lmin[v], lmax = s_lmax[v];
    double bmin = bmn[v], bmax = bmx[v];
#pragma unroll
    for (int f = 1; f < 2 * DIM; f++) {
      bmin = fmin(bmin, bmn[f * a.nobs + v]);
      bmax = fmax(bmax, bmx[f * a.nobs + v]);
    }
    double sd = (bmax - bmin) * a.scale;
    sd = fmax(sd, a.relax);
    bool ok = !((lmin < bmin - sd) || (lmax > bmax + sd));
    ok = ok && isfinite(lmin) && isfinite(lmax);
    if (!ok) a.ok[c] = 0;
    bmn[v] = lmin;
    bmx[v] = lmax;
    bmn[a.nobs + v] = bmin;
    bmx[a.nobs + v] = bmax;
  }
}

}  // namespace exa
