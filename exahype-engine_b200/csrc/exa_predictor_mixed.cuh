// Mixed-precision space-time predictor (EXA_PREC_MIXED, PDEs without NCP).
//
// Same algorithm, work decomposition and outputs as predictor_kernel (exa_predictor.cuh), with the
// Picard sweeps after sweep 0 written as corrections to sweep 0:
//
//   sweep 0 (FP64, as in the FP64 kernel): the iterate is luh at every time node, so its flux F(luh)
//   is contracted once (o = sum_d of the scaled Kxi contractions) and its time solve has the closed
//   form q1[t] = luh A[t] - o B[t] / w_p (+ source terms).
//
//   sweep s >= 1: the flux of the old iterate splits as F(q) = F(luh) + dF, and F(luh)'s part of the
//   rhs is the one sweep 0 already solved, so exactly (reference 3d/spaceTimePredictorNonlinear.cpph
//   :231-405, rearranged)
//       q_new[t] = q1[t] + delta[t],   delta[t] = -(1/w_p) sum_i iK1[t][i] c_i,
//   where c_i is the scaled Kxi contraction of dF at time node i. The old iterate is kept as its
//   FP32 difference to q1, dq = q_old - q1 (the previous sweep's delta; zero after sweep 0), which
//   is far smaller than q_old - luh, so its rounding stays well below the residual tolerance.
//   dF = F(q1 + dq) - F(luh) is formed in FP64 and rounded to FP32; its contraction, c_i and the
//   delta accumulation run in FP32; q1, the iterates q1 + dq and q1 + delta, the residual test
//   |q_new - q_old|^2 = |delta - dq|^2 < 1e-14, the time averages, the face extrapolation and the
//   volume integral stay FP64.
//
// The FP32 corrections are small against the state (dF ~ dt * dF/dt), so their rounding error is
// far below the FP64 path's discretisation error, and the Picard fixed point, which recomputes dF
// from the FP64 iterate every sweep, does not accumulate it (iterative refinement).
//
// Shared memory per cell is about half the FP64 kernel's (FP32 slices and flux blocks), so more
// cells are resident per SM; OCC is the targeted number of CTAs per SM (its register budget), and
// the launcher measures which OCC is faster per instantiation.
#pragma once

namespace exa {

template <class PDE, int DIM, int N, int P>
struct MixShape {
  using S = Shape<PDE, DIM, N, P>;
  static constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, CPB = S::CPB, TPB = S::TPB, NL = S::NL;
  static constexpr int DQ = S::DQ;
  static constexpr int VQ = V | 1;  // odd float stride of a node in the dq slices
  static constexpr int VO = V | 1;  // odd double stride of a node in o_s
  // float flux blocks: an x line is padded by one word, a 3D y-z plane by PY words, so that both
  // access patterns (thread per node, thread per line) spread over the 32 banks
  static constexpr int PY = ((n - n * n) % 32 + 32) % 32;
  static __host__ __device__ constexpr int foff(int d, int p) {
    return d == 0 ? p + p / n : ((DIM == 3 && d == 1) ? p + (p / (n * n)) * PY : p);
  }
  static constexpr int fmax_off() {
    int m = 0;
    for (int d = 0; d < DIM; d++) m = foff(d, nd - 1) + 1 > m ? foff(d, nd - 1) + 1 : m;
    return m;
  }
  static constexpr int BSF = fmax_off() | 1;                          // one (cell, dir, var) block
  static constexpr int FCSF = DIM * V * BSF + ((DIM * V * BSF) % 2 == 0 ? 1 : 0);
  static constexpr int dq_floats = CPB * n * nd * VQ;
  static constexpr int f32_floats = CPB * FCSF;
  // region R holds either the FP32 sweep state (dq slices + FP32 flux blocks) or the FP64 flux
  // blocks + lQhi of sweep 0 and the tail
  static constexpr int r_sweep = (dq_floats + f32_floats + 1) / 2;
  static constexpr int r_fp64 = CPB * S::FCS + CPB * nd * DQ;
  static constexpr int even(int x) { return (x + 1) / 2 * 2; }
  static constexpr int regionR = even(r_sweep > r_fp64 ? r_sweep : r_fp64);
  static constexpr int smemU = CPB * nd * DQ;
  static constexpr int smemO = even(CPB * nd * VO);
  static constexpr size_t smem_for(int) { return sizeof(double) * (size_t)(regionR + smemU + smemO); }
  static constexpr int items = S::items, rounds = S::rounds;
  // registers per thread for occ resident CTAs: the SM's four 16K-register partitions hold
  // ceil(occ * warps / 4) warps each
  static constexpr int regs(int occ) {
    return (512 / ((occ * (TPB / 32) + 3) / 4)) / 8 * 8 > 255 ? 255 : (512 / ((occ * (TPB / 32) + 3) / 4)) / 8 * 8;
  }
};

template <class PDE, int DIM, int N, int P, int OCC>
__global__ void __launch_bounds__((Shape<PDE, DIM, N, P>::TPB)) __maxnreg__((MixShape<PDE, DIM, N, P>::regs(OCC)))
predictor_mixed_kernel(CellArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using M = MixShape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf, NL = S::NL, CPB = S::CPB, BS = S::BS;
  constexpr int DQ = S::DQ, FCS = S::FCS, VQ = M::VQ, VO = M::VO, BSF = M::BSF, FCSF = M::FCSF;
  static_assert(!PDE::kNCP, "the mixed-precision sweeps are built for PDEs without NCP");
  static_assert(CPB <= 32, "the per-CTA cell mask holds 32 cells");
  extern __shared__ __align__(128) double smem[];
  // sweeps >= 1: dq [CPB][n][nd][VQ] floats, then the FP32 flux blocks [CPB][FCSF]
  float* dqs = reinterpret_cast<float*>(smem);
  float* sF32 = dqs + M::dq_floats;
  // sweep 0 and the tail: FP64 flux blocks [CPB][FCS], then lQhi [CPB][nd][DQ]
  double* sF = smem;
  double* sQh = smem + CPB * FCS;
  double* sU = smem + M::regionR;        // luh [CPB][nd][DQ]
  double* sO = sU + M::smemU;            // o [CPB][nd][VO]
  __shared__ double s_A[n], s_B[n];
  __shared__ double s_w[n], s_Kxi[n * n];
  __shared__ double s_lw[CPB * DIM * NL];
  __shared__ double s_dt[CPB], s_invdx[CPB][3];
  __shared__ unsigned long long s_res[2][CPB];  // per-cell residual (residual_units), by sweep parity

  const int tid = threadIdx.x;
  const bool inr = tid < CPB * nd;
  const int lc = inr ? tid / nd : 0;
  const int p = inr ? tid % nd : 0;
  const int cell0 = a.cell_begin + (int)blockIdx.x * CPB;
  const int cell = cell0 + lc;
  const bool live = inr && cell < a.ncells;
  unsigned active = 0;
#pragma unroll
  for (int c = 0; c < CPB; c++) active |= (cell0 + c < a.ncells ? 1u : 0u) << c;

  if (tid < n) {
    s_w[tid] = G::weights(tid);
    double A = 0.0, B = 0.0;
#pragma unroll
    for (int i = 0; i < n; i++) {
      A = fma(G::iK1(tid, i), G::F0(i), A);
      B = fma(G::iK1(tid, i), G::weights(i), B);
    }
    s_A[tid] = A;
    s_B[tid] = B;
  }
  if (tid < n * n) s_Kxi[tid] = G::Kxi(tid / n, tid % n);
  if (tid < CPB) {
    const int c = cell0 + tid;
    const int g = (c < a.ncells && a.cell_grid) ? a.cell_grid[c] : 0;
    s_dt[tid] = a.grid_dt ? a.grid_dt[g] : a.u_dt;
#pragma unroll
    for (int d = 0; d < 3; d++)
      s_invdx[tid][d] = d < DIM ? 1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 0.0;
    s_res[0][tid] = 0;
    s_res[1][tid] = 0;
  }
  double* u = sU + ((size_t)lc * nd + p) * DQ;
  if (inr) {
    const double* luh = a.luh + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
    for (int m = 0; m < D; m++) u[m] = live ? luh[m] : 1.0;
  }
  __syncthreads();
  for (int j = tid; j < CPB * DIM * NL; j += S::TPB) {
    const int c = j / (DIM * NL), d = (j / NL) % DIM, L = j % NL;
    const double wt = DIM == 3 ? s_w[L / n] * s_w[L % n] : s_w[L];
    s_lw[j] = wt * s_dt[c] * s_invdx[c][d];
  }

  int co[3];
  node_coords<DIM, n>(p, co);
  const double w_sp = DIM == 3 ? s_w[co[2]] * s_w[co[1]] * s_w[co[0]] : s_w[co[1]] * s_w[co[0]];
  const double iweight = 1.0 / w_sp;
  const double dt = s_dt[lc];
  float* dq = dqs + (size_t)lc * n * nd * VQ;
  double* f_s = sF + (size_t)lc * FCS;
  float* f32 = sF32 + (size_t)lc * FCSF;

  // point source (algebraicSource at x_p, t + node_i dt): only cells near the source
  bool srcOn = false;
  double tcell = 0.0;
  if (PDE::kSource && a.src && live) {
    const int g = a.cell_grid ? a.cell_grid[cell] : 0;
    const double dxv[3] = {1.0 / s_invdx[lc][0], DIM > 1 ? 1.0 / s_invdx[lc][1] : 1.0,
                           DIM > 2 ? 1.0 / s_invdx[lc][2] : 1.0};
    double cc[3];
    cell_centre(a, cell, g, dxv, cc);
    srcOn = source_near<DIM>(a.src, cc, dxv);
    tcell = a.grid_t ? a.grid_t[g] : a.u_t;
  }
  auto src_at = [&](int i) -> double {
    const int g = a.cell_grid ? a.cell_grid[cell] : 0;
    const double dxv[3] = {1.0 / s_invdx[lc][0], DIM > 1 ? 1.0 / s_invdx[lc][1] : 1.0,
                           DIM > 2 ? 1.0 / s_invdx[lc][2] : 1.0};
    double cc[3], x[3];
    cell_centre(a, cell, g, dxv, cc);
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = cc[d] + dxv[d] * (G::nodes(co[d]) - 0.5);
    return point_source<DIM>(a.src, x, tcell + G::nodes(i) * s_dt[lc]);
  };
  const int srcVar = (PDE::kSource && a.src) ? (int)a.src[7] : -1;
  // the source part of sweep 0's closed form: dt sum_i iK1[t][i] w_i src_i (source cells only)
  double cs[PDE::kSource ? n : 1];
#pragma unroll
  for (int t = 0; t < (PDE::kSource ? n : 1); t++) cs[t] = 0.0;
  if (PDE::kSource && srcOn) {
    for (int i = 0; i < n; i++) {
      const double wsi = G::weights(i) * dt * src_at(i);
#pragma unroll
      for (int t = 0; t < (PDE::kSource ? n : 1); t++) cs[t] = fma(G::iK1(t, i), wsi, cs[t]);
    }
  }
  // o: sweep 0's contraction of F(luh), summed over the directions (this node, per variable)
  double* o_s = sO + ((size_t)lc * nd + p) * VO;
  // sweep 0's closed-form iterate q1[t][m] (the same expression as the FP64 kernel's sweep 0)
  auto q1 = [&](int t, int m) -> double {
    double v = u[m] * s_A[t] - iweight * o_s[m] * s_B[t];
    if (PDE::kSource && srcOn && m == srcVar) v += cs[PDE::kSource ? t : 0];
    return v;
  };

  __syncthreads();  // s_lw

  // FP64 contraction of sweep 0, in place on the FP64 flux blocks (the FP64 kernel's phase 2)
  auto contract64 = [&]() {
#pragma unroll
    for (int r = 0; r < S::rounds; r++) {
      const int it = tid + r * S::TPB;
      if (it >= S::items) continue;
      const int L = it % NL, m = (it / NL) % V, d = (it / (NL * V)) % DIM, c = it / (NL * V * DIM);
      double* f = sF + c * FCS + (d * V + m) * BS + flux_off<DIM, n>(d, line_base<DIM, n>(d, L));
      const int st = d == 0 ? 1 : (d == 1 ? n : n * n);
      const double coef = s_lw[(c * DIM + d) * NL + L];
      double x[n], acc[n];
#pragma unroll
      for (int k = 0; k < n; k++) x[k] = f[k * st];
#pragma unroll
      for (int l = 0; l < n; l++) acc[l] = 0.0;
#pragma unroll
      for (int k = 0; k < n; k++)
#pragma unroll
        for (int l = 0; l < n; l++) acc[l] = fma(x[k], G::Kxi(k, l), acc[l]);
#pragma unroll
      for (int l = 0; l < n; l++) f[l * st] = coef * acc[l];
    }
  };
  // FP32 contraction of the flux corrections at time node i, in place, scaled by w_i w_a w_b dt/dx_d
  auto contract32 = [&](float wi) {
#pragma unroll
    for (int r = 0; r < S::rounds; r++) {
      const int it = tid + r * S::TPB;
      if (it >= S::items) continue;
      const int L = it % NL, m = (it / NL) % V, d = (it / (NL * V)) % DIM, c = it / (NL * V * DIM);
      float* f = sF32 + c * FCSF + (d * V + m) * BSF + M::foff(d, line_base<DIM, n>(d, L));
      const int st = d == 0 ? 1 : (d == 1 ? n : n * n);
      const float coef = wi * (float)s_lw[(c * DIM + d) * NL + L];
      float x[n];
#pragma unroll
      for (int k = 0; k < n; k++) x[k] = f[k * st];
#pragma unroll
      for (int l = 0; l < n; l++) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k < n; k++) acc = fmaf(x[k], G::Kxif(k, l), acc);
        f[l * st] = coef * acc;
      }
    }
  };

  const int maxIter = a.max_picard > 0 ? a.max_picard : S::maxSweeps;
  float delta[n][V];  // correction of the new iterate to q1, accumulated over the time nodes
#pragma unroll
  for (int t = 0; t < n; t++)
#pragma unroll
    for (int m = 0; m < V; m++) delta[t][m] = 0.0f;
  int sweeps = 0;
  bool done = false;
  bool last_old_is_luh = true;
  for (int s = 0; s < maxIter; s++) {
    const bool work = live && ((active >> lc) & 1u);
    double res = 0.0;
    if (s == 0) {
      double F[DIM * V];
      PDE::template flux<DIM>(u, F);
      if (inr) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) f_s[(d * V + m) * BS + flux_off<DIM, n>(d, p)] = F[d * V + m];
      }
      __syncthreads();
      contract64();
      __syncthreads();
      if (work) {
#pragma unroll
        for (int m = 0; m < V; m++) {
          double acc = f_s[(0 * V + m) * BS + flux_off<DIM, n>(0, p)];
#pragma unroll
          for (int d = 1; d < DIM; d++) acc += f_s[(d * V + m) * BS + flux_off<DIM, n>(d, p)];
          o_s[m] = acc;
        }
#pragma unroll
        for (int m = 0; m < V; m++)
#pragma unroll
          for (int t = 0; t < n; t++) {
            const double dl = q1(t, m) - u[m];
            res = fma(dl, dl, res);
          }
      }
    } else {
      if (work) {
#pragma unroll
        for (int t = 0; t < n; t++)
#pragma unroll
          for (int m = 0; m < V; m++) delta[t][m] = 0.0f;
      }
      const float iwf = (float)iweight;
#pragma unroll
      for (int i = 0; i < n; i++) {
        // phase 1: dF = F(q1_i + dq_i) - F(luh) in FP64, stored as FP32
        if (inr) {
          double q[D];
#pragma unroll
          for (int m = 0; m < D; m++) q[m] = m < V ? q1(i, m) + (double)dq[(i * nd + p) * VQ + m] : u[m];
          double F[DIM * V];
          PDE::template flux<DIM>(q, F);
          double Fu[DIM * V];
          PDE::template flux<DIM>(u, Fu);
#pragma unroll
          for (int d = 0; d < DIM; d++)
#pragma unroll
            for (int m = 0; m < V; m++) f32[(d * V + m) * BSF + M::foff(d, p)] = (float)(F[d * V + m] - Fu[d * V + m]);
        }
        __syncthreads();
        contract32((float)G::weights(i));
        __syncthreads();
        // phase 3: delta[t] -= (1/w_p) iK1[t][i] c_i
        if (work) {
#pragma unroll
          for (int m = 0; m < V; m++) {
            float c = f32[(0 * V + m) * BSF + M::foff(0, p)];
#pragma unroll
            for (int d = 1; d < DIM; d++) c += f32[(d * V + m) * BSF + M::foff(d, p)];
            const float r = -iwf * c;
#pragma unroll
            for (int t = 0; t < n; t++) delta[t][m] = fmaf(r, G::iK1f(t, i), delta[t][m]);
          }
        }
      }
      if (work) {
        // q_new - q_old = (q1 + delta) - (q1 + dq) = delta - dq
#pragma unroll
        for (int t = 0; t < n; t++)
#pragma unroll
          for (int m = 0; m < V; m++) {
            const double dl = (double)delta[t][m] - (double)dq[(t * nd + p) * VQ + m];
            res = fma(dl, dl, res);
          }
      }
    }
    {
      const int lane = tid & 31;
      const int seg_end = (lc + 1) * nd - 1;
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) {
        const double v = __shfl_down_sync(0xffffffffu, res, o2);
        if (lane + o2 < 32 && tid + o2 <= seg_end) res += v;
      }
      if ((p == 0 || lane == 0) && work) {
          atomicAdd(&s_res[s & 1][lc], residual_units(res));
          if (!finite(res) && a.status) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
        }
    }
    __syncthreads();
    unsigned conv = 0;
    if (a.max_picard <= 0) {
#pragma unroll
      for (int c = 0; c < CPB; c++) conv |= ((double)s_res[s & 1][c] < kResidualTolUnits ? 1u : 0u) << c;
    }
    conv &= active;
    if (work) {
      sweeps = s + 1;
      done = (conv >> lc) & 1u;
      if (!done && s + 1 < maxIter) {
        // the new iterate becomes the old one: dq = delta (sweep 0's FP64 flux blocks, which alias
        // these slices, were last read before the barrier above)
#pragma unroll
        for (int t = 0; t < n; t++)
#pragma unroll
          for (int m = 0; m < V; m++) dq[(t * nd + p) * VQ + m] = delta[t][m];
      } else {
        last_old_is_luh = s == 0;
      }
    }
    if (tid < CPB) s_res[(s + 1) & 1][tid] = 0;
    active &= ~conv;
    if (!active) break;
  }
  if (live && a.picard && p == 0) a.picard[cell] = sweeps;
  if (live && p == 0 && a.max_picard <= 0 && !done && a.status) atomicOr(a.status, ST_PICARD_CAP);

  // ---------------- time averaging, FP64 ----------------
  double qh[D];
#pragma unroll
  for (int m = 0; m < D; m++) {
    double acc = 0.0;
#pragma unroll
    for (int t = 0; t < n; t++) acc = fma(m < V ? q1(t, m) + (double)delta[t][m] : u[m], G::weights(t), acc);
    qh[m] = acc;
  }
  if (live && a.ex_lQi) {
    double* e = a.ex_lQi + (size_t)cell * nd * n * D + (size_t)p * n * D;
#pragma unroll
    for (int t = 0; t < n; t++)
#pragma unroll
      for (int m = 0; m < D; m++) e[t * D + m] = m < V ? q1(t, m) + (double)delta[t][m] : u[m];
  }
  // lFhi = sum_i w_i F(old iterate of the last sweep at i)
  double fa[DIM * V];
#pragma unroll
  for (int k = 0; k < DIM * V; k++) fa[k] = 0.0;
  if (inr) {
    if (last_old_is_luh) {
      double F[DIM * V];
      PDE::template flux<DIM>(u, F);
#pragma unroll
      for (int i = 0; i < n; i++) {
        const double wi = G::weights(i);
#pragma unroll
        for (int k = 0; k < DIM * V; k++) fa[k] = fma(F[k], wi, fa[k]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < n; i++) {
        double q[D], F[DIM * V];
#pragma unroll
        for (int m = 0; m < D; m++) q[m] = m < V ? q1(i, m) + (double)dq[(i * nd + p) * VQ + m] : u[m];
        PDE::template flux<DIM>(q, F);
        const double wi = G::weights(i);
#pragma unroll
        for (int k = 0; k < DIM * V; k++) fa[k] = fma(F[k], wi, fa[k]);
      }
    }
  }
  __syncthreads();  // every dq read is done: region R takes the FP64 tail staging
  double* qh_s = sQh + (size_t)lc * nd * DQ;
  if (inr) {
#pragma unroll
    for (int m = 0; m < D; m++) qh_s[p * DQ + m] = qh[m];
#pragma unroll
    for (int d = 0; d < DIM; d++)
#pragma unroll
      for (int m = 0; m < V; m++) f_s[(d * V + m) * BS + flux_off<DIM, n>(d, p)] = fa[d * V + m];
  }
  if (live && a.ex_lQhi) {
    for (int m = 0; m < D; m++) a.ex_lQhi[(size_t)cell * nd * D + p * D + m] = qh[m];
  }
  if (live && a.ex_lFhi) {
    double* e = a.ex_lFhi + (size_t)cell * (DIM + 1) * nd * V;
    for (int d = 0; d < DIM; d++) {
      const int idx = node_line<DIM, n>(p, d) * n + co[d];
      for (int m = 0; m < V; m++) e[(size_t)d * nd * V + idx * V + m] = fa[d * V + m];
    }
    for (int m = 0; m < V; m++) e[(size_t)DIM * nd * V + p * V + m] = 0.0;
  }
  __syncthreads();

  // ---------------- volume integral, FP64 ----------------
  if (live) {
    double* lduh = a.lduh + (size_t)cell * nd * V + (size_t)p * V;
    double acc[V];
#pragma unroll
    for (int m = 0; m < V; m++) acc[m] = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int L = node_line<DIM, n>(p, d);
      const int base = flux_off<DIM, n>(d, line_base<DIM, n>(d, L)), st = d == 0 ? 1 : (d == 1 ? n : n * n);
      const double wt = DIM == 3 ? s_w[L / n] * s_w[L % n] : s_w[L];
      const double us = wt * s_invdx[lc][d];
      double kr[n];
#pragma unroll
      for (int mm = 0; mm < n; mm++) kr[mm] = s_Kxi[co[d] * n + mm];
#pragma unroll
      for (int m = 0; m < V; m++)
#pragma unroll
        for (int mm = 0; mm < n; mm++) acc[m] += kr[mm] * f_s[(d * V + m) * BS + base + mm * st] * us;
    }
    if (PDE::kSource && srcOn) {
      double sa = 0.0;
      for (int i = 0; i < n; i++) sa = fma(src_at(i), G::weights(i), sa);
#pragma unroll
      for (int m = 0; m < V; m++)
        if (m == srcVar) acc[m] += w_sp * sa;
    }
    bool ok = true;
#pragma unroll
    for (int m = 0; m < V; m++) {
      lduh[m] = acc[m];
      ok &= finite(acc[m]);
    }
    if (!ok && a.status) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
  }

  // ---------------- extrapolation to the faces, FP64 ----------------
  constexpr int LQ = DIM * NL;
  for (int j = tid; j < CPB * 2 * LQ; j += S::TPB) {
    const int c = j / (2 * LQ);
    const int gc = cell0 + c;
    if (gc >= a.ncells) continue;
    const int r = j % (2 * LQ);
    const bool isQ = r < LQ;
    const int rl = isQ ? r : r - LQ;
    const int d = rl / NL, L = rl % NL;
    const int st = d == 0 ? 1 : (d == 1 ? n : n * n);
    if (isQ) {
      const double* src = sQh + (size_t)c * nd * DQ + (size_t)line_base<DIM, n>(d, L) * DQ;
      double* o0 = a.lQhbnd + (size_t)gc * S::sizeQhb + (size_t)((2 * d) * nf + L) * D;
      double* o1 = a.lQhbnd + (size_t)gc * S::sizeQhb + (size_t)((2 * d + 1) * nf + L) * D;
#pragma unroll
      for (int m = 0; m < D; m++) {
        double a0 = 0.0, a1 = 0.0;
        if (!(DIM == 2 && d == 0 && m >= V)) {
#pragma unroll
          for (int l = 0; l < n; l++) {
            const double x = src[(size_t)l * st * DQ + m];
            a0 = fma(x, G::F0(l), a0);
            a1 = fma(x, G::F1(l), a1);
          }
        }
        o0[m] = a0;
        o1[m] = a1;
      }
    } else {
      const double* src = sF + (size_t)c * FCS + (size_t)d * V * BS + flux_off<DIM, n>(d, line_base<DIM, n>(d, L));
      double* o0 = a.lFhbnd + (size_t)gc * S::sizeFhb + (size_t)((2 * d) * nf + L) * V;
      double* o1 = a.lFhbnd + (size_t)gc * S::sizeFhb + (size_t)((2 * d + 1) * nf + L) * V;
#pragma unroll
      for (int m = 0; m < V; m++) {
        double a0 = 0.0, a1 = 0.0;
#pragma unroll
        for (int l = 0; l < n; l++) {
          const double x = src[(size_t)m * BS + l * st];
          a0 = fma(x, G::F0(l), a0);
          a1 = fma(x, G::F1(l), a1);
        }
        o0[m] = a0;
        o1[m] = a1;
      }
    }
  }
}

}  // namespace exa
