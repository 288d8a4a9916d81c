// Fused space-time predictor + time averaging + face extrapolation + volume integral.
//
// Reference: ExaHyPE/kernels/aderdg/generic/c/3d/spaceTimePredictorNonlinear.cpph
//   aderPicardLoopNonlinear :39-433, aderPredictorNonlinear :441-515,
//   aderExtrapolatorNonlinear :517-687, entry :816-864 (2D: 2d/spaceTimePredictorNonlinear.cpph),
// and 3d/volumeIntegralNonlinear.cpph:133-223 (time-averaged branch), as the generated glue
// calls them in fusedSpaceTimePredictorVolumeIntegral (AbstractGenericADERDGSolverImplementation
// .template:168-211).
//
// Work decomposition: one CTA per cell (several cells per CTA when a cell has fewer than 256
// nodes), one thread per spatial node. A Picard sweep walks the n time nodes; per time node
//   phase 1  each thread evaluates the flux (and the source, algebraicSource - NCP) of the old
//            iterate at its node and writes it to shared memory,
//   phase 2  every thread contracts whole lines (direction, variable, line) with Kxi, in place
//            and already scaled by w_t w_a w_b dt/dx_d,
//   phase 3  each thread forms its node's rhs of time node i, scaled by 1/w_xyz, and folds it
//            into the new iterate at every time node t through iK1[t][i] (the iK1 time solve
//            distributed over the time nodes).
// The new iterate lives in registers (n*V doubles per thread); the old iterate stays in the
// shared slices [t][node][D] for the whole sweep (phase 1 and the residual read only the
// thread's own node; the gradients of an NCP or of a viscous flux read neighbours) and is
// overwritten by the new one once the per-cell residual has decided that another sweep follows.
// A viscous flux (useViscousFlux) is evaluated from the node's state and the gradient of the old
// iterate at the same time node (:99-212).
//
// Sweep 0 starts from lQi[., t] = luh (:71-82), which is constant in time, so its flux and
// contractions are computed once and its time solve has a closed form (an exact identity, not
// an approximation). For PDEs with neither an NCP nor a viscous flux the time-averaged flux lFhi
// is accumulated in registers from the final old iterate after the loop instead of being carried
// through every sweep.
#pragma once

namespace exa {

template <int DIM, int n>
__device__ __forceinline__ int pline_base(int d, int L) {
  // start of line L of direction d inside a padded (dir, var) block; its nodes follow with the
  // unpadded stride (1, n, n^2), because the padding groups hold whole lines
  return flux_off<DIM, n>(d, line_base<DIM, n>(d, L));
}
template <int DIM, int n>
__device__ __forceinline__ int pnode_off(int d, int p) {
  // offset of node p inside a padded (dir, var) block
  return flux_off<DIM, n>(d, p);
}

// PERSIST: a persistent grid whose CTAs walk groups blockIdx.x, blockIdx.x + gridDim.x, ... and
// fetch the next group's luh by bulk copy while computing the current one; otherwise one group per
// CTA (shorter register live ranges). The launcher picks the faster form per instantiation.
template <class PDE, int DIM, int N, int P, bool PERSIST>
__global__ void __launch_bounds__((Shape<PDE, DIM, N, P>::TPB)) __maxnreg__((Shape<PDE, DIM, N, P>::MaxRegs))
predictor_kernel(CellArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf, NL = S::NL, CPB = S::CPB, BS = S::BS;
  constexpr int DQ = S::DQ;  // per-node stride of the iterate slices and the luh block (odd)
  constexpr int FCS = S::FCS;  // stride between the cells' flux blocks
  constexpr bool NCP = PDE::kNCP;
  constexpr bool VISC = is_viscous<PDE>::value;  // viscousFlux(Q, gradQ) replaces flux(Q)
  constexpr bool GRAD = NCP || VISC;               // the sweeps need the iterate's gradient
  // the time-averaged flux is accumulated during the sweeps only where the flux needs the gradient;
  // otherwise the tail recomputes it from the last old iterate (fewer registers in the sweeps)
  constexpr bool FHACC = VISC;
  constexpr bool ALG = has_algebraic_source<PDE, DIM>::value;  // algebraicSource (useSource)
  constexpr bool SRCT = NCP || ALG;                // a source slot S = algebraicSource - NCP
  static_assert(CPB <= 32, "the per-CTA cell mask holds 32 cells");
  extern __shared__ __align__(128) double smem[];
  double* sQ = smem;              // [CPB][n][nd][DQ]: old iterate slices, lQhi in the tail
  double* sF = smem + S::smemQ;   // [CPB][FCS >= DIM*V*BS]: fluxes, contracted in place
  double* stage = smem + S::stage_off();  // [CPB][nd][D]: bulk copy of the next group's luh
  __shared__ double s_w[n], s_Kxi[n * n], s_dudx[n * n];
  __shared__ double s_A[n], s_B[n];  // sum_i iK1[t][i] F0[i] and sum_i iK1[t][i] w_i (sweep 0)
  __shared__ double s_lw[CPB * DIM * NL];  // w_a w_b dt / dx_d of every line
  __shared__ double s_dt[CPB], s_invdx[CPB][3];
  __shared__ unsigned long long s_res[2][CPB];  // per-cell residual (residual_units), by sweep parity
  __shared__ __align__(8) uint64_t s_bar;  // completion of the staging copy

  const int tid = threadIdx.x;
  const bool inr = tid < CPB * nd;   // tail threads of the last warp only help in line loops
  const int lc = inr ? tid / nd : 0;
  const int p = inr ? tid % nd : 0;
  // persistent CTAs: groups of CPB consecutive cells, blockIdx.x, blockIdx.x + gridDim.x, ...
  const int ngroups = (a.ncells - a.cell_begin + CPB - 1) / CPB;

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
  if (tid < n * n) {
    s_Kxi[tid] = G::Kxi(tid / n, tid % n);
    s_dudx[tid] = G::dudx(tid / n, tid % n);
  }
  // the staging copy of a group: live cells only, one bulk copy (thread 0)
  auto issue = [&](int g) {
    const int c0 = a.cell_begin + g * CPB;
    const int nlive = a.ncells - c0 < CPB ? a.ncells - c0 : CPB;
    const uint32_t bytes = (uint32_t)(nlive * nd * D * sizeof(double));
    mbar_arrive_expect_tx(&s_bar, bytes);
    bulk_g2s(stage, a.luh + (size_t)c0 * nd * D, bytes, &s_bar);
  };
  if (PERSIST && tid == 0 && a.bulk_luh) {
    mbar_init(&s_bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (PERSIST && tid == 0 && a.bulk_luh && (int)blockIdx.x < ngroups) issue(blockIdx.x);
  int stall_parity = -1;  // parity of a copy that ran out of time

  const int srcVar = (PDE::kSource && a.src) ? (int)a.src[7] : -1;
  const int maxIter = a.max_picard > 0 ? a.max_picard : S::maxSweeps;

#pragma unroll 1
  for (int iter = 0;; iter++) {
    // this CTA's iter-th group; the staging copy of group iter completes phase iter & 1
    const int grp = blockIdx.x + iter * gridDim.x;
    if (grp >= ngroups || (!PERSIST && iter > 0)) break;
    // per-thread constants, set per group so that they are not live across the whole loop
    int co[3];
    node_coords<DIM, n>(p, co);
    const double w_sp = DIM == 3 ? s_w[co[2]] * s_w[co[1]] * s_w[co[0]] : s_w[co[1]] * s_w[co[0]];
    const double iweight = 1.0 / w_sp;
    int off[DIM];
#pragma unroll
    for (int d = 0; d < DIM; d++) off[d] = pnode_off<DIM, n>(d, p);

    // this thread's line contractions, packed: start offset in sF (bits 0-17), direction
    // (bits 18-19), index of the line weight (bits 20-31); -1 when the thread has none
    static_assert(S::smemF < (1 << 18) && CPB * DIM * NL < (1 << 12), "packed line descriptor overflow");
    int it_pack[S::rounds];
#pragma unroll
    for (int r = 0; r < S::rounds; r++) {
      const int it = tid + r * S::TPB;
      if (it < S::items) {
        const int L = it % NL;
        const int m = (it / NL) % V;
        const int d = (it / (NL * V)) % DIM;
        const int c = it / (NL * V * DIM);
        it_pack[r] = (c * FCS + (d * V + m) * BS + pline_base<DIM, n>(d, L)) | (d << 18) |
                     (((c * DIM + d) * NL + L) << 20);
      } else {
        it_pack[r] = -1;
      }
    }
    // luh of this node, kept in shared memory (read once per phase, not worth 2*D registers);
    // the old iterate starts as lQi[., t] = luh (:71-82)
    double* u = sQ + S::smemQ + S::smemF + ((size_t)lc * nd + p) * DQ;
    double* q_s = sQ + (size_t)lc * S::QCS;
    double* f_s = sF + (size_t)lc * FCS;
    const int cell0 = a.cell_begin + grp * CPB;
    const int cell = cell0 + lc;
    const bool live = inr && cell < a.ncells;
    // cells of the group that exist (identical in every thread)
    unsigned active = 0;
#pragma unroll
    for (int c = 0; c < CPB; c++) active |= (cell0 + c < a.ncells ? 1u : 0u) << c;
    // the previous group's last reads of shared memory (face extrapolation) are done
    __syncthreads();
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
    bool timed_out = false;
    if (PERSIST && a.bulk_luh) timed_out = !mbar_wait_bounded(&s_bar, iter & 1, kBulkWaitLimitNs);
    if (__syncthreads_or(timed_out)) {
      // the copy did not arrive: report, issue nothing more, leave
      if (tid == 0 && a.status) atomicOr(a.status, ST_TIMEOUT);
      stall_parity = iter & 1;
      break;
    }
    if (inr) {
      const double* src = (PERSIST && a.bulk_luh) ? stage + ((size_t)lc * nd + p) * D : a.luh + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
      for (int m = 0; m < D; m++) u[m] = live ? src[m] : 1.0;
    }
    // every thread has its luh row and s_dt / s_invdx are visible: the staging buffer is free
    __syncthreads();
    if (PERSIST && tid == 0 && a.bulk_luh && grp + (int)gridDim.x < ngroups) issue(grp + gridDim.x);
    for (int j = tid; j < CPB * DIM * NL; j += S::TPB) {
      const int c = j / (DIM * NL), d = (j / NL) % DIM, L = j % NL;
      const double wt = DIM == 3 ? s_w[L / n] * s_w[L % n] : s_w[L];
      s_lw[j] = wt * s_dt[c] * s_invdx[c][d];
    }
    const double dt = s_dt[lc];

    // point source (algebraicSource at x_p, t + node_i dt, :323-337): only cells near the source
    // (slot >= 0), whose values source_values_kernel evaluated ahead of this launch. Only patches
    // carry a source, and a patch's source always comes with its slot table.
    const int srcSlot = (PDE::kSource && a.src && a.src_slot && live) ? a.src_slot[cell] : -1;
    const bool srcOn = srcSlot >= 0;
    double tcell = 0.0;
    if (ALG && live) {
      const int g = a.cell_grid ? a.cell_grid[cell] : 0;
      tcell = a.grid_t ? a.grid_t[g] : a.u_t;
    }
    // position of this node: cell centre + dx (node - 0.5), dx as 1 / (1 / dx) (:339-342)
    auto node_x = [&](double* x) {
      const int g = a.cell_grid ? a.cell_grid[cell] : 0;
      const double dxv[3] = {1.0 / s_invdx[lc][0], DIM > 1 ? 1.0 / s_invdx[lc][1] : 1.0,
                             DIM > 2 ? 1.0 / s_invdx[lc][2] : 1.0};
      double cc[3];
      cell_centre(a, cell, g, dxv, cc);
#pragma unroll
      for (int d = 0; d < 3; d++) x[d] = d < DIM ? cc[d] + dxv[d] * (G::nodes(co[d]) - 0.5) : 0.0;
    };
    // S = algebraicSource(x, t + node_i dt, q) - NCP at time node i (:323-367); ncp_part holds -NCP
    auto source_at = [&](int i, const double* q, const double* ncp_part, double* Sv) {
      if constexpr (ALG) {
        double x[3];
        node_x(x);
        PDE::template algebraic_source<DIM>(x, tcell + G::nodes(i) * dt, q, Sv);
      } else {
#pragma unroll
        for (int m = 0; m < V; m++) Sv[m] = 0.0;
      }
      if (NCP) {
#pragma unroll
        for (int m = 0; m < V; m++) Sv[m] = ALG ? Sv[m] + ncp_part[m] : ncp_part[m];
      }
    };
    // source value of this node at time node i (read only where srcOn)
    auto src_at = [&](int i) -> double { return a.src_vals[((size_t)srcSlot * n + i) * nd + p]; };

    // new iterate of the sweep, accumulated in registers time node by time node (the iK1 time
    // solve distributed over phase 3); the old iterate is staged in the slices q_s [t][node][D]
    double qn[n][V];
    if (GRAD && inr) {  // neighbours' old iterate is read by the gradients
#pragma unroll
      for (int t = 0; t < n; t++)
#pragma unroll
        for (int m = 0; m < D; m++) q_s[(t * nd + p) * DQ + m] = u[m];
    }
    double fh[FHACC ? DIM : 1][V];  // time-averaged flux of the sweep (viscous flux only)
    double sh[V];
    (void)fh;
    (void)sh;
    // s_lw and the gradient path's slices are visible
    __syncthreads();

    // gradient of the old iterate at time node ti and this node (:111-175), NCP or viscous flux only
    auto gradient = [&](int ti, double* gq) {
      const double invDx[3] = {s_invdx[lc][0], s_invdx[lc][1], s_invdx[lc][2]};
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int st = d == 0 ? 1 : (d == 1 ? n : n * n);
        const int base = p - co[d] * st;
        const int l = co[d];
#pragma unroll
        for (int m = 0; m < V; m++) {
          double g = 0.0;
#pragma unroll
          for (int k = 0; k < n; k++) g += 1.0 * invDx[d] * q_s[(ti * nd + base + k * st) * DQ + m] * s_dudx[l * n + k];
          gq[d * V + m] = g;
        }
      }
    };
    // phase 2: contraction of every line with Kxi, in place, scaled by wi * w_a w_b dt/dx_d (:248-321)
    auto contract = [&](double wi) {
      // two lines at a time: both lines' loads are issued before either line's math
#pragma unroll
      for (int r = 0; r < S::rounds; r += 2) {
        const int pk0 = it_pack[r];
        const int pk1 = r + 1 < S::rounds ? it_pack[r + 1] : -1;
        if (pk0 < 0) continue;
        double* f0 = sF + (pk0 & 0x3ffff);
        double* f1 = sF + (pk1 < 0 ? (pk0 & 0x3ffff) : (pk1 & 0x3ffff));
        const int d0 = (pk0 >> 18) & 3, d1 = pk1 < 0 ? d0 : ((pk1 >> 18) & 3);
        const int st0 = d0 == 0 ? 1 : (d0 == 1 ? n : n * n);
        const int st1 = d1 == 0 ? 1 : (d1 == 1 ? n : n * n);
        const double c0 = wi * s_lw[(unsigned)pk0 >> 20];
        const double c1 = pk1 < 0 ? 0.0 : wi * s_lw[(unsigned)pk1 >> 20];
        double x0[n], x1[n];
#pragma unroll
        for (int k = 0; k < n; k++) {
          x0[k] = f0[k * st0];
          x1[k] = f1[k * st1];
        }
        // k outermost: 2n independent accumulation chains instead of two (the DFMA latency is
        // hidden inside the warp); each output still sums k = 0..n-1 in order
        double a0[n], a1[n];
#pragma unroll
        for (int l = 0; l < n; l++) a0[l] = a1[l] = 0.0;
#pragma unroll
        for (int k = 0; k < n; k++)
#pragma unroll
          for (int l = 0; l < n; l++) {
            a0[l] = fma(x0[k], G::Kxi(k, l), a0[l]);
            a1[l] = fma(x1[k], G::Kxi(k, l), a1[l]);
          }
#pragma unroll
        for (int l = 0; l < n; l++) {
          f0[l * st0] = c0 * a0[l];
          if (pk1 >= 0) f1[l * st1] = c1 * a1[l];
        }
      }
    };
    auto store_flux = [&](const double* F) {
      if (inr) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) f_s[(d * V + m) * BS + off[d]] = F[d * V + m];
      }
    };
    auto export_flux = [&](int i, const double* F, const double* Sv) {
      double* e = a.ex_lFi + (size_t)cell * n * nd * (DIM + 1) * V + ((size_t)(i * nd + p) * (DIM + 1)) * V;
      for (int d = 0; d < DIM; d++)
        for (int m = 0; m < V; m++) e[d * V + m] = F[d * V + m];
      for (int m = 0; m < V; m++) e[DIM * V + m] = SRCT ? Sv[m] : 0.0;
    };

    int sweeps = 0;
    bool done = false;
    bool last_old_is_luh = true;  // the last sweep started from lQi = luh (sweep 0)
    for (int s = 0; s < maxIter; s++) {
      const bool work = live && ((active >> lc) & 1u);
      if ((FHACC || SRCT) && work) {
#pragma unroll
        for (int d = 0; d < (FHACC ? DIM : 1); d++)
#pragma unroll
          for (int m = 0; m < V; m++) fh[d][m] = 0.0;
#pragma unroll
        for (int m = 0; m < V; m++) sh[m] = 0.0;
      }
      double res = 0.0;
      if (s == 0) {
        // the iterate is luh at every time node: one flux, one set of contractions
        double F[DIM * V];
        double S0[V];
        double gq0[GRAD ? DIM * V : 1];
        if constexpr (GRAD) gradient(0, gq0);
        if constexpr (VISC)
          PDE::template viscous_flux<DIM>(u, gq0, F);
        else
          PDE::template flux<DIM>(u, F);
        store_flux(F);
        if constexpr (NCP) {
          double B[V];
          PDE::template ncp<DIM>(u, gq0, B);
#pragma unroll
          for (int m = 0; m < V; m++) S0[m] = -B[m];
        }
        if ((FHACC || (NCP && !ALG)) && work) {
          for (int i = 0; i < n; i++) {
            const double wi = G::weights(i);
            if (FHACC) {
#pragma unroll
              for (int d = 0; d < (FHACC ? DIM : 1); d++)
#pragma unroll
                for (int m = 0; m < V; m++) fh[d][m] = fma(F[d * V + m], wi, fh[d][m]);
            }
            if (NCP && !ALG) {
#pragma unroll
              for (int m = 0; m < V; m++) sh[m] = fma(S0[m], wi, sh[m]);
            }
          }
        }
        // an algebraic source depends on the time node: lShi, and its part of the closed-form
        // time solve, dt sum_i iK1[t][i] w_i S_i, accumulated in qn
        if (ALG && work) {
#pragma unroll
          for (int t = 0; t < n; t++)
#pragma unroll
            for (int m = 0; m < V; m++) qn[t][m] = 0.0;
          for (int i = 0; i < n; i++) {
            const double wi = G::weights(i);
            double Si[V];
            source_at(i, u, S0, Si);
#pragma unroll
            for (int m = 0; m < V; m++) sh[m] = fma(Si[m], wi, sh[m]);
            const double wdt = wi * dt;
#pragma unroll
            for (int m = 0; m < V; m++)
#pragma unroll
              for (int t = 0; t < n; t++) qn[t][m] = fma(G::iK1(t, i), wdt * Si[m], qn[t][m]);
            if (a.ex_lFi) export_flux(i, F, Si);
          }
        } else if (GRAD && a.ex_lFi && work) {
          for (int i = 0; i < n; i++) export_flux(i, F, S0);
        }
        __syncthreads();
        contract(1.0);
        __syncthreads();
        if (work) {
          double o[V];
#pragma unroll
          for (int m = 0; m < V; m++) {
            double acc = f_s[(0 * V + m) * BS + off[0]];
#pragma unroll
            for (int d = 1; d < DIM; d++) acc += f_s[(d * V + m) * BS + off[d]];
            o[m] = acc;
          }
          // The sweep-0 rhs of time node i is (w_p F0[i] luh - w_i o + w_i w_p dt (S0 + src_i)) / w_p,
          // so the iK1 time solve has the closed form
          //   q1[t] = luh A[t] - o B[t] / w_p + dt S0 B[t] + dt sum_i iK1[t][i] w_i src_i
          // with A[t] = sum_i iK1[t][i] F0[i] and B[t] = sum_i iK1[t][i] w_i.
          double cs[n];
#pragma unroll
          for (int t = 0; t < n; t++) cs[t] = 0.0;
          if (PDE::kSource && srcOn) {
            for (int i = 0; i < n; i++) {
              const double wsi = G::weights(i) * dt * src_at(i);
#pragma unroll
              for (int t = 0; t < n; t++) cs[t] = fma(G::iK1(t, i), wsi, cs[t]);
            }
          }
#pragma unroll
          for (int m = 0; m < V; m++) {
#pragma unroll
            for (int t = 0; t < n; t++) {
              double q1 = u[m] * s_A[t] - iweight * o[m] * s_B[t];
              if (NCP && !ALG) q1 += dt * S0[m] * s_B[t];
              if (ALG) q1 += qn[t][m];
              if (PDE::kSource && srcOn && m == srcVar) q1 += cs[t];
              const double dl = q1 - u[m];
              res = fma(dl, dl, res);
              qn[t][m] = q1;
            }
          }
        }
      } else {
        if (work) {
#pragma unroll
          for (int t = 0; t < n; t++)
#pragma unroll
            for (int m = 0; m < V; m++) qn[t][m] = 0.0;
        }
#pragma unroll
        for (int i = 0; i < n; i++) {
          // phase 1: flux (and source) of the old iterate at time node i (:196-227, :323-367)
          double q[D];
#pragma unroll
          for (int m = 0; m < D; m++) q[m] = m < V ? q_s[(i * nd + p) * DQ + m] : u[m];
          double F[DIM * V];
          double Si[V];
          double gqi[GRAD ? DIM * V : 1];
          if constexpr (GRAD) gradient(i, gqi);
          if constexpr (VISC)
            PDE::template viscous_flux<DIM>(q, gqi, F);
          else
            PDE::template flux<DIM>(q, F);
          store_flux(F);
          const double wi = G::weights(i);
          if constexpr (NCP) {
            double B[V];
            PDE::template ncp<DIM>(q, gqi, B);
#pragma unroll
            for (int m = 0; m < V; m++) Si[m] = -B[m];
          }
          if constexpr (ALG) {
            double nS[V];
#pragma unroll
            for (int m = 0; m < V; m++) nS[m] = NCP ? Si[m] : 0.0;
            source_at(i, q, nS, Si);
          }
          if ((FHACC || SRCT) && work) {
            if (FHACC) {
#pragma unroll
              for (int d = 0; d < (FHACC ? DIM : 1); d++)
#pragma unroll
                for (int m = 0; m < V; m++) fh[d][m] = fma(F[d * V + m], wi, fh[d][m]);
            }
            if (SRCT) {
#pragma unroll
              for (int m = 0; m < V; m++) sh[m] = fma(Si[m], wi, sh[m]);
            }
          }
          if ((GRAD || SRCT) && a.ex_lFi && work) export_flux(i, F, Si);
          __syncthreads();
          // phase 2
          contract(wi);
          __syncthreads();
          // phase 3: rhs of time node i, scaled by 1/w_xyz, as slice i (:231-246, :323-367)
          if (work) {
            const double f0 = G::F0(i);
            const double si = (PDE::kSource && srcOn) ? src_at(i) : 0.0;
#pragma unroll
            for (int m = 0; m < V; m++) {
              double rhs = w_sp * f0 * u[m];
              if (PDE::kSource && srcOn && m == srcVar) rhs += wi * w_sp * dt * si;
#pragma unroll
              for (int d = 0; d < DIM; d++) rhs -= f_s[(d * V + m) * BS + off[d]];
              if (SRCT) rhs += wi * w_sp * dt * Si[m];
              // iK1 time solve (:370-405), one time node of the rhs at a time
              const double r = iweight * rhs;
#pragma unroll
              for (int t = 0; t < n; t++) qn[t][m] = fma(r, G::iK1(t, i), qn[t][m]);
            }
          }
          // no barrier: the next phase 1 rewrites only this thread's own flux slots, and the slices
          // hold the old iterate for the whole sweep
        }
        // residual against the old iterate
        if (work) {
#pragma unroll
          for (int t = 0; t < n; t++)
#pragma unroll
            for (int m = 0; m < V; m++) {
              const double dl = qn[t][m] - q_s[(t * nd + p) * DQ + m];
              res = fma(dl, dl, res);
            }
        }
      }
      // per-cell residual: segmented warp tree, one shared atomic per segment head, into this
      // sweep's buffer (zeroed at least one barrier before any thread adds to it)
      {
        const int lane = tid & 31;
        const int seg_end = (lc + 1) * nd - 1;
#pragma unroll
        for (int off2 = 16; off2 > 0; off2 >>= 1) {
          const double o2 = __shfl_down_sync(0xffffffffu, res, off2);
          if (lane + off2 < 32 && tid + off2 <= seg_end) res += o2;
        }
        if ((p == 0 || lane == 0) && work) {
          atomicAdd(&s_res[s & 1][lc], residual_units(res));
          if (!finite(res) && a.status) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
        }
      }
      __syncthreads();
      // exit test (:407-412): |res|^2 < 1e-7^2, unless a fixed sweep count is requested; every
      // thread evaluates it for every cell of the CTA from the same sums, so the decision is uniform
      unsigned conv = 0;
      if (a.max_picard <= 0) {
#pragma unroll
        for (int c = 0; c < CPB; c++) conv |= ((double)s_res[s & 1][c] < kResidualTolUnits ? 1u : 0u) << c;
      }
      conv &= active;
      if (work) {
        sweeps = s + 1;
        done = (conv >> lc) & 1u;
        // the new iterate becomes the old one, except after the last sweep: lFhi is the flux of
        // the iterate that sweep started from (a fixed sweep count, or the cap without convergence)
        if (!done && s + 1 < maxIter) {
#pragma unroll
          for (int t = 0; t < n; t++)
#pragma unroll
            for (int m = 0; m < V; m++) q_s[(t * nd + p) * DQ + m] = qn[t][m];
          if (a.ex_iter) {
            // [cell][sweep][t][V][node]: node-fastest, one coalesced run per (t, variable)
            double* e = a.ex_iter + ((size_t)cell * maxIter + s + 1) * n * nd * V + p;
#pragma unroll
            for (int t = 0; t < n; t++)
#pragma unroll
              for (int m = 0; m < V; m++) e[(size_t)(t * V + m) * nd] = qn[t][m];
          }
        } else {
          last_old_is_luh = s == 0;
        }
      }
      // the buffer of the next sweep: its last readers (the previous sweep's test) passed the
      // barrier above; the next sweep's first barrier separates this from the next additions
      if (tid < CPB) s_res[(s + 1) & 1][tid] = 0;
      active &= ~conv;
      // the gradients of the next sweep read the neighbours' copied iterate
      if (GRAD) __syncthreads();
      if (!active) break;
    }
    if (live && a.picard && p == 0) a.picard[cell] = sweeps;
    if (live && p == 0 && a.max_picard <= 0 && !done && a.status) atomicOr(a.status, ST_PICARD_CAP);

    // ---------------- time averaging (:441-515) ----------------
    // lQhi from the new iterate (registers); lFhi from the flux of the old iterate (the slices, or
    // luh when the last sweep was sweep 0)
    double qh[D];
#pragma unroll
    for (int m = 0; m < D; m++) {
      double acc = 0.0;
#pragma unroll
      for (int t = 0; t < n; t++) acc = fma(m < V ? qn[t][m] : u[m], G::weights(t), acc);
      qh[m] = acc;
    }
    if (live && a.ex_lQi) {
      double* e = a.ex_lQi + (size_t)cell * nd * n * D + (size_t)p * n * D;
#pragma unroll
      for (int t = 0; t < n; t++)
#pragma unroll
        for (int m = 0; m < D; m++) e[t * D + m] = m < V ? qn[t][m] : u[m];
    }
    // the old iterate of the last sweep, before its slot 0 takes lQhi (each thread reads and
    // writes only its own node, so no barrier is needed in between)
    double fa[FHACC ? 1 : DIM * V];
    (void)fa;
    if (!FHACC && inr) {
      // lFhi = sum_t w_t F(old iterate at t), accumulated in registers
#pragma unroll
      for (int k = 0; k < (FHACC ? 1 : DIM * V); k++) fa[k] = 0.0;
      if (last_old_is_luh) {
        // the old iterate is luh at every time node: one flux, the same weighted sum
        double F[DIM * V];
        PDE::template flux<DIM>(u, F);
#pragma unroll
        for (int i = 0; i < n; i++) {
          const double wi = G::weights(i);
#pragma unroll
          for (int k = 0; k < (FHACC ? 1 : DIM * V); k++) fa[k] = fma(F[k], wi, fa[k]);
          if (!SRCT && live && a.ex_lFi) export_flux(i, F, nullptr);  // else exported by the sweeps
        }
      } else {
#pragma unroll
        for (int i = 0; i < n; i++) {
          double q[D], F[DIM * V];
#pragma unroll
          for (int m = 0; m < D; m++) q[m] = m < V ? q_s[(i * nd + p) * DQ + m] : u[m];
          PDE::template flux<DIM>(q, F);
          const double wi = G::weights(i);
#pragma unroll
          for (int k = 0; k < (FHACC ? 1 : DIM * V); k++) fa[k] = fma(F[k], wi, fa[k]);
          if (!SRCT && live && a.ex_lFi) export_flux(i, F, nullptr);  // else exported by the sweeps
        }
      }
    }
    __syncthreads();
    // stage lQhi [node][DQ] and lShi [node][V] in the slice region, lFhi in the flux blocks
    double* qh_s = q_s;
    double* sh_s = q_s + nd * DQ;
    if (inr) {
#pragma unroll
      for (int m = 0; m < D; m++) qh_s[p * DQ + m] = qh[m];
      if (FHACC) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) f_s[(d * V + m) * BS + off[d]] = fh[FHACC ? d : 0][m];
      } else {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) f_s[(d * V + m) * BS + off[d]] = fa[(FHACC ? 0 : d * V + m)];
      }
      if (SRCT) {
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
        const int idx = node_line<DIM, n>(p, d) * n + co[d];
        for (int m = 0; m < V; m++) e[(size_t)d * nd * V + idx * V + m] = f_s[(d * V + m) * BS + off[d]];
      }
      for (int m = 0; m < V; m++) e[(size_t)DIM * nd * V + p * V + m] = SRCT ? sh[m] : 0.0;
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
        const int base = pline_base<DIM, n>(d, L), st = d == 0 ? 1 : (d == 1 ? n : n * n);
        const double wt = DIM == 3 ? s_w[L / n] * s_w[L % n] : s_w[L];
        const double us = wt * s_invdx[lc][d];
        // this node's row of Kxi, read once for every variable
        double kr[n];
#pragma unroll
        for (int mm = 0; mm < n; mm++) kr[mm] = s_Kxi[co[d] * n + mm];
#pragma unroll
        for (int m = 0; m < V; m++)
#pragma unroll
          for (int mm = 0; mm < n; mm++) acc[m] += kr[mm] * f_s[(d * V + m) * BS + base + mm * st] * us;
      }
      if (SRCT) {  // time-averaged source lShi (volumeIntegralNonlinear :211-221)
#pragma unroll
        for (int m = 0; m < V; m++) acc[m] += w_sp * sh_s[p * V + m];
      }
      if (PDE::kSource && srcOn) {  // time-averaged point source lShi (volumeIntegralNonlinear :211-221)
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

    // ---------------- extrapolation to the faces (:517-687) ----------------
    // one thread per (cell, lQhbnd or lFhbnd, direction, line): both faces of the line from one
    // read of it; the D (or V) values of a face node are contiguous in HBM
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
        const double* src = smem + (size_t)c * S::QCS + (size_t)line_base<DIM, n>(d, L) * DQ;
        double* o0 = a.lQhbnd + (size_t)gc * S::sizeQhb + (size_t)((2 * d) * nf + L) * D;
        double* o1 = a.lQhbnd + (size_t)gc * S::sizeQhb + (size_t)((2 * d + 1) * nf + L) * D;
#pragma unroll
        for (int m = 0; m < D; m++) {
          double a0 = 0.0, a1 = 0.0;
          // 2D x faces extrapolate only the evolved variables (2d/spaceTimePredictorNonlinear.cpph:436-445)
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
        const double* src = sF + (size_t)c * FCS + (size_t)d * V * BS + pline_base<DIM, n>(d, L);
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
  // a copy that ran out of time may still be in flight into this CTA's shared memory: give it one
  // more bounded wait before the CTA exits
  if (stall_parity >= 0 && tid == 0) (void)mbar_wait_bounded(&s_bar, (uint32_t)stall_parity, kBulkWaitLimitNs);
}

}  // namespace exa
