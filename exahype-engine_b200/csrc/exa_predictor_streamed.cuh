// Space-time predictor for cells whose space-time state does not fit a CTA's shared memory
// (high orders with many variables, e.g. the elastic system at N=7: 8^4 x 9 doubles = 295 KB of
// Picard iterate per cell). Same algorithm, same references and same results as
// predictor_kernel (exa_predictor.cuh); only where the state lives differs:
//
//   shared memory  the flux blocks of one time node [dir][var][node] (contracted in place);
//                  one row per node [node][DP]: its luh during the sweeps, lQhi in the tail,
//                  and w_p, 1/w_p in the spare entries; the per-cell constants. Registers are
//                  the limit at 512 threads, so these stay out of them (a runtime-indexed
//                  register array would go to local memory, which misses L1 next to the
//                  scratch traffic).
//   global scratch per resident CTA, two slabs [t][V][node]: the old Picard iterate, and the
//                  rhs slices, which the time solve overwrites in place with the new iterate
//                  (each thread reads all n slices of its own (node, variable) before writing).
//                  Node-fastest, so that a warp's access to one (t, variable) is one coalesced
//                  256-byte run.
//                  With one CTA per SM the scratch of all CTAs (148 x 2 x 8 x 512 x 9 doubles =
//                  87 MB) fits in L2.
//
// The kernel is persistent: gridDim.x CTAs walk the cells, CTA b using scratch slot b. One CTA
// holds one cell, one thread per node (n^3 <= 1024). PDEs without NCP only.
#pragma once

namespace exa {

template <class PDE, int DIM, int N, int P>
struct StreamShape {
  using S = Shape<PDE, DIM, N, P>;
  static constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, NL = S::NL, BS = S::BS;
  static constexpr int TPB = (nd + 31) / 32 * 32;
  static constexpr int items = DIM * V * NL;
  // row of the luh / lQhi block: D entries, then w_p and 1/w_p of the node (read from shared
  // memory where they are needed instead of occupying registers); the stride is odd, so that a
  // warp's rows fall in distinct bank pairs
  static constexpr int DP = (D + 2) | 1;
  static constexpr size_t smem = sizeof(double) * ((size_t)DIM * V * BS + (size_t)TPB * DP);
  static constexpr size_t slot_doubles = 2 * (size_t)n * nd * V;  // old iterate; rhs, then new iterate
};

template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__((StreamShape<PDE, DIM, N, P>::TPB))
predictor_streamed_kernel(CellArgs a) {
  using T = StreamShape<PDE, DIM, N, P>;
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = T::n, V = T::V, D = T::D, nd = T::nd, NL = T::NL, BS = T::BS, nf = S::nf;
  static_assert(!PDE::kNCP && !is_viscous<PDE>::value && !has_algebraic_source<PDE, DIM>::value,
                "the streamed predictor is built for PDEs without NCP, viscous flux or algebraic source");
  static_assert(T::TPB <= 1024, "one thread per node");
  extern __shared__ double smem[];
  double* sF = smem;                          // [DIM][V][BS]
  constexpr int DP = T::DP;
  double* sQh = smem + (size_t)DIM * V * BS;  // [TPB][DP]: each node's luh, lQhi in the tail
  __shared__ double s_lw[DIM * NL];
  __shared__ double s_A[n], s_B[n];  // sum_i iK1[t][i] F0[i] and sum_i iK1[t][i] w_i (sweep 0)
  __shared__ double s_red[T::TPB / 32];
  __shared__ double s_res;
  // per-cell constants read after the set-up (kept out of registers, which are the limit at
  // 512 threads): dt, 1/dx[3], dx[3] (as 1/(1/dx), the value the source geometry uses), t
  __shared__ double s_cd[8];
  __shared__ int s_grid;

  const int p = threadIdx.x;
  // the tail threads of the last warp (n^3 not a multiple of 32: N = 8, 9) own no node; they
  // take line items in the contractions and the extrapolation only
  const bool live_node = T::TPB == nd || p < nd;
  int co[3] = {0, 0, 0};
  node_coords<DIM, n>(live_node ? p : 0, co);
  {
    const double w = DIM == 3 ? G::weights(co[2]) * G::weights(co[1]) * G::weights(co[0])
                              : G::weights(co[1]) * G::weights(co[0]);
    sQh[(size_t)p * DP + D] = w;
    sQh[(size_t)p * DP + D + 1] = 1.0 / w;
  }
  int off[DIM];
#pragma unroll
  for (int d = 0; d < DIM; d++) off[d] = flux_off<DIM, n>(d, live_node ? p : 0);
  const size_t slab = (size_t)n * nd * V;
  if (p < n) {
    double A = 0.0, B = 0.0;
#pragma unroll
    for (int i = 0; i < n; i++) {
      A = fma(G::iK1(p, i), G::F0(i), A);
      B = fma(G::iK1(p, i), G::weights(i), B);
    }
    s_A[p] = A;
    s_B[p] = B;
  }
  double* slot = a.scratch + (size_t)blockIdx.x * T::slot_doubles;

  for (int cell = a.cell_begin + (int)blockIdx.x; cell < a.ncells; cell += (int)gridDim.x) {
    const int g = a.cell_grid ? a.cell_grid[cell] : 0;
    const double dt = a.grid_dt ? a.grid_dt[g] : a.u_dt;
    double invdx[3];
#pragma unroll
    for (int d = 0; d < 3; d++) invdx[d] = d < DIM ? 1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 0.0;
    for (int j = p; j < DIM * NL; j += T::TPB) {
      const int d = j / NL, L = j % NL;
      const double wt = DIM == 3 ? G::weights(L / n) * G::weights(L % n) : G::weights(L);
      s_lw[j] = wt * dt * (d == 0 ? invdx[0] : (d == 1 ? invdx[1] : invdx[2]));  // no runtime-indexed array
    }
    // the node's luh, read by this thread only (the previous cell's tail ended with a barrier)
    double* u = sQh + (size_t)p * DP;
    const double& w_sp = u[D];         // w_p (the tail overwrites only entries 0..D-1)
    const double& iweight = u[D + 1];  // 1 / w_p
    {
      const double* luh = a.luh + (size_t)cell * nd * D + (size_t)(live_node ? p : 0) * D;
      const uint64_t once = l2_policy_evict_first();  // luh is read once per step
#pragma unroll
      for (int m = 0; m < D; m++) u[m] = live_node ? ld_hint(luh + m, once) : 1.0;
    }
    // point source (algebraicSource at x_p, t + node_i dt)
    bool srcOn = false;
    double tcell = 0.0;
    const double dxv[3] = {1.0 / invdx[0], DIM > 1 ? 1.0 / invdx[1] : 1.0, DIM > 2 ? 1.0 / invdx[2] : 1.0};
    if (PDE::kSource && a.src) {
      double cc[3];
      cell_centre(a, cell, g, dxv, cc);
      srcOn = source_near<DIM>(a.src, cc, dxv);
      tcell = a.grid_t ? a.grid_t[g] : a.u_t;
    }
    if (p == 0) {
      s_cd[0] = dt;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        s_cd[1 + d] = invdx[d];
        s_cd[4 + d] = dxv[d];
      }
      s_cd[7] = tcell;
      s_grid = g;
    }
    const int srcVar = (PDE::kSource && a.src) ? (int)a.src[7] : -1;
    auto src_at = [&](int i) -> double {
      const double dxs[3] = {s_cd[4], s_cd[5], s_cd[6]};
      double cc[3], x[3];
      cell_centre(a, cell, s_grid, dxs, cc);
#pragma unroll
      for (int d = 0; d < 3; d++) x[d] = cc[d] + dxs[d] * (G::nodes(co[d]) - 0.5);
      return point_source<DIM>(a.src, x, s_cd[7] + G::nodes(i) * s_cd[0]);
    };
    __syncthreads();

    // contraction of every line with Kxi, in place, scaled by coef * s_lw
    auto contract = [&](double coef) {
      for (int it = p; it < T::items; it += T::TPB) {
        const int L = it % NL, d = it / (V * NL), m = (it / NL) % V;
        double* f = sF + (size_t)(d * V + m) * BS + flux_off<DIM, n>(d, line_base<DIM, n>(d, L));
        const int st = line_stride<n>(d);
        const double c = coef * s_lw[d * NL + L];
        double x[n];
#pragma unroll
        for (int k = 0; k < n; k++) x[k] = f[k * st];
#pragma unroll
        for (int l = 0; l < n; l++) {
          double acc = 0.0;
#pragma unroll
          for (int k = 0; k < n; k++) acc = fma(x[k], G::Kxi(k, l), acc);
          f[l * st] = c * acc;
        }
      }
    };
    auto store_flux = [&](const double* q) {
      double F[DIM * V];
      PDE::template flux<DIM>(q, F);
      if (live_node) {
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) sF[(d * V + m) * BS + off[d]] = F[d * V + m];
      }
    };

    double* qo = slot;             // old iterate [t][V][node]
    double* qn = slot + slab;      // rhs slices (scaled by 1/w_p), then the new iterate
    // entry (t, m) of this thread's node in a slab
    auto at = [&](int t, int m) -> size_t { return ((size_t)t * V + m) * nd + p; };
    // the slot is re-read every sweep: ask L2 to keep it over the streamed luh and outputs
    const uint64_t keep = l2_policy_evict_last();
    const int maxIter = a.max_picard > 0 ? a.max_picard : S::maxSweeps;
    int sweeps = 0;
    bool last_old_is_luh = true;   // the last sweep started from lQi = luh
    for (int s = 0; s < maxIter; s++) {
      double res = 0.0;
      if (s == 0) {
        // lQi[., t] = luh (:71-82): one flux and one set of contractions for every time node.
        // The rhs of time node i is (w_p F0[i] luh - w_i o + w_i w_p dt src_i) / w_p, so the iK1
        // time solve has the closed form q1[t] = luh A[t] - o B[t] / w_p + dt sum_i iK1[t][i] w_i src_i.
        store_flux(u);
        __syncthreads();
        contract(1.0);
        __syncthreads();
        if (live_node) {
          double cs[n];
#pragma unroll
          for (int t = 0; t < n; t++) cs[t] = 0.0;
          if (PDE::kSource && srcOn) {
            for (int i = 0; i < n; i++) {
              const double wsi = G::weights(i) * s_cd[0] * src_at(i);
#pragma unroll
              for (int t = 0; t < n; t++) cs[t] = fma(G::iK1(t, i), wsi, cs[t]);
            }
          }
#pragma unroll 1
          for (int m = 0; m < V; m++) {
            double o = 0.0;
            const double um = u[m];
#pragma unroll
            for (int d = 0; d < DIM; d++) o += sF[(d * V + m) * BS + off[d]];
#pragma unroll
            for (int t = 0; t < n; t++) {
              double q1 = um * s_A[t] - iweight * o * s_B[t];
              if (PDE::kSource && srcOn && m == srcVar) q1 += cs[t];
              const double dl = q1 - um;
              res = fma(dl, dl, res);
              st_hint(qn + at(t, m), q1, keep);
            }
          }
        }
      } else {
        double* R = qn;
        for (int i = 0; i < n; i++) {
          double q[D];
#pragma unroll
          for (int m = 0; m < D; m++) q[m] = (m < V && live_node) ? ld_hint(qo + at(i, m), keep) : u[m];
          store_flux(q);
          __syncthreads();
          contract(G::weights(i));
          __syncthreads();
          if (live_node) {
            const double wi = G::weights(i);
            const double si = (PDE::kSource && srcOn) ? src_at(i) : 0.0;
#pragma unroll
            for (int m = 0; m < V; m++) {
              double rhs = w_sp * G::F0(i) * u[m];
#pragma unroll
              for (int d = 0; d < DIM; d++) rhs -= sF[(d * V + m) * BS + off[d]];
              if (PDE::kSource && srcOn && m == srcVar) rhs += wi * w_sp * s_cd[0] * si;
              st_hint(R + at(i, m), iweight * rhs, keep);
            }
          }
          // no barrier: the next phase 1 rewrites only this thread's own flux slots, which this
          // thread has just read (every node's slots are written and read by its own thread)
        }
      }
      // iK1 time solve (:370-405) per node, in place over the rhs slices (all n slices of a
      // (node, variable) are read before any is overwritten), residual against the old iterate
      if (live_node && s > 0) {
#pragma unroll 1
        for (int m = 0; m < V; m++) {
          // both columns are loaded before the first store: a store to qn may alias a later qo
          // load as far as the compiler knows, which would serialise one round trip per load
          double r[n], ol[n];
#pragma unroll
          for (int i = 0; i < n; i++) {
            r[i] = ld_hint(qn + at(i, m), keep);
            ol[i] = ld_hint(qo + at(i, m), keep);
          }
#pragma unroll
          for (int t = 0; t < n; t++) {
            double q = 0.0;
#pragma unroll
            for (int i = 0; i < n; i++) q = fma(r[i], G::iK1(t, i), q);
            const double dl = q - ol[t];
            res = fma(dl, dl, res);
            st_hint(qn + at(t, m), q, keep);
          }
        }
      }
      // residual of the cell: warp tree, then the warp partials
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) res += __shfl_xor_sync(0xffffffffu, res, o2);
      if ((p & 31) == 0) s_red[p >> 5] = res;
      __syncthreads();
      if (p == 0) {
        double t = 0.0;
        for (int w = 0; w < T::TPB / 32; w++) t += s_red[w];
        s_res = t;
      }
      __syncthreads();
      const double rr = s_res;
      sweeps = s + 1;
      if (!finite(rr) && a.status && p == 0) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
      const bool done = a.max_picard <= 0 && rr < 1e-7 * 1e-7;
      if (done || s + 1 == maxIter) {
        if (!done && a.max_picard <= 0 && a.status && p == 0) atomicOr(a.status, ST_PICARD_CAP);
        last_old_is_luh = s == 0;
        break;
      }
      // the new iterate becomes the old one
      double* t = qo;
      qo = qn;
      qn = t;
      __syncthreads();
    }
    if (a.picard && p == 0) a.picard[cell] = sweeps;

    // ---------------- time averaging (:441-515) ----------------
    // lQhi from the new iterate; lFhi = sum_t w_t F(old iterate of the last sweep at t)
    double qh[D] = {};
    if (live_node) {
#pragma unroll
      for (int m = 0; m < D; m++) {
        double acc = 0.0;
#pragma unroll
        for (int t = 0; t < n; t++) acc = fma(m < V ? ld_hint(qn + at(t, m), keep) : u[m], G::weights(t), acc);
        qh[m] = acc;
      }
      if (a.ex_lQi) {
        double* e = a.ex_lQi + (size_t)cell * nd * n * D + (size_t)p * n * D;
        for (int t = 0; t < n; t++)
          for (int m = 0; m < D; m++) e[t * D + m] = m < V ? ld_hint(qn + at(t, m), keep) : u[m];
      }
      if (a.ex_lQhi)
        for (int m = 0; m < D; m++) a.ex_lQhi[(size_t)cell * nd * D + p * D + m] = qh[m];
#pragma unroll
      for (int d = 0; d < DIM; d++)
#pragma unroll
        for (int m = 0; m < V; m++) sF[(d * V + m) * BS + off[d]] = 0.0;
#pragma unroll 1
      for (int i = 0; i < n; i++) {
        double q[D], F[DIM * V];
#pragma unroll
        for (int m = 0; m < D; m++) q[m] = (m < V && !last_old_is_luh) ? ld_hint(qo + at(i, m), keep) : u[m];
        PDE::template flux<DIM>(q, F);
        const double wi = G::weights(i);
#pragma unroll
        for (int d = 0; d < DIM; d++)
#pragma unroll
          for (int m = 0; m < V; m++) {
            double* sl = &sF[(d * V + m) * BS + off[d]];
            *sl = fma(F[d * V + m], wi, *sl);
          }
        if (a.ex_lFi) {
          double* e = a.ex_lFi + (size_t)cell * n * nd * (DIM + 1) * V + ((size_t)(i * nd + p) * (DIM + 1)) * V;
          for (int d = 0; d < DIM; d++)
            for (int m = 0; m < V; m++) e[d * V + m] = F[d * V + m];
          for (int m = 0; m < V; m++) e[DIM * V + m] = 0.0;
        }
      }
      if (a.ex_lFhi) {
        double* e = a.ex_lFhi + (size_t)cell * (DIM + 1) * nd * V;
        for (int d = 0; d < DIM; d++) {
          const int idx = node_line<DIM, n>(p, d) * n + co[d];
          for (int m = 0; m < V; m++) e[(size_t)d * nd * V + idx * V + m] = sF[(d * V + m) * BS + off[d]];
        }
        for (int m = 0; m < V; m++) e[(size_t)DIM * nd * V + p * V + m] = 0.0;
      }
      // lQhi replaces the node's luh row only now: the flux loop above still read luh
#pragma unroll
      for (int m = 0; m < D; m++) u[m] = qh[m];
    }
    __syncthreads();

    // ---------------- volume integral (volumeIntegralNonlinear :133-223) ----------------
    if (live_node) {
      double acc[V];
#pragma unroll
      for (int m = 0; m < V; m++) acc[m] = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int L = node_line<DIM, n>(p, d);
        const int base = flux_off<DIM, n>(d, line_base<DIM, n>(d, L)), st = line_stride<n>(d);
        const double wt = DIM == 3 ? G::weights(L / n) * G::weights(L % n) : G::weights(L);
        const double us = wt * s_cd[1 + d];
        const int k = co[d];
#pragma unroll
        for (int m = 0; m < V; m++)
#pragma unroll
          for (int mm = 0; mm < n; mm++) acc[m] += G::Kxi(k, mm) * sF[(d * V + m) * BS + base + mm * st] * us;
      }
      if (PDE::kSource && srcOn) {
        double sa = 0.0;
        for (int i = 0; i < n; i++) sa = fma(src_at(i), G::weights(i), sa);
#pragma unroll
        for (int m = 0; m < V; m++)
          if (m == srcVar) acc[m] += w_sp * sa;
      }
      bool ok = true;
      double* lduh = a.lduh + (size_t)cell * nd * V + (size_t)p * V;
#pragma unroll
      for (int m = 0; m < V; m++) {
        lduh[m] = acc[m];
        ok &= finite(acc[m]);
      }
      if (!ok && a.status) atomicOr(a.status, ST_NONFINITE_PREDICTOR);
    }

    // ---------------- extrapolation to the faces (:517-687) ----------------
    // one thread per (lQhbnd or lFhbnd, direction, line): both faces of the line from one read
    constexpr int LQ = DIM * NL;
    for (int j = p; j < 2 * LQ; j += T::TPB) {
      const bool isQ = j < LQ;
      const int rl = isQ ? j : j - LQ;
      const int d = rl / NL, L = rl % NL;
      const int st = line_stride<n>(d);
      if (isQ) {
        const double* src = sQh + (size_t)line_base<DIM, n>(d, L) * DP;
        double* o0 = a.lQhbnd + (size_t)cell * S::sizeQhb + (size_t)((2 * d) * nf + L) * D;
        double* o1 = a.lQhbnd + (size_t)cell * S::sizeQhb + (size_t)((2 * d + 1) * nf + L) * D;
#pragma unroll 1
        for (int m = 0; m < D; m++) {
          double a0 = 0.0, a1 = 0.0;
          if (!(DIM == 2 && d == 0 && m >= V)) {
#pragma unroll
            for (int l = 0; l < n; l++) {
              const double x = src[(size_t)l * st * DP + m];
              a0 = fma(x, G::F0(l), a0);
              a1 = fma(x, G::F1(l), a1);
            }
          }
          o0[m] = a0;
          o1[m] = a1;
        }
      } else {
        const double* src = sF + (size_t)d * V * BS + flux_off<DIM, n>(d, line_base<DIM, n>(d, L));
        double* o0 = a.lFhbnd + (size_t)cell * S::sizeFhb + (size_t)((2 * d) * nf + L) * V;
        double* o1 = a.lFhbnd + (size_t)cell * S::sizeFhb + (size_t)((2 * d + 1) * nf + L) * V;
#pragma unroll 1
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
    __syncthreads();  // shared memory and scratch are reused by the next cell
  }
}

}  // namespace exa
