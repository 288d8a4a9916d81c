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

#include "exa_async.cuh"
#include "exa_pde.cuh"
#include "exa_tables.cuh"

namespace exa {

enum : unsigned {
  ST_NONFINITE_PREDICTOR = 1u,
  ST_PICARD_CAP = 2u,
  ST_NONFINITE_UPDATE = 4u,
  ST_BAD_DT = 8u,
  ST_TIMEOUT = 16u,  // a bounded wait (bulk copy) ran out; the launch's results are not valid
};

// Shared-memory layout of the predictor's flux blocks (one block per cell, direction, variable).
// Node p of direction d's block sits at p + (p / G1) S1 + (p / G2) S2: whole lines stay
// contiguous (the groups are multiples of the line's footprint: n nodes for x lines, an n^2
// plane for y lines), and the padding spreads the accesses of phase 1/3 (one thread per node)
// and of phase 2 (one thread per line) over the 32 banks. BS is the block stride. The values
// were chosen per (DIM, n) by counting shared-memory wavefronts of every access of a time node
// (64-bit accesses, 16 lanes per wavefront) over candidate paddings.
// per direction d: the group sizes G1, G2 (0 = none) and the padding S1, S2 per group
#define EXA_FLUX_LAYOUT(g1x, g1y, s1x, s1y, g2x, s2x, ext)                                   \
  static __host__ __device__ constexpr int G1(int d) { return d == 0 ? g1x : (d == 1 ? g1y : 0); } \
  static __host__ __device__ constexpr int S1(int d) { return d == 0 ? s1x : (d == 1 ? s1y : 0); } \
  static __host__ __device__ constexpr int G2(int d) { return d == 0 ? g2x : 0; }                  \
  static __host__ __device__ constexpr int S2(int d) { return d == 0 ? s2x : 0; }                  \
  static constexpr int extra = ext;
template <int DIM, int n>
struct FluxLayout {  // default: unpadded, odd block stride
  EXA_FLUX_LAYOUT(0, 0, 0, 0, 0, 0, 1)
};
template <>
struct FluxLayout<3, 6> {  // N=5: 1700 -> 1386 wavefronts per time node (ideal 1248)
  EXA_FLUX_LAYOUT(48, 36, 3, 2, 96, 10, 0)
};
template <>
struct FluxLayout<3, 4> {  // N=3: conflict-free
  EXA_FLUX_LAYOUT(16, 16, 1, 4, 0, 0, 0)
};
template <>
struct FluxLayout<3, 8> {  // N=7: 9792 -> 5184 wavefronts per time node (conflict-free per direction)
  EXA_FLUX_LAYOUT(16, 64, 1, 8, 0, 0, 0)
};
template <>
struct FluxLayout<3, 5> {  // N=4: unpadded lines, block stride 137
  EXA_FLUX_LAYOUT(0, 0, 0, 0, 0, 0, 12)
};
template <>
struct FluxLayout<2, 4> {
  EXA_FLUX_LAYOUT(0, 0, 0, 0, 0, 0, 5)
};
template <>
struct FluxLayout<2, 5> {
  EXA_FLUX_LAYOUT(0, 0, 0, 0, 0, 0, 0)
};
#undef EXA_FLUX_LAYOUT
template <int DIM, int n>
__host__ __device__ constexpr int flux_off(int d, int p) {
  using F = FluxLayout<DIM, n>;
  return p + (F::G1(d) ? (p / F::G1(d)) * F::S1(d) : 0) + (F::G2(d) ? (p / F::G2(d)) * F::S2(d) : 0);
}
template <int DIM, int n>
constexpr int flux_block() {
  constexpr int nd = DIM == 3 ? n * n * n : n * n;
  int mx = 0;
  for (int d = 0; d < DIM; d++) mx = flux_off<DIM, n>(d, nd - 1) + 1 > mx ? flux_off<DIM, n>(d, nd - 1) + 1 : mx;
  return mx + FluxLayout<DIM, n>::extra;
}

template <class PDE, int DIM, int N, int P>
struct Shape {
  static constexpr int n = N + 1;
  static constexpr int V = PDE::V;
  static constexpr int D = V + P;
  static constexpr int nd = DIM == 3 ? n * n * n : n * n;  // nodes per cell
  static constexpr int nf = DIM == 3 ? n * n : n;          // nodes per face
  static constexpr int NL = nd / n;                        // lines per direction
  // cells per CTA: about 256 threads, at most 32 cells (the predictors' per-CTA cell masks)
  // threads per CTA aimed at: 256, or 128 for the n=5, V=4 shapes (2D SWE N=4: 5 cells per CTA;
  // 3D acoustics N=4: one cell), whose four resident CTAs per SM then wait at their barriers in
  // groups of four warps instead of eight (measured: SWE 512-grid step -5.5%, acoustic 32^3
  // forward step -9.4%, bit-identical results)
  static constexpr int kThreads = (n == 5 && V == 4) ? 128 : 256;
  static constexpr int CPB = nd >= kThreads ? 1 : (kThreads / nd > 32 ? 32 : kThreads / nd);
  static constexpr int TPB = (CPB * nd + 31) / 32 * 32;    // whole warps; the tail threads idle
  static constexpr int sizeQhb = 2 * DIM * nf * D;
  static constexpr int sizeFhb = 2 * DIM * nf * V;
  static constexpr int maxSweeps = 2 * n;
  // flux/partials block of one (cell, dir, var), laid out by FluxLayout
  static constexpr int BS = flux_block<DIM, n>();
  // stride between the flux blocks of the CTA's cells: in 2D, where a warp spans parts of two
  // cells, one pad double makes it odd, so the next cell's lanes land on other bank pairs than
  // the ones the first cell's lanes already use twice
  static constexpr int FCS = DIM * V * BS + ((DIM == 2 && CPB > 1 && (DIM * V * BS) % 2 == 0) ? 1 : 0);
  static constexpr int smemF = CPB * FCS;
  static constexpr int smemStage = CPB * nd * D;               // bulk-copy target of the next cells' luh
  static constexpr int even(int x) { return (x + 1) / 2 * 2; }  // 16-byte boundary in doubles
  // predictor shared memory for a given per-node stride dq of the iterate slices and the luh
  // block; the staging buffer of the persistent form comes last
  // per-cell stride of the iterate slices [t][node][dq]: where a warp spans two cells (CPB > 1),
  // padded to a stride congruent to nd*dq modulo 16 words, so that the next cell's nodes continue
  // the bank-pair progression of the node stride dq instead of landing on pairs the first cell's
  // lanes already use (2D N=4: 625 -> 637 words)
  static constexpr int qcs(int dq) {
    return CPB > 1 ? n * nd * dq + ((nd * dq - n * nd * dq) % 16 + 16) % 16 : n * nd * dq;
  }
  static constexpr size_t smem_for(int dq) {
    return sizeof(double) * (size_t)(even(CPB * qcs(dq) + smemF + CPB * nd * dq) + smemStage);
  }
  // resident CTAs per SM: two when their shared memory fits (228 KB per SM, 1 KB reserved per CTA)
  // (up to four for CTAs of at most 128 threads)
  static constexpr int blocks_for(int dq) {
    return TPB <= 128 ? ((int)(228 * 1024 / (smem_for(dq) + 3 * 1024)) > 4 ? 4 : ((int)(228 * 1024 / (smem_for(dq) + 3 * 1024)) < 1 ? 1 : (int)(228 * 1024 / (smem_for(dq) + 3 * 1024))))
                      : (2 * (smem_for(dq) + 3 * 1024) <= 228 * 1024 ? 2 : 1);
  }
  static constexpr bool fits_cta(size_t bytes) { return bytes + 4096 <= 227 * 1024; }
  // per-node stride of the iterate slices and the luh block in shared memory: D rounded up to an
  // odd count (an even stride puts several lanes of a warp on one bank), unless the padding
  // would cost a resident CTA or push a form of the kernel past one CTA's shared memory
  static constexpr bool pad_ok = D % 2 == 0 && blocks_for(D | 1) >= blocks_for(D) &&
                                 fits_cta(smem_for(D | 1)) >= fits_cta(smem_for(D));
  static constexpr int DQ = pad_ok ? (D | 1) : D;
  // dynamic shared memory of the predictor: iterate/rhs slices [cell][t][node][DQ] + flux/partials
  static constexpr int QCS = qcs(DQ);
  static constexpr int smemQ = CPB * QCS;
  static constexpr int items = CPB * DIM * V * NL;             // line contractions per time node
  static constexpr int rounds = (items + TPB - 1) / TPB;       // per thread
  static constexpr int smemU = CPB * nd * DQ;                  // luh of the CTA's cells
  // offset of the luh staging buffer (doubles, even: 16-byte aligned for the bulk copy)
  static constexpr int stage_off() { return even(smemQ + smemF + smemU); }
  // dynamic shared memory of the one-group-per-CTA form (no staging buffer) and the persistent one
  static constexpr size_t predictor_smem = sizeof(double) * (smemQ + smemF + smemU);
  static constexpr size_t predictor_smem_persist = sizeof(double) * (stage_off() + smemStage);
  static constexpr int MinBlocks = blocks_for(DQ);
  // registers are split over the SM's four 16K-register partitions: B blocks of W warps need
  // ceil(B*W/4) warps' worth of registers in one partition
  static constexpr int WarpsPerSmsp = (MinBlocks * (TPB / 32) + 3) / 4;
  static constexpr int MaxRegs = (512 / WarpsPerSmsp) / 8 * 8 > 255 ? 255 : (512 / WarpsPerSmsp) / 8 * 8;
};

// Arguments shared by the cell kernels (device pointers).
struct CellArgs {
  int ncells;               // end of the cell range the launch covers (exclusive)
  int cell_begin;           // first cell of the range (launches cover [cell_begin, ncells))
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
  double pnpm;              // PNPM alone (the viscous term of the CFL denominator)
  // point source (nullable): {x, y, z, f0, t0, amplitude, width, variable}; needs the geometry
  const double* src;
  const double* grid_geo;        // [grid][6]: lower corner xyz, cells per axis xyz
  const long long* grid_first;   // [grid] first cell of the grid in the batch
  const double* centres;         // [cell][3] cell centres (nullable: from grid_geo), for sources
  const double* grid_t;          // [grid] time at the start of the step (nullable: u_t)
  double u_t;
  // the point source's values, evaluated ahead of the FP64 predictor (source_values_kernel):
  // src_slot [cell] = the cell's slot, -1 for cells the source does not reach; src_cells [slot]
  // = its cell; src_vals [slot][t][node] = the source at the node and time node t (nullable)
  const int* src_slot;
  const int* src_cells;
  double* src_vals;
  int nsrc;
  // optional export of the predictor's internals, reference layouts (per-cell shims, tests)
  // scratch of the streamed predictor: one slot per resident CTA (set by the launcher)
  double* scratch;
  // optional export of every sweep's new iterate [cell][S][n][V][nd] (slot s holds q^s; the
  // adjoint reads them back instead of recomputing the Picard sweeps)
  double* ex_iter;
  double* ex_lQi;
  double* ex_lFi;
  double* ex_lQhi;
  double* ex_lFhi;
  // the predictor may fetch luh with 16-byte bulk copies (luh 16-byte aligned and nd*D even;
  // set by the launcher)
  int bulk_luh;
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
  const int8_t* btype;      // boundary type (EXA_BC_WALL, EXA_BC_OUTFLOW, EXA_BC_USER)
  unsigned* status;         // error bits (nullable): bounded waits that ran out
  // geometry and time of the boundary faces' cells (EXA_BC_USER: the functor's boundary_values
  // is evaluated at the face nodes' coordinates); nullable grid arrays as in CellArgs
  const int* cell_grid;
  const double* grid_dx;
  const double* grid_geo;
  const long long* grid_first;
  const double* grid_t;
  const double* grid_dt;
  double u_dx[3];
  double u_t, u_dt;
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

// Regularised point source S_var(x, t) = A r(t - t0) exp(-|x - xs|^2 / (2 w^2)) / ((2 pi)^(d/2) w^d)
// with the Ricker wavelet r(s) = (1 - 2 pi^2 f0^2 s^2) exp(-pi^2 f0^2 s^2); the pointwise
// algebraicSource(x, t, Q, S) of the reference's solver API for a source at xs.
template <int DIM>
__device__ __forceinline__ double point_source(const double* src, const double* x, double t) {
  const double pi = 3.14159265358979323846;
  double r2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; d++) r2 += (x[d] - src[d]) * (x[d] - src[d]);
  const double w = src[6];
  const double a = pi * src[3] * (t - src[4]);
  const double ricker = (1.0 - 2.0 * a * a) * exp(-a * a);
  const double norm = DIM == 3 ? 1.0 / (15.749609945722419 * w * w * w) : 1.0 / (6.283185307179586 * w * w);
  return src[5] * ricker * exp(-0.5 * r2 / (w * w)) * norm;
}
// The source acts on cells whose centre lies within 6 widths plus a cell diagonal of xs.
template <int DIM>
__device__ __forceinline__ bool source_near(const double* src, const double* centre, const double* dx) {
  double r2 = 0.0, h2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    r2 += (centre[d] - src[d]) * (centre[d] - src[d]);
    h2 += dx[d] * dx[d];
  }
  const double reach = 6.0 * src[6] + sqrt(h2);
  return r2 <= reach * reach;
}
// centre of cell `cell` of grid g from the grid geometry
__device__ __forceinline__ void cell_centre(const CellArgs& a, long cell, int g, const double* dx, double* c) {
  if (a.centres) {  // the caller's cell centres
#pragma unroll
    for (int k = 0; k < 3; k++) c[k] = a.centres[3 * cell + k];
    return;
  }
  const double* G = a.grid_geo + 6 * g;
  const long long loc = cell - (a.grid_first ? a.grid_first[g] : 0);
  const long long nx = (long long)G[3], ny = (long long)G[4];
  const long long ix = loc % nx, iy = (loc / nx) % ny, iz = loc / (nx * ny);
  c[0] = G[0] + (ix + 0.5) * dx[0];
  c[1] = G[1] + (iy + 0.5) * dx[1];
  c[2] = G[2] + (iz + 0.5) * dx[2];
}

// node spacing as the predictor derives it: 1 / (1 / dx), the reference's 1 / invDx (:339-342)
template <int DIM>
__device__ __forceinline__ void source_dx(const CellArgs& a, int g, double* dxv) {
#pragma unroll
  for (int d = 0; d < 3; d++) dxv[d] = d < DIM ? 1.0 / (1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d])) : 1.0;
}

// The cells the point source reaches (source_near, the predictor's test) get consecutive slots;
// one thread per cell. count starts at zero; the slots' order is immaterial.
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) source_slot_kernel(CellArgs a, int* slot, int* cells, int* count) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.ncells) return;
  int sl = -1;
  if (PDE::kSource && a.src) {
    const int g = a.cell_grid ? a.cell_grid[c] : 0;
    double dxv[3], cc[3];
    source_dx<DIM>(a, g, dxv);
    cell_centre(a, c, g, dxv, cc);
    if (source_near<DIM>(a.src, cc, dxv)) {
      sl = atomicAdd(count, 1);
      cells[sl] = (int)c;
    }
  }
  slot[c] = sl;
}

// The point source at every node and time node of every slot's cell for the coming step (the
// algebraicSource values the predictor adds, :323-337): one CTA per slot. It does not depend on
// the iterate, so the predictor reads these values instead of evaluating the source itself, which
// keeps that code out of the sweeps' registers.
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) source_values_kernel(CellArgs a) {
  using G = GL<N>;
  constexpr int n = N + 1, nd = DIM == 3 ? n * n * n : n * n;
  const int sl = blockIdx.x;
  if (sl >= a.nsrc) return;
  const long c = a.src_cells[sl];
  if (c < a.cell_begin || c >= a.ncells) return;  // another launch's range
  const int g = a.cell_grid ? a.cell_grid[c] : 0;
  double dxv[3], cc[3];
  source_dx<DIM>(a, g, dxv);
  cell_centre(a, c, g, dxv, cc);
  const double tcell = a.grid_t ? a.grid_t[g] : a.u_t;
  const double dt = a.grid_dt ? a.grid_dt[g] : a.u_dt;
  for (int p = threadIdx.x; p < nd; p += blockDim.x) {
    int co[3];
    node_coords<DIM, n>(p, co);
    double x[3];
#pragma unroll
    for (int d = 0; d < 3; d++) x[d] = cc[d] + dxv[d] * (G::nodes(co[d]) - 0.5);
#pragma unroll 1
    for (int i = 0; i < n; i++)
      a.src_vals[((size_t)sl * n + i) * nd + p] = point_source<DIM>(a.src, x, tcell + G::nodes(i) * dt);
  }
}

// Picard residual of a cell whose nodes span several warps: each warp's partial (a fixed shuffle
// tree) is added to the cell's sum as an unsigned 64-bit fixed-point number in units of 2^-100.
// Integer addition does not depend on the order in which the warps arrive, so a cell at the
// tolerance takes the same number of sweeps in every run (shared-memory atomics on doubles add in
// arrival order, whose rounding varies). A partial is clamped to 2^60 units (about 9e-13, far
// above the 1e-14 tolerance; at most 8 warps per cell keep the sum below 2^63); non-finite
// partials clamp there too, so their cell does not converge, and the caller flags them.
__device__ __forceinline__ unsigned long long residual_units(double res) {
  return (unsigned long long)fmin(res * 0x1p100, 0x1p60);
}
constexpr double kResidualTolUnits = 1e-7 * 1e-7 * 0x1p100;  // the exit test |res|^2 < 1e-7^2

__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMin(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

}  // namespace exa

#include "exa_predictor.cuh"
#include "exa_predictor_mixed.cuh"
#include "exa_predictor_streamed.cuh"

namespace exa {

// ------------------------------------------------------------------------------------------
// Rusanov on interior faces: one warp per face, in place on lFhbnd
// ------------------------------------------------------------------------------------------
// Ghost state of a domain face (boundaryValues): a reflective wall mirrors the normal velocity;
// normal < 0 selects outflow, the inner state itself (transparent / absorbing for normal waves).
template <class PDE, int DIM, int D>
__device__ __forceinline__ void ghost_state(const double* qin, int normal, double* qout) {
  if (normal < 0) {
#pragma unroll
    for (int m = 0; m < D; m++) qout[m] = qin[m];
  } else {
    PDE::template wall<DIM>(qin, normal, qout);
  }
}

// Rusanov flux of one face (riemannSolverNonlinear :37-128), in place on FL / FR. ghostL / ghostR:
// that side is the outside of a domain face; ghost(fn, qin, fin, qout, fout) then supplies the outer
// state (D values) and its normal flux (V values) at face node fn from the inner ones, as the
// reference's boundaryConditions + boundaryValues do (3d/boundaryConditions.cpph:29-122).
// face_dx: the cells' size along the face normal; a viscous flux (useViscousFlux) adds
// 2 (2N+1) / (face_dx sqrt(pi/2)) times the larger side's maximal viscous eigenvalue to the
// Rusanov speed (riemannSolverNonlinear :73-87).
template <class PDE, int DIM, int N, int P, class Ghost>
__device__ __forceinline__ void rusanov_face(const double* QL, const double* QR, double* FL, double* FR, int d,
                                             int lane, bool ghostL, bool ghostR, Ghost ghost, double face_dx) {
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
    if (ghostL || ghostR) {
      double fg[V];
      if (ghostL) ghost(fn, qr, FR + fn * V, ql, fg);
      if (ghostR) ghost(fn, ql, FL + fn * V, qr, fg);
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
  double smax = fmax(sL, sR);
  if constexpr (is_viscous<PDE>::value) {
    PDE::template viscous_eigenvalues<DIM>(aL, d, lL);
    PDE::template viscous_eigenvalues<DIM>(aR, d, lR);
    double vL = fabs(lL[0]), vR = fabs(lR[0]);
#pragma unroll
    for (int m = 1; m < V; m++) {
      vL = fmax(vL, fabs(lL[m]));
      vR = fmax(vR, fabs(lR[m]));
    }
    const double factor = 2 * (2 * N + 1) / (face_dx * sqrt(0.5 * 3.14159265358979323846));
    smax += factor * fmax(vL, vR);
  } else {
    (void)face_dx;
  }
  for (int fn = lane; fn < nf; fn += 32) {
    double ql[D], qr[D], fl[V], fr[V];
#pragma unroll
    for (int m = 0; m < D; m++) {
      ql[m] = QL[fn * D + m];
      qr[m] = QR[fn * D + m];
    }
    if (ghostL || ghostR) {
      double fg[V];
      if (ghostL) ghost(fn, qr, FR + fn * V, ql, fg);
      if (ghostR) ghost(fn, ql, FL + fn * V, qr, fg);
#pragma unroll
      for (int m = 0; m < V; m++) {
        fl[m] = ghostL ? fg[m] : FL[fn * V + m];
        fr[m] = ghostR ? fg[m] : FR[fn * V + m];
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
      for (int k = 0; k < DIM; k++)
#pragma unroll
        for (int m = 0; m < V; m++) gq[k * V + m] = k == d ? qr[m] - ql[m] : 0.0;
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

// the built-in domain faces: a reflective wall (the functor's wall, its normal flux) or outflow
// (normal < 0: the inner state itself); material parameters are copied from the inside
template <class PDE, int DIM, int N, int P>
struct BuiltinGhost {
  int normal, d;
  __device__ __forceinline__ void operator()(int, const double* qin, const double*, double* qout, double* fout) const {
    constexpr int V = PDE::V, D = Shape<PDE, DIM, N, P>::D;
    ghost_state<PDE, DIM, D>(qin, normal, qout);
#pragma unroll
    for (int m = V; m < D; m++) qout[m] = qin[m];
    double Fg[DIM * V];
    PDE::template flux<DIM>(qout, Fg);
#pragma unroll
    for (int m = 0; m < V; m++) {
      double f = Fg[m];
#pragma unroll
      for (int k = 1; k < DIM; k++)
        if (k == d) f = Fg[k * V + m];
      fout[m] = f;
    }
  }
};

// EXA_BC_USER faces: the functor's boundary_values at the face node's position x (the reference's
// node coordinates, 3d/boundaryConditions.cpph:79-103: the normal coordinate on the face, the
// tangential ones at the Gauss-Legendre nodes of the cell)
template <class PDE, int DIM, int N, int P>
struct UserGhost {
  double centre[3], dx[3], t, dt;
  int face, d;
  __device__ __forceinline__ void operator()(int fn, const double* qin, const double* fin, double* qout,
                                             double* fout) const {
    if constexpr (has_boundary_values<PDE, DIM>::value) {
      using G = GL<N>;
      constexpr int n = N + 1, D = Shape<PDE, DIM, N, P>::D;
      double x[3] = {centre[0], centre[1], centre[2]};
      x[d] = centre[d] + (-0.5 + (face & 1)) * dx[d];
      // tangential axes, slower first: (z, y) for x faces, (z, x) for y faces, (y, x) for z faces
      const int d1 = d == 0 ? 1 : 0, d2 = DIM == 3 ? (d == 2 ? 1 : 2) : -1;
      if (DIM == 3) {
        x[d2] = centre[d2] + dx[d2] * (G::nodes(fn / n) - 0.5);
        x[d1] = centre[d1] + dx[d1] * (G::nodes(fn % n) - 0.5);
      } else {
        x[d1] = centre[d1] + dx[d1] * (G::nodes(fn) - 0.5);
      }
#pragma unroll
      for (int m = 0; m < D; m++) qout[m] = qin[m];
      PDE::template boundary_values<DIM>(x, t, dt, face, d, fin, qin, fout, qout);
    } else {
      (void)fn, (void)qin, (void)fin, (void)qout, (void)fout;
    }
  }
};

// CFL denominator of one node (stableTimeStepSize :36-56): sum_d max_m |lambda_d| / dx_d, where
// a viscous flux adds max_m |viscous lambda_d| 2 / PNPM / dx_d to the maximum
template <class PDE, int DIM>
__device__ __forceinline__ double cfl_denominator(const double* q, const double* invDx, double pnpm) {
  constexpr int V = PDE::V;
  double den = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; d++) {
    double lam[V];
    PDE::template eigenvalues<DIM>(q, d, lam);
    double mx = 0.0;
#pragma unroll
    for (int m = 0; m < V; m++) mx = fmax(fabs(lam[m]), mx);
    if constexpr (is_viscous<PDE>::value) {
      PDE::template viscous_eigenvalues<DIM>(q, d, lam);
      double mv = 0.0;
#pragma unroll
      for (int m = 0; m < V; m++) mv = fmax(fabs(lam[m]), mv);
      mx += mv * (2.0 / pnpm) * invDx[d];
    } else {
      (void)pnpm;
    }
    den += mx * invDx[d];
  }
  return den;
}

// the size along direction d of cell c's cells (its grid's, or the uniform one)
__device__ __forceinline__ double face_size(const FaceArgs& f, long c, int d) {
  const int g = f.cell_grid ? f.cell_grid[c] : 0;
  return f.grid_dx ? f.grid_dx[g * 3 + d] : f.u_dx[d];
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
  rusanov_face<PDE, DIM, N, P>(QL, QR, FL, FR, d, lane, false, false, BuiltinGhost<PDE, DIM, N, P>{d, d},
                               is_viscous<PDE>::value ? face_size(f, cl, d) : 1.0);
}

// Rusanov on interior faces with bulk copies: persistent warps (8 per CTA), each walking faces
// w, w + W, ... (W warps in the grid); a face's four trace blocks (QL, QR: nf*D doubles; FL, FR: nf*V)
// arrive in the warp's own shared-memory buffer by bulk copy -- the next face's while the current
// one is solved, two buffers per warp -- and FL, FR leave by bulk store. For trace blocks whose
// sizes are multiples of 16 bytes (RiemannBulk::ok) and 16-byte aligned arrays.
template <class PDE, int DIM, int N, int P>
struct RiemannBulk {
  using S = Shape<PDE, DIM, N, P>;
  static constexpr int nQ = S::nf * S::D, nF = S::nf * S::V;
  static constexpr int face = 2 * nQ + 2 * nF;                    // doubles of one face
  static constexpr int WPB = 8;                                   // warps per CTA
  static constexpr size_t smem = sizeof(double) * (size_t)(2 * WPB * face);
  static constexpr bool ok = nQ % 2 == 0 && nF % 2 == 0 && smem <= 200 * 1024;
};
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) riemann_bulk_kernel(FaceArgs f) {
  using S = Shape<PDE, DIM, N, P>;
  using R = RiemannBulk<PDE, DIM, N, P>;
  extern __shared__ __align__(128) double smem[];
  __shared__ __align__(8) uint64_t s_bar[R::WPB][2];
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int warps = gridDim.x * R::WPB;
  double* base = smem + (size_t)wl * 2 * R::face;
  auto issue = [&](int fc, int b) {  // lane 0: the face's four blocks into buffer b
    const int d = f.dir[fc];
    const long cl = f.left[fc], cr = f.right[fc];
    double* st = base + (size_t)b * R::face;
    mbar_arrive_expect_tx(&s_bar[wl][b], (2 * R::nQ + 2 * R::nF) * 8);
    bulk_g2s(st, f.lQhbnd + cl * S::sizeQhb + (2 * d + 1) * R::nQ, R::nQ * 8, &s_bar[wl][b]);
    bulk_g2s(st + R::nQ, f.lQhbnd + cr * S::sizeQhb + (2 * d) * R::nQ, R::nQ * 8, &s_bar[wl][b]);
    bulk_g2s(st + 2 * R::nQ, f.lFhbnd + cl * S::sizeFhb + (2 * d + 1) * R::nF, R::nF * 8, &s_bar[wl][b]);
    bulk_g2s(st + 2 * R::nQ + R::nF, f.lFhbnd + cr * S::sizeFhb + (2 * d) * R::nF, R::nF * 8, &s_bar[wl][b]);
  };
  const int w0 = blockIdx.x * R::WPB + wl;
  if (lane == 0) {
    mbar_init(&s_bar[wl][0], 1);
    mbar_init(&s_bar[wl][1], 1);
    fence_mbar_init();
    if (w0 < f.nfaces) issue(w0, 0);
  }
  __syncwarp();
  int stall = -1;
  for (int it = 0;; it++) {
    const int fc = w0 + it * warps;
    if (fc >= f.nfaces) break;
    const int b = it & 1;
    const bool to = !mbar_wait_bounded(&s_bar[wl][b], (it >> 1) & 1, kBulkWaitLimitNs);
    if (__any_sync(0xffffffffu, to)) {
      if (lane == 0 && f.status) atomicOr(f.status, ST_TIMEOUT);
      stall = b | (((it >> 1) & 1) << 1);
      break;
    }
    if (lane == 0 && fc + warps < f.nfaces) {
      bulk_wait_read_all();  // the other buffer's bulk stores have read it
      issue(fc + warps, b ^ 1);
    }
    double* st = base + (size_t)b * R::face;
    const int d = f.dir[fc];
    rusanov_face<PDE, DIM, N, P>(st, st + R::nQ, st + 2 * R::nQ, st + 2 * R::nQ + R::nF, d, lane, false, false,
                                 BuiltinGhost<PDE, DIM, N, P>{d, d},
                                 is_viscous<PDE>::value ? face_size(f, f.left[fc], d) : 1.0);
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      const long cl = f.left[fc], cr = f.right[fc];
      bulk_s2g(f.lFhbnd + cl * S::sizeFhb + (2 * d + 1) * R::nF, st + 2 * R::nQ, R::nF * 8);
      bulk_s2g(f.lFhbnd + cr * S::sizeFhb + (2 * d) * R::nF, st + 2 * R::nQ + R::nF, R::nF * 8);
      bulk_commit();
    }
    __syncwarp();
  }
  if (lane == 0) {
    if (stall >= 0) (void)mbar_wait_bounded(&s_bar[wl][stall & 1], (uint32_t)(stall >> 1), kBulkWaitLimitNs);
    bulk_wait_all();
  }
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
  const int type = f.btype ? f.btype[warp] : 1;
  if (has_boundary_values<PDE, DIM>::value && type == 4) {  // EXA_BC_USER
    UserGhost<PDE, DIM, N, P> gh;
    const int g = f.cell_grid ? f.cell_grid[c] : 0;
#pragma unroll
    for (int k = 0; k < 3; k++) gh.dx[k] = k < DIM ? (f.grid_dx ? f.grid_dx[g * 3 + k] : f.u_dx[k]) : 1.0;
    const double* Gg = f.grid_geo + 6 * g;
    const long long loc = c - (f.grid_first ? f.grid_first[g] : 0);
    const long long nx = (long long)Gg[3], ny = (long long)Gg[4];
    const long long ix = loc % nx, iy = (loc / nx) % ny, iz = loc / (nx * ny);
    gh.centre[0] = Gg[0] + (ix + 0.5) * gh.dx[0];
    gh.centre[1] = Gg[1] + (iy + 0.5) * gh.dx[1];
    gh.centre[2] = Gg[2] + (iz + 0.5) * gh.dx[2];
    gh.t = f.grid_t ? f.grid_t[g] : f.u_t;
    gh.dt = f.grid_dt ? f.grid_dt[g] : f.u_dt;
    gh.face = face;
    gh.d = d;
    if (o == 0)
      rusanov_face<PDE, DIM, N, P>(Q, Q, F, F, d, lane, true, false, gh, gh.dx[d]);
    else
      rusanov_face<PDE, DIM, N, P>(Q, Q, F, F, d, lane, false, true, gh, gh.dx[d]);
    return;
  }
  // EXA_BC_OUTFLOW (3): ghost = inner state; otherwise the functor's reflective wall
  const BuiltinGhost<PDE, DIM, N, P> gh{type == 3 ? -1 : d, d};
  const double fdx = is_viscous<PDE>::value ? face_size(f, c, d) : 1.0;
  if (o == 0)
    rusanov_face<PDE, DIM, N, P>(Q, Q, F, F, d, lane, true, false, gh, fdx);
  else
    rusanov_face<PDE, DIM, N, P>(Q, Q, F, F, d, lane, false, true, gh, fdx);
}

// adjustPointSolution at every node (3d/solutionAdjustment.cpph:17-58): x = cell centre +
// dx (node - 0.5) per axis, the grid's time t and step dt; in place on luh_out
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) adjust_kernel(CellArgs a) {
  if constexpr (has_adjust_point_solution<PDE, DIM>::value) {
    using S = Shape<PDE, DIM, N, P>;
    using G = GL<N>;
    constexpr int n = S::n, nd = S::nd, D = S::D;
    const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (long long)a.ncells * nd) return;
    const long long cell = k / nd;
    const int p = (int)(k % nd);
    const int g = a.cell_grid ? a.cell_grid[cell] : 0;
    double dx[3];
#pragma unroll
    for (int d = 0; d < 3; d++) dx[d] = d < DIM ? (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 1.0;
    double c[3];
    cell_centre(a, cell, g, dx, c);
    int co[3];
    node_coords<DIM, n>(p, co);
    double x[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < DIM; d++) x[d] = c[d] + dx[d] * (G::nodes(co[d]) - 0.5);
    const double t = a.grid_t ? a.grid_t[g] : a.u_t;
    const double dt = a.grid_dt ? a.grid_dt[g] : a.u_dt;
    PDE::template adjust_point_solution<DIM>(x, t, dt, a.luh_out + (size_t)k * D);
  } else {
    (void)a;
  }
}

// ------------------------------------------------------------------------------------------
// Surface integral + solution update + CFL of the new state
// ------------------------------------------------------------------------------------------
// Memory-bound: the register cap keeps enough CTAs resident to cover the loads (one 512-thread
// cell per CTA: 2 CTAs per SM; at most 6 entries per node: 6 CTAs), at the cost of a few
// spilled bytes; wider nodes in smaller CTAs keep the uncapped allocation (they would spill more).
template <class PDE, int DIM, int N, int P>
struct UpdateOcc {
  using S = Shape<PDE, DIM, N, P>;
  static constexpr int value = S::TPB >= 512 ? 2 : (S::D <= 6 ? 6 : 1);
};
template <class PDE, int DIM, int N, int P, bool SURFACE, bool UPDATE>
__global__ void __launch_bounds__(Shape<PDE, DIM, N, P>::TPB, (UpdateOcc<PDE, DIM, N, P>::value))
update_kernel(CellArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf, CPB = S::CPB;
  __shared__ double sFb[CPB * S::sizeFhb];
  __shared__ double s_w[n], s_F0[n], s_F1[n], s_min[CPB];
  const int tid = threadIdx.x;
  const bool inr = tid < CPB * nd;
  const int lc = inr ? tid / nd : 0, p = inr ? tid % nd : 0;
  const long cell = (long)a.cell_begin + (long)blockIdx.x * CPB + lc;
  const bool live = inr && cell < a.ncells;
  if (tid < n) {
    s_w[tid] = G::weights(tid);
    s_F0[tid] = G::F0(tid);
    s_F1[tid] = G::F1(tid);
  }
  if (tid < CPB) s_min[tid] = __longlong_as_double(0x7ff0000000000000ll);
  // this node's state and volume update, loaded before the face fluxes are staged so that the
  // three input streams are in flight together
  double q[D], du[UPDATE ? V : 1];
  if (live) {
    const double* luh = a.luh + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
    for (int m = 0; m < D; m++) q[m] = luh[m];
    if (UPDATE) {
      const double* lduh = a.lduh + (size_t)cell * nd * V + (size_t)p * V;
#pragma unroll
      for (int m = 0; m < (UPDATE ? V : 1); m++) du[m] = lduh[m];
    }
  }
  if (SURFACE) {
    for (int j = tid; j < CPB * S::sizeFhb; j += S::TPB) {
      const long gc = (long)a.cell_begin + (long)blockIdx.x * CPB + j / S::sizeFhb;
      sFb[j] = gc < a.ncells ? a.lFhbnd[((size_t)a.cell_begin + (size_t)blockIdx.x * CPB) * S::sizeFhb + j] : 0.0;
    }
  }
  __syncthreads();
  const int g = (live && a.cell_grid) ? a.cell_grid[cell] : 0;
  double invDx[3];
#pragma unroll
  for (int d = 0; d < 3; d++) invDx[d] = d < DIM ? 1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 0.0;
  int co[3];
  node_coords<DIM, n>(p, co);
  bool ok = true;
  if (live) {
    if (UPDATE) {
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
            du[UPDATE ? m : 0] -= (Fb[((2 * d + 1) * nf + fn) * V + m] * s_F1[k] - Fb[((2 * d) * nf + fn) * V + m] * s_F0[k]) * us;
        }
      }
      const double w_sp = DIM == 3 ? s_w[co[2]] * s_w[co[1]] * s_w[co[0]] : s_w[co[1]] * s_w[co[0]];
      const double updateSize = (a.grid_dt ? a.grid_dt[g] : a.u_dt) / w_sp;
      double* out = a.luh_out + (size_t)cell * nd * D + (size_t)p * D;
#pragma unroll
      for (int m = 0; m < V; m++) {
        q[m] = q[m] + du[UPDATE ? m : 0] * updateSize;
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
    const double den = cfl_denominator<PDE, DIM>(q, invDx, a.pnpm);
    dtp = a.cfl_pnpm / den;
    // a non-finite state gives no time step (fmax drops NaN eigenvalues, so den alone can look fine)
    bool qok = true;
#pragma unroll
    for (int m = 0; m < D; m++) qok &= finite(q[m]);
    if (!(dtp > 0.0) || !qok) {  // NaN, non-positive, or from a non-finite state
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

// Per-cell integrals of the generic-kernel interface on one cell, thread per node, in the
// reference's operation order:
//   mode 0  volumeIntegralNonlinear (3d/volumeIntegralNonlinear.cpph:133-223): lduh = sum over the
//           directions of Kxi[k][m] lFhi_d[line][m] w_a w_b / dx_d (+ w_xyz lShi with a source or
//           NCP) from the reference lFhi blocks x [z][y][x], y [z][x][y], z [y][x][z], source;
//   mode 1  surfaceIntegralNonlinear (3d/surfaceIntegralNonlinear.cpph:21-90): lduh -= the six
//           faces' terms from lFhbnd [2*DIM][face node][V];
//   mode 2  faceIntegralNonlinear (3d/faceIntegralNonlinear.cpph:21-103): lduh -= w_a w_b
//           (2 orientation - 1) / dx_d FCoeff[orientation][k] F of one face block.
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(256) cell_integral_kernel(int mode, double* lduh, const double* in, int direction,
                                                            int orientation, double dx0, double dx1, double dx2) {
  using S = Shape<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, nd = S::nd, nf = S::nf;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nd) return;
  const double dxv[3] = {dx0, dx1, dx2};
  int co[3];
  node_coords<DIM, n>(p, co);
  double* du = lduh + (size_t)p * V;
  if (mode == 0) {
    double acc[V];
#pragma unroll
    for (int m = 0; m < V; m++) acc[m] = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int L = node_line<DIM, n>(p, d);
      const double wt = DIM == 3 ? G::weights(L / n) * G::weights(L % n) : G::weights(L);
      const double us = wt * (1.0 / dxv[d]);
      const double* F = in + (size_t)d * nd * V + (size_t)L * n * V;
#pragma unroll
      for (int m = 0; m < V; m++)
#pragma unroll
        for (int mm = 0; mm < n; mm++) acc[m] += G::Kxi(co[d], mm) * F[mm * V + m] * us;
    }
    if (PDE::kNCP || PDE::kSource) {
      const double w = DIM == 3 ? G::weights(co[2]) * G::weights(co[1]) * G::weights(co[0])
                                : G::weights(co[1]) * G::weights(co[0]);
#pragma unroll
      for (int m = 0; m < V; m++) acc[m] += w * in[(size_t)DIM * nd * V + (size_t)p * V + m];
    }
#pragma unroll
    for (int m = 0; m < V; m++) du[m] = acc[m];
  } else if (mode == 1) {
#pragma unroll
    for (int d = 0; d < DIM; d++) {
      const int fn = node_line<DIM, n>(p, d);
      const double wt = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
      const double us = wt * (1.0 / dxv[d]);
      const int k = co[d];
#pragma unroll
      for (int m = 0; m < V; m++)
        du[m] -= (in[((2 * d + 1) * nf + fn) * V + m] * G::F1(k) - in[((2 * d) * nf + fn) * V + m] * G::F0(k)) * us;
    }
  } else {
    const int d = direction;
    const int fn = node_line<DIM, n>(p, d);
    const double scaling = 1.0 / dxv[d] * (2.0 * orientation - 1.0);
    const double sw = (DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn)) * scaling;
    const double fc = orientation ? G::F1(co[d]) : G::F0(co[d]);
#pragma unroll
    for (int m = 0; m < V; m++) du[m] -= sw * fc * in[fn * V + m];
  }
}

// Surface integral + solution update + CFL (update_kernel<..., true, true>) as a persistent kernel
// over cell groups: each group's luh, lduh and lFhbnd blocks (contiguous per group) arrive in shared
// memory by bulk copy -- the next group's while the current one is computed, two buffers -- and the
// new luh block leaves by one bulk store. For blocks whose sizes are multiples of 16 bytes
// (UpdateBulk::ok) and 16-byte aligned arrays; the launcher falls back to update_kernel otherwise.
template <class PDE, int DIM, int N, int P>
struct UpdateBulk {
  using S = Shape<PDE, DIM, N, P>;
  static constexpr int nL = S::CPB * S::nd * S::D, nU = S::CPB * S::nd * S::V, nF = S::CPB * S::sizeFhb;
  static constexpr int stage = nL + nU + nF;                         // doubles of one buffer
  static constexpr size_t smem = 2 * sizeof(double) * (size_t)stage;
  static constexpr bool ok =
      (S::nd * S::D) % 2 == 0 && (S::nd * S::V) % 2 == 0 && S::sizeFhb % 2 == 0 && smem <= 200 * 1024;
};
template <class PDE, int DIM, int N, int P>
__global__ void __launch_bounds__(Shape<PDE, DIM, N, P>::TPB) update_bulk_kernel(CellArgs a) {
  using S = Shape<PDE, DIM, N, P>;
  using B = UpdateBulk<PDE, DIM, N, P>;
  using G = GL<N>;
  constexpr int n = S::n, V = S::V, D = S::D, nd = S::nd, nf = S::nf, CPB = S::CPB;
  extern __shared__ __align__(128) double smem[];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ double s_min[CPB];
  const int tid = threadIdx.x;
  const bool inr = tid < CPB * nd;
  const int lc = inr ? tid / nd : 0, p = inr ? tid % nd : 0;
  const int ngroups = (a.ncells - a.cell_begin + CPB - 1) / CPB;
  auto live_cells = [&](int g) { return min(CPB, a.ncells - (a.cell_begin + g * CPB)); };
  auto issue = [&](int g, int b) {  // thread 0: the group's three blocks into buffer b
    const size_t c0 = (size_t)a.cell_begin + (size_t)g * CPB;
    const int nl = live_cells(g);
    double* st = smem + (size_t)b * B::stage;
    const uint32_t bl = nl * nd * D * 8, bu = nl * nd * V * 8, bf = nl * S::sizeFhb * 8;
    mbar_arrive_expect_tx(&s_bar[b], bl + bu + bf);
    bulk_g2s(st, a.luh + c0 * nd * D, bl, &s_bar[b]);
    bulk_g2s(st + B::nL, a.lduh + c0 * nd * V, bu, &s_bar[b]);
    bulk_g2s(st + B::nL + B::nU, a.lFhbnd + c0 * S::sizeFhb, bf, &s_bar[b]);
  };
  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
  }
  // per-cell CFL minima; from then on the thread that reads a cell's minimum resets it, so that
  // every reset is ordered before the next group's additions by the barrier that ends a group
  if (tid < CPB) s_min[tid] = __longlong_as_double(0x7ff0000000000000ll);
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < ngroups) issue(blockIdx.x, 0);
  int co[3];
  node_coords<DIM, n>(p, co);
  const double w_sp = DIM == 3 ? G::weights(co[2]) * G::weights(co[1]) * G::weights(co[0])
                               : G::weights(co[1]) * G::weights(co[0]);
  int stall = -1;
  for (int it = 0;; it++) {
    const int grp = blockIdx.x + it * gridDim.x;
    if (grp >= ngroups) break;
    const int b = it & 1;
    const bool to = !mbar_wait_bounded(&s_bar[b], (it >> 1) & 1, kBulkWaitLimitNs);
    if (__syncthreads_or(to)) {
      if (tid == 0 && a.status) atomicOr(a.status, ST_TIMEOUT);
      stall = b | (((it >> 1) & 1) << 1);
      break;
    }
    if (tid == 0 && grp + (int)gridDim.x < ngroups) {
      // the other buffer's last bulk store (group it - 1) must have read it before it is refilled
      bulk_wait_read_all();
      issue(grp + gridDim.x, b ^ 1);
    }
    double* st = smem + (size_t)b * B::stage;
    const int cell = a.cell_begin + grp * CPB + lc;
    const bool live = inr && cell < a.ncells;
    const int g = (live && a.cell_grid) ? a.cell_grid[cell] : 0;
    double invDx[3];
#pragma unroll
    for (int d = 0; d < 3; d++) invDx[d] = d < DIM ? 1.0 / (a.grid_dx ? a.grid_dx[g * 3 + d] : a.u_dx[d]) : 0.0;
    double* q = st + ((size_t)lc * nd + p) * D;
    double qv[D];
    bool ok = true;
    if (live) {
      const double* du = st + B::nL + ((size_t)lc * nd + p) * V;
      const double* Fb = st + B::nL + B::nU + (size_t)lc * S::sizeFhb;
      double dv[V];
#pragma unroll
      for (int m = 0; m < V; m++) dv[m] = du[m];
#pragma unroll
      for (int d = 0; d < DIM; d++) {
        const int fn = node_line<DIM, n>(p, d);
        const double wt = DIM == 3 ? G::weights(fn / n) * G::weights(fn % n) : G::weights(fn);
        const double us = wt * invDx[d];
        const int k = co[d];
#pragma unroll
        for (int m = 0; m < V; m++)
          dv[m] -= (Fb[((2 * d + 1) * nf + fn) * V + m] * G::F1(k) - Fb[((2 * d) * nf + fn) * V + m] * G::F0(k)) * us;
      }
      const double updateSize = (a.grid_dt ? a.grid_dt[g] : a.u_dt) / w_sp;
#pragma unroll
      for (int m = 0; m < D; m++) qv[m] = q[m];
#pragma unroll
      for (int m = 0; m < V; m++) {
        qv[m] = qv[m] + dv[m] * updateSize;
        ok &= finite(qv[m]);
        q[m] = qv[m];
      }
    }
    // CFL of the new state (stableTimeStepSize :14-62)
    double dtp = __longlong_as_double(0x7ff0000000000000ll);
    if (live && (a.grid_dt_next || a.cell_dt)) {
      const double den = cfl_denominator<PDE, DIM>(qv, invDx, a.pnpm);
      dtp = a.cfl_pnpm / den;
      bool qok = true;
#pragma unroll
      for (int m = 0; m < D; m++) qok &= finite(qv[m]);
      if (!(dtp > 0.0) || !qok) {
        if (a.status) atomicOr(a.status, ST_BAD_DT);
        dtp = __longlong_as_double(0x7ff0000000000000ll);
      }
    }
    if (live && !ok && a.status) atomicOr(a.status, ST_NONFINITE_UPDATE);
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
    // the new luh block is complete in shared memory: one bulk store (thread 0)
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      const size_t c0 = (size_t)a.cell_begin + (size_t)grp * CPB;
      bulk_s2g(a.luh_out + c0 * nd * D, st, live_cells(grp) * nd * D * 8);
      bulk_commit();
    }
    if (p == 0 && live) {
      const double mn = s_min[lc];
      s_min[lc] = __longlong_as_double(0x7ff0000000000000ll);
      if (a.cell_dt) a.cell_dt[cell] = mn;
      if (a.grid_dt_next) atomic_min_pos(&a.grid_dt_next[g], mn);
    }
    // s_min is reused by the next group, this buffer two groups on
    __syncthreads();
  }
  if (tid == 0) {
    if (stall >= 0) (void)mbar_wait_bounded(&s_bar[stall & 1], (uint32_t)(stall >> 1), kBulkWaitLimitNs);
    bulk_wait_all();
  }
}

// t += dt, dt = dt_next, dt_next = +inf for every grid (one thread per grid).
// dt_next == nullptr: a fixed time step, dt stays as it is
__global__ void advance_kernel(int ngrids, double* t, double* dt, double* dt_next, long long* steps) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ngrids) return;
  t[g] += dt[g];
  if (dt_next) {
    dt[g] = dt_next[g];
    dt_next[g] = __longlong_as_double(0x7ff0000000000000ll);
  }
  if (g == 0 && steps) steps[0] += 1;
}

__global__ void fill_kernel(int count, double* x, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) x[i] = v;
}

}  // namespace exa
