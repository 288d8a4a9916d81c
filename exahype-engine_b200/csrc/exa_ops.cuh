// Launchers of every kernel of one PDE instantiation (PDE functor, DIM, order N, nPar P), behind
// the virtual interface the C ABI (exa_aderdg.cu) dispatches through. The library instantiates
// OpsImpl for its built-in functors; an application instantiates it for its own functor through
// include/exa_aderdg_user.cuh and registers the object with exa_register_pde.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "exa_kernels.cuh"
#include "exa_adjoint.cuh"
#include "exa_amr.cuh"

namespace exa {

// One instantiation (PDE, DIM, N, P): launchers of every kernel.
struct Ops {
  // layout version of this interface: an application library compiled against another layout is
  // refused by exa_register_pde (its object would be read with the wrong offsets)
  static constexpr int kAbi = 7;
  int abi = kAbi;
  int dim, order, nvar, npar, nd, nf, cpb;
  size_t sz_luh, sz_lduh, sz_qhb, sz_fhb, sz_lQi, sz_lFi, sz_lQhi, sz_lFhi;
  bool ncp;
  bool viscous = false;  // the flux depends on the gradient (useViscousFlux)
  bool alg_source = false;  // the functor has an algebraic source (useSource): needs cell positions
  virtual ~Ops() {}
  bool mixed_ok = false;  // mixed-precision predictor instantiated
  // Riemann launch form for all solvers of this instantiation: 0 riemann_kernel, otherwise
  // riemann_bulk_kernel where the trace blocks allow it (exa_solver_set_update_variant sets it)
  int riemann_variant = -1;
  // variant: 0 one cell group per CTA, 1 persistent CTAs with a prefetched next group, -1 the
  // variant tune() measured as faster on this device (0 until tuned)
  virtual cudaError_t predictor(const CellArgs& a, cudaStream_t st, bool mixed, int variant) = 0;
  // times every predictor variant on (up to kTuneCells of) the given cells and keeps the faster
  // one for this device; the launch writes the predictor outputs of those cells. Not during capture.
  virtual cudaError_t tune(const CellArgs& a, cudaStream_t st, bool mixed) = 0;
  virtual int tuned_variant(bool mixed) = 0;
  // device scratch the predictor needs for a launch over ncells (outside stream capture)
  virtual cudaError_t reserve(long long ncells) = 0;
  // variant (surface + update only): 0 update_kernel; 1 update_bulk_kernel (persistent, bulk copies),
  // where the block sizes and the arrays' alignment allow it; -1 the latter where possible
  virtual cudaError_t update(const CellArgs& a, bool surface, bool upd, cudaStream_t st, int variant = -1) = 0;
  virtual cudaError_t riemann(const FaceArgs& f, cudaStream_t st) = 0;
  virtual cudaError_t boundary(const FaceArgs& f, cudaStream_t st) = 0;
  // discrete adjoint of one step (linear systems only)
  bool adjoint_ok = false;
  virtual cudaError_t adjoint(const AdjArgs& a, cudaStream_t st) = 0;
  // optional functor hooks: adjust_point_solution (device initial conditions) and boundary_values
  // (faces of type EXA_BC_USER)
  bool adjust_ok = false, user_bc_ok = false;
  virtual cudaError_t adjust(const CellArgs& a, cudaStream_t st) = 0;
  // the point source's slot table: slot[cell] (-1 off the source), cells[slot], *count slots
  // (count zeroed by the caller); the FP64 predictor then reads the values source_values_kernel
  // evaluates ahead of it
  virtual cudaError_t source_slots(const CellArgs& a, int* slot, int* cells, int* count, cudaStream_t st) = 0;
  // per-cell volume (mode 0), surface (1) and face (2) integrals of one cell (cell_integral_kernel)
  virtual cudaError_t cell_integral(int mode, double* lduh, const double* in, int direction, int orientation,
                                    const double* dx, cudaStream_t st) = 0;
  // mesh levels: volume (face = false: luh blocks) or face (lQhbnd and lFhbnd blocks) unknowns,
  // prolongation / restriction / flux-only restriction (AmrArgs::mode)
  virtual cudaError_t amr(const AmrArgs& a, bool face, cudaStream_t st) = 0;
  // limiter cell kernels (LimArgs::op)
  virtual cudaError_t limiter(const LimArgs& a, cudaStream_t st) = 0;
};

template <class PDE, int DIM, int N, int P>
struct OpsImpl final : Ops {
  using S = Shape<PDE, DIM, N, P>;
  bool smem_set = false;
  // cells whose space-time state does not fit a CTA run the streamed predictor
  static constexpr bool kStreamed = S::predictor_smem + 4096 > 227 * 1024;
  // the mixed form needs PDEs without NCP and its larger shared-memory footprint must fit a CTA
  static constexpr bool kMixed = !kStreamed && !PDE::kNCP && !is_viscous<PDE>::value &&
                                 !has_algebraic_source<PDE, DIM>::value &&
                                 MixShape<PDE, DIM, N, P>::smem_for(2) + 4096 <= 227 * 1024;
  static constexpr bool kAdj = PDE::kAdjoint && !PDE::kNCP && !is_viscous<PDE>::value &&
                               !has_algebraic_source<PDE, DIM>::value &&
                               AdjShape<PDE, DIM, N, P>::smem <= 227 * 1024;
  // streamed predictor: scratch per device, grown on demand
  std::mutex scratch_mu;
  double* scratch[64] = {};
  size_t scratch_slots[64] = {};
  int stream_grid[64] = {};
  cudaError_t reserve(long long ncells) override {
    if constexpr (kStreamed) {
      using T = StreamShape<PDE, DIM, N, P>;
      static_assert(T::smem + 4096 <= 227 * 1024, "streamed predictor shared memory exceeds one CTA");
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e != cudaSuccess) return e;
      if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
      std::lock_guard<std::mutex> lk(scratch_mu);
      if (!smem_set) {
        e = cudaFuncSetAttribute(predictor_streamed_kernel<PDE, DIM, N, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)T::smem);
        if (e != cudaSuccess) return e;
        smem_set = true;
      }
      int sms = 0, occ = 0;
      if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, predictor_streamed_kernel<PDE, DIM, N, P>, T::TPB,
                                                             T::smem)) != cudaSuccess)
        return e;
      const long long want = std::max(1LL, std::min<long long>(ncells, (long long)sms * std::max(occ, 1)));
      if ((size_t)want > scratch_slots[dev]) {
        if (scratch[dev]) cudaFree(scratch[dev]);
        scratch[dev] = nullptr;
        scratch_slots[dev] = 0;
        e = cudaMalloc(&scratch[dev], (size_t)want * T::slot_doubles * sizeof(double));
        if (e != cudaSuccess) return e;
        scratch_slots[dev] = (size_t)want;
      }
      stream_grid[dev] = (int)scratch_slots[dev];
    } else {
      (void)ncells;
    }
    return cudaSuccess;
  }
  // resident CTAs of the persistent predictor per device (FP64 form [0])
  int pred_grid[2][64] = {};
  bool pred_attr[2][2] = {};  // dynamic shared memory set: [FP64, mixed][variant]
  // measured variant per device and form: 0 untuned, 1 + the variant otherwise
  int pred_tuned[2][64] = {};
  // FP64 form: PERSIST selects the persistent grid with a prefetched next group
  template <bool PERSIST>
  cudaError_t launch_predictor(const CellArgs& a, cudaStream_t st) {
    static_assert(!kStreamed, "cells of this size run the streamed predictor");
    static_assert(S::predictor_smem_persist + 4096 <= 227 * 1024, "predictor shared memory exceeds one CTA");
    const size_t smem = PERSIST ? S::predictor_smem_persist : S::predictor_smem;
    auto kern = predictor_kernel<PDE, DIM, N, P, PERSIST>;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!pred_attr[0][PERSIST ? 1 : 0]) {
      e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      pred_attr[0][PERSIST ? 1 : 0] = true;
    }
    const long long groups = ((long long)a.ncells - a.cell_begin + S::CPB - 1) / S::CPB;
    long long blocks = groups;
    if (PERSIST) {
      // persistent CTAs, one group of CPB cells after another; each fetches its next group's luh
      // with a bulk copy while it computes the current one (16-byte aligned blocks only)
      int& grid = pred_grid[0][dev];
      if (grid == 0) {
        int sms = 0, occ = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, S::TPB, smem)) != cudaSuccess) return e;
        grid = sms * std::max(occ, 1);
      }
      blocks = std::min<long long>(groups, grid);
    }
    if constexpr (PDE::kSource) {
      // the point source's values at the slot cells' nodes, ahead of the predictor that reads them
      if (a.src && a.src_slot && a.nsrc > 0) {
        constexpr int tpb = S::nd >= 256 ? 256 : (S::nd + 31) / 32 * 32;
        source_values_kernel<PDE, DIM, N, P><<<(unsigned)a.nsrc, tpb, 0, st>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
    }
    CellArgs b = a;
    b.bulk_luh = (reinterpret_cast<uintptr_t>(a.luh) % 16 == 0) && ((S::nd * S::D) % 2 == 0);
    kern<<<(unsigned)blocks, S::TPB, smem, st>>>(b);
    return cudaGetLastError();
  }
  // mixed form: OCC resident CTAs per SM (the register budget of the instantiation)
  template <int OCC>
  cudaError_t launch_mixed(const CellArgs& a, cudaStream_t st) {
    if constexpr (!kMixed) {
      (void)a, (void)st;
      return cudaErrorNotSupported;
    } else {
      using MS = MixShape<PDE, DIM, N, P>;
      auto kern = predictor_mixed_kernel<PDE, DIM, N, P, OCC>;
      if (!pred_attr[1][OCC == 3 ? 1 : 0]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MS::smem_for(OCC));
        if (e != cudaSuccess) return e;
        pred_attr[1][OCC == 3 ? 1 : 0] = true;
      }
      const unsigned blocks = (unsigned)(((long long)a.ncells - a.cell_begin + S::CPB - 1) / S::CPB);
      kern<<<blocks, S::TPB, MS::smem_for(OCC), st>>>(a);
      return cudaGetLastError();
    }
  }
  template <bool M>
  cudaError_t launch_variant(const CellArgs& a, cudaStream_t st, int v) {
    if constexpr (M) {
      return v == 1 ? launch_mixed<3>(a, st) : launch_mixed<2>(a, st);
    } else {
      return v == 1 ? launch_predictor<true>(a, st) : launch_predictor<false>(a, st);
    }
  }
  int tuned_variant(bool mixed) override {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    const int t = pred_tuned[mixed && kMixed ? 1 : 0][dev];
    return t > 0 ? t - 1 : 0;
  }
  cudaError_t tune(const CellArgs& a, cudaStream_t st, bool mixed) override {
    if constexpr (kStreamed) {
      (void)a, (void)st, (void)mixed;
      return cudaSuccess;
    } else {
      if (mixed && !kMixed) return cudaErrorNotSupported;
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e != cudaSuccess) return e;
      if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
      int& slot = pred_tuned[mixed ? 1 : 0][dev];
      if (slot > 0) return cudaSuccess;
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if ((e = cudaStreamIsCapturing(st, &cs)) != cudaSuccess) return e;
      if (cs != cudaStreamCaptureStatusNone) return cudaSuccess;
      // enough cells that every CTA of the persistent grid walks several groups
      constexpr long long kTuneCells = 65536;
      CellArgs b = a;
      b.ncells = (int)std::min<long long>(a.ncells, (long long)a.cell_begin + kTuneCells);
      if (b.ncells <= b.cell_begin) return cudaSuccess;
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if ((e = cudaEventCreate(&e0)) != cudaSuccess) return e;
      if ((e = cudaEventCreate(&e1)) != cudaSuccess) {
        cudaEventDestroy(e0);
        return e;
      }
      // one untimed launch of each form (first-use costs), then three interleaved rounds; the best
      // time of each form counts, and the second form must win by 3% to replace the first
      float best[2] = {1e30f, 1e30f};
      for (int v = 0; v < 2 && e == cudaSuccess; v++) e = mixed ? launch_variant<true>(b, st, v) : launch_variant<false>(b, st, v);
      for (int round = 0; round < 3 && e == cudaSuccess; round++)
        for (int v = 0; v < 2 && e == cudaSuccess; v++) {
          e = cudaEventRecord(e0, st);
          if (e == cudaSuccess) e = mixed ? launch_variant<true>(b, st, v) : launch_variant<false>(b, st, v);
          if (e == cudaSuccess) e = cudaEventRecord(e1, st);
          if (e == cudaSuccess) e = cudaEventSynchronize(e1);
          float ms = 0.0f;
          if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
          if (e == cudaSuccess) best[v] = std::min(best[v], ms);
        }
      const int best_v = best[1] < 0.97f * best[0] ? 1 : 0;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (e == cudaSuccess) slot = best_v + 1;
      return e;
    }
  }
  bool adj_smem_set = false;
  cudaError_t adjoint(const AdjArgs& a, cudaStream_t st) override {
    if constexpr (kAdj) {
      using A = AdjShape<PDE, DIM, N, P>;
      static_assert(A::smem <= 227 * 1024, "adjoint shared memory exceeds one CTA");
      if (a.f.nfaces > 0) {
        adjoint_face_kernel<PDE, DIM, N, P><<<(unsigned)((a.f.nfaces + 7) / 8), 256, 0, st>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
      }
      if (a.fb.nfaces > 0) {
        adjoint_boundary_kernel<PDE, DIM, N, P><<<(unsigned)((a.fb.nfaces + 7) / 8), 256, 0, st>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
      }
      if (a.c.ncells <= 0) return cudaSuccess;
      if (!adj_smem_set) {
        cudaError_t e = cudaFuncSetAttribute(adjoint_predictor_kernel<PDE, DIM, N, P>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)A::smem);
        if (e != cudaSuccess) return e;
        adj_smem_set = true;
      }
      adjoint_predictor_kernel<PDE, DIM, N, P><<<(unsigned)a.c.ncells, A::TPB, A::smem, st>>>(a);
      return cudaGetLastError();
    } else {
      (void)a;
      (void)st;
      return cudaErrorNotSupported;
    }
  }
  cudaError_t amr(const AmrArgs& a, bool face, cudaStream_t st) override {
    if (a.ngroups <= 0) return cudaSuccess;
    if (face) {
      if constexpr (DIM > 1) {
        using Sh = AmrShape<N, DIM - 1, S::D>;
        amr_kernel<N, DIM - 1, S::D, S::V, true><<<a.ngroups, 256, Sh::smem, st>>>(a);
      }
    } else {
      using Sh = AmrShape<N, DIM, S::D>;
      static_assert(Sh::smem <= 227 * 1024, "mesh-level kernel shared memory exceeds one CTA");
      if (!amr_attr) {
        cudaError_t e = cudaFuncSetAttribute(amr_kernel<N, DIM, S::D, S::V, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Sh::smem);
        if (e != cudaSuccess) return e;
        amr_attr = true;
      }
      amr_kernel<N, DIM, S::D, S::V, false><<<a.ngroups, 256, Sh::smem, st>>>(a);
    }
    return cudaGetLastError();
  }
  bool lim_attr = false, amr_attr = false, lim_mm_attr = false;
  cudaError_t limiter(const LimArgs& a, cudaStream_t st) override {
    using L = LimShape<N, DIM, S::D>;
    static_assert(L::smem <= 227 * 1024, "limiter shared memory exceeds one CTA");
    if (a.ncells <= 0) return cudaSuccess;
    if (!lim_attr) {
      cudaError_t e = cudaFuncSetAttribute(limiter_kernel<N, DIM, S::D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)L::smem);
      if (e != cudaSuccess) return e;
      lim_attr = true;
    }
    if (a.op >= 2) {
      using M = LimMinMaxShape<N, DIM, S::D>;
      static_assert(M::smem <= 227 * 1024, "limiter min / max shared memory exceeds one CTA");
      if (!lim_mm_attr) {
        cudaError_t e = cudaFuncSetAttribute(limiter_minmax_kernel<N, DIM, S::D>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)M::smem);
        if (e != cudaSuccess) return e;
        lim_mm_attr = true;
      }
      limiter_minmax_kernel<N, DIM, S::D><<<a.ncells, 32 * M::WPC, M::smem, st>>>(a);
    } else {
      limiter_kernel<N, DIM, S::D><<<a.ncells, 256, L::smem, st>>>(a);
    }
    return cudaGetLastError();
  }
  cudaError_t cell_integral(int mode, double* lduh, const double* in, int direction, int orientation,
                            const double* dx, cudaStream_t st) override {
    cell_integral_kernel<PDE, DIM, N, P><<<(S::nd + 255) / 256, 256, 0, st>>>(
        mode, lduh, in, direction, orientation, dx[0], DIM > 1 ? dx[1] : 1.0, DIM > 2 ? dx[2] : 1.0);
    return cudaGetLastError();
  }
  cudaError_t adjust(const CellArgs& a, cudaStream_t st) override {
    if constexpr (has_adjust_point_solution<PDE, DIM>::value) {
      const long long nodes = (long long)a.ncells * S::nd;
      if (nodes <= 0) return cudaSuccess;
      adjust_kernel<PDE, DIM, N, P><<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(a);
      return cudaGetLastError();
    } else {
      (void)a, (void)st;
      return cudaErrorNotSupported;
    }
  }
  cudaError_t source_slots(const CellArgs& a, int* slot, int* cells, int* count, cudaStream_t st) override {
    if (a.ncells <= 0) return cudaSuccess;
    source_slot_kernel<PDE, DIM, N, P><<<(unsigned)((a.ncells + 255) / 256), 256, 0, st>>>(a, slot, cells, count);
    return cudaGetLastError();
  }
  OpsImpl() {
    adjoint_ok = kAdj;
    mixed_ok = kMixed;
    viscous = is_viscous<PDE>::value;
    alg_source = has_algebraic_source<PDE, DIM>::value;
    adjust_ok = has_adjust_point_solution<PDE, DIM>::value;
    user_bc_ok = has_boundary_values<PDE, DIM>::value;
    dim = DIM;
    order = N;
    nvar = S::V;
    npar = P;
    nd = S::nd;
    nf = S::nf;
    cpb = S::CPB;
    ncp = PDE::kNCP;
    sz_luh = (size_t)S::nd * S::D;
    sz_lduh = (size_t)S::nd * S::V;
    sz_qhb = S::sizeQhb;
    sz_fhb = S::sizeFhb;
    sz_lQi = (size_t)S::nd * S::n * S::D;
    sz_lFi = (size_t)S::n * S::nd * (DIM + 1) * S::V;
    sz_lQhi = (size_t)S::nd * S::D;
    sz_lFhi = (size_t)(DIM + 1) * S::nd * S::V;
  }
  cudaError_t predictor(const CellArgs& a, cudaStream_t st, bool mixed, int variant) override {
    if (a.ncells <= a.cell_begin) return cudaSuccess;
    if constexpr (kStreamed) {
      using T = StreamShape<PDE, DIM, N, P>;
      if (mixed) return cudaErrorNotSupported;
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e != cudaSuccess) return e;
      if (dev < 0 || dev >= 64 || !scratch[dev]) return cudaErrorNotReady;  // reserve() first
      CellArgs b = a;
      b.scratch = scratch[dev];
      const unsigned blocks = (unsigned)std::min<long long>(a.ncells - a.cell_begin, stream_grid[dev]);
      predictor_streamed_kernel<PDE, DIM, N, P><<<blocks, T::TPB, T::smem, st>>>(b);
      return cudaGetLastError();
    }
    const int v = variant >= 0 ? variant : tuned_variant(mixed);
    if (mixed) {
      if constexpr (!kMixed) {
        return cudaErrorNotSupported;
      } else {
        return launch_variant<true>(a, st, v);
      }
    }
    if constexpr (!kStreamed) return launch_variant<false>(a, st, v);
    return cudaErrorNotSupported;
  }
  int upd_grid[64] = {};
  bool upd_bulk_attr = false;
  cudaError_t update(const CellArgs& a, bool surface, bool upd, cudaStream_t st, int variant) override {
    if (a.ncells <= a.cell_begin) return cudaSuccess;
    using UB = UpdateBulk<PDE, DIM, N, P>;
    auto al = [](const void* q) { return reinterpret_cast<uintptr_t>(q) % 16 == 0; };
    if constexpr (UB::ok) {
      if (surface && upd && variant != 0 && al(a.luh) && al(a.luh_out) && al(a.lduh) && al(a.lFhbnd)) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
        auto kern = update_bulk_kernel<PDE, DIM, N, P>;
        if (!upd_bulk_attr) {
          if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)UB::smem)) !=
              cudaSuccess)
            return e;
          upd_bulk_attr = true;
        }
        if (upd_grid[dev] == 0) {
          int sms = 0, occ = 0;
          if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
          if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, S::TPB, UB::smem)) != cudaSuccess) return e;
          upd_grid[dev] = sms * std::max(occ, 1);
        }
        const long long groups = ((long long)a.ncells - a.cell_begin + S::CPB - 1) / S::CPB;
        kern<<<(unsigned)std::min<long long>(groups, upd_grid[dev]), S::TPB, UB::smem, st>>>(a);
        return cudaGetLastError();
      }
    }
    const unsigned blocks = (unsigned)((a.ncells - a.cell_begin + S::CPB - 1) / S::CPB);
    if (surface && upd)
      update_kernel<PDE, DIM, N, P, true, true><<<blocks, S::TPB, 0, st>>>(a);
    else if (upd)
      update_kernel<PDE, DIM, N, P, false, true><<<blocks, S::TPB, 0, st>>>(a);
    else
      update_kernel<PDE, DIM, N, P, false, false><<<blocks, S::TPB, 0, st>>>(a);
    return cudaGetLastError();
  }
  int rie_grid[64] = {};
  bool rie_bulk_attr = false;
  cudaError_t riemann(const FaceArgs& f, cudaStream_t st) override {
    if (f.nfaces <= 0) return cudaSuccess;
    using RB = RiemannBulk<PDE, DIM, N, P>;
    auto al = [](const void* q) { return reinterpret_cast<uintptr_t>(q) % 16 == 0; };
    if constexpr (RB::ok) {
      if (riemann_variant != 0 && al(f.lQhbnd) && al(f.lFhbnd)) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
        auto kern = riemann_bulk_kernel<PDE, DIM, N, P>;
        if (!rie_bulk_attr) {
          if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RB::smem)) !=
              cudaSuccess)
            return e;
          rie_bulk_attr = true;
        }
        if (rie_grid[dev] == 0) {
          int sms = 0, occ = 0;
          if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
          if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * RB::WPB, RB::smem)) != cudaSuccess)
            return e;
          rie_grid[dev] = sms * std::max(occ, 1);
        }
        const long long ctas = ((long long)f.nfaces + RB::WPB - 1) / RB::WPB;
        kern<<<(unsigned)std::min<long long>(ctas, rie_grid[dev]), 32 * RB::WPB, RB::smem, st>>>(f);
        return cudaGetLastError();
      }
    }
    const unsigned blocks = (unsigned)((f.nfaces + 7) / 8);
    riemann_kernel<PDE, DIM, N, P><<<blocks, 256, 0, st>>>(f);
    return cudaGetLastError();
  }
  cudaError_t boundary(const FaceArgs& f, cudaStream_t st) override {
    if (f.nfaces <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((f.nfaces + 7) / 8);
    boundary_kernel<PDE, DIM, N, P><<<blocks, 256, 0, st>>>(f);
    return cudaGetLastError();
  }
};

}  // namespace exa
