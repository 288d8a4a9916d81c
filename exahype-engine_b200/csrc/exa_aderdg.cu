// Host runtime and C ABI of the B200 ADER-DG cell update (include/exa_aderdg.h).
//
// One shared library, libexa_aderdg.so, compiled for sm_100a. The PDE functors, dimensions and
// orders are template instantiations registered in find_ops(); the C ABI dispatches to them
// through the Ops interface. Everything device-side lives in exa_kernels.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/exa_aderdg.h"
#include "exa_ops.cuh"
#include "exa_checkpoint.h"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return EXA_ERR_CUDA;
}
#define EXA_CUDA(call)                                      \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);     \
  } while (0)

// ADER-DG PNPM table by order (Toolkit/exahype/toolkit/solverController.py:17-23)
// cell chunks of a host-buffer step (exa_patch_step_host)
constexpr int kHostChunks = 32;

double default_pnpm(int order) {
  static const double t[10] = {1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015};
  if (order < 10) return t[order];
  static const double c[6] = {0.18525, 0.1204125, 0.078268125, 0.05087428125, 0.0330682828125, 0.021494383828125};
  if (order < 16) return c[order - 10] / (2 * order + 1);
  return 0.0;
}

}  // namespace

namespace exa {

// The instantiations this library carries: one function-local static launcher object each
// (constructed on first use, never on the heap; shared by every solver handle).
// instantiations registered by applications (exa_register_pde), ids >= EXA_PDE_USER_BASE
struct UserOps {
  int pde, dim, order, npar;
  Ops* ops;
};
std::mutex& user_mu() {
  static std::mutex m;
  return m;
}
std::vector<UserOps>& user_ops() {
  static std::vector<UserOps> v;
  return v;
}

Ops* find_ops(int pde, int dim, int order, int npar) {
  if (pde >= EXA_PDE_USER_BASE) {
    std::lock_guard<std::mutex> lk(user_mu());
    for (const UserOps& u : user_ops())
      if (u.pde == pde && u.dim == dim && u.order == order && u.npar == npar) return u.ops;
    return nullptr;
  }
#define EXA_CASE(PDEID, PDET, D_, N_, P_)                         \
  if (pde == PDEID && dim == D_ && order == N_ && npar == P_) {    \
    static OpsImpl<PDET, D_, N_, P_> inst;                         \
    return &inst;                                                  \
  }
  EXA_CASE(EXA_PDE_EULER, EulerPDE, 3, 5, 0)
  EXA_CASE(EXA_PDE_EULER, EulerPDE, 3, 3, 0)
  EXA_CASE(EXA_PDE_EULER, EulerPDE, 3, 3, 1)
  EXA_CASE(EXA_PDE_EULER, EulerPDE, 2, 3, 0)
  EXA_CASE(EXA_PDE_EULER, EulerPDE, 2, 3, 1)
  EXA_CASE(EXA_PDE_SWE, SWEPDE, 2, 4, 0)
  EXA_CASE(EXA_PDE_ACOUSTIC, AcousticPDE, 3, 4, 2)
  EXA_CASE(EXA_PDE_ELASTIC, ElasticPDE, 3, 3, 3)
  EXA_CASE(EXA_PDE_ELASTIC, ElasticPDE, 3, 4, 3)
  EXA_CASE(EXA_PDE_ELASTIC, ElasticPDE, 3, 7, 3)
#undef EXA_CASE
  return nullptr;
}

}  // namespace exa

// ------------------------------------------------------------------------------------------
// solver handle
// ------------------------------------------------------------------------------------------
struct exa_solver {
  exa_solver_config cfg;
  exa::Ops* ops = nullptr;  // static launcher object, not owned
  double cfl = 0.9, pnpm = 0.0;
  unsigned* d_status = nullptr;
  std::mutex mu;
  // scratch of the per-cell shims (grown on demand)
  double* d_scratch = nullptr;
  size_t scratch_doubles = 0;
  int* d_iscratch = nullptr;
  int pred_variant = -1;  // predictor launch variant (-1: the measured one)
  int upd_variant = -1;   // update launch variant (-1: bulk-copy form where possible)
  // device memory goes with the handle, also when exa_solver_create fails half-way
  ~exa_solver() {
    cudaFree(d_status);
    cudaFree(d_scratch);
    cudaFree(d_iscratch);
  }
};

static exa::CellArgs base_args(exa_solver* s, int ncells) {
  exa::CellArgs a;
  memset(&a, 0, sizeof(a));
  a.ncells = ncells;
  a.status = s->d_status;
  a.max_picard = s->cfg.max_picard;
  a.cfl_pnpm = s->cfl * s->pnpm;
  a.pnpm = s->pnpm;
  return a;
}

extern "C" {

const char* exa_last_error(void) { return g_err.c_str(); }

int exa_quadrature(int order, double* nodes, double* weights) {
  if (order < 1 || order > 9 || !nodes || !weights) return fail(EXA_ERR_INVALID, "order must be in 1..9");
  for (int i = 0; i <= order; i++) {
    nodes[i] = exa::h_nodes[order - 1][i];
    weights[i] = exa::h_weights[order - 1][i];
  }
  return EXA_OK;
}

int exa_pde_available(int pde, int dim, int order, int npar) {
  return exa::find_ops(pde, dim, order, npar) != nullptr ? 1 : 0;
}

int exa_register_pde(int pde, int dim, int order, int npar, void* ops) {
  exa::Ops* o = static_cast<exa::Ops*>(ops);
  if (!o || pde < EXA_PDE_USER_BASE) return fail(EXA_ERR_INVALID, "user PDE ids start at EXA_PDE_USER_BASE");
  if (o->abi != exa::Ops::kAbi)
    return fail(EXA_ERR_INVALID, "the application library was compiled against another version of "
                                 "exa_ops.cuh: rebuild it");
  if (o->dim != dim || o->order != order || o->npar != npar)
    return fail(EXA_ERR_INVALID, "registration arguments do not match the instantiation");
  std::lock_guard<std::mutex> lk(exa::user_mu());
  for (const exa::UserOps& u : exa::user_ops())
    if (u.pde == pde && u.dim == dim && u.order == order && u.npar == npar)
      return fail(EXA_ERR_INVALID, "this (pde, dim, order, npar) is registered already");
  exa::user_ops().push_back({pde, dim, order, npar, o});
  return EXA_OK;
}
const char* exa_version(void) { return "exa_aderdg 0.1 (sm_100a)"; }

int exa_solver_create(const exa_solver_config* cfg, exa_solver** out) {
  if (!cfg || !out) return fail(EXA_ERR_INVALID, "null argument");
  *out = nullptr;
  if (cfg->dim != 2 && cfg->dim != 3) return fail(EXA_ERR_INVALID, "dim must be 2 or 3");
  if (cfg->order < 1 || cfg->order > 9) return fail(EXA_ERR_INVALID, "order must be in 1..9");
  if (cfg->npar < 0) return fail(EXA_ERR_INVALID, "npar must be >= 0");
  if (cfg->max_picard < 0) return fail(EXA_ERR_INVALID, "max_picard must be >= 0");
  if (cfg->precision != EXA_PREC_FP64 && cfg->precision != EXA_PREC_MIXED)
    return fail(EXA_ERR_INVALID, "unknown precision");
  exa::Ops* ops = exa::find_ops(cfg->pde, cfg->dim, cfg->order, cfg->npar);
  if (!ops || (cfg->precision == EXA_PREC_MIXED && !ops->mixed_ok))
    return fail(EXA_ERR_UNSUPPORTED, "no kernel instantiation for pde=" + std::to_string(cfg->pde) +
                                         " dim=" + std::to_string(cfg->dim) + " order=" +
                                         std::to_string(cfg->order) + " npar=" + std::to_string(cfg->npar) +
                                         " precision=" + std::to_string(cfg->precision));
  std::unique_ptr<exa_solver> s(new exa_solver());
  s->cfg = *cfg;
  s->ops = ops;
  s->cfl = cfg->cfl > 0 ? cfg->cfl : 0.9;
  s->pnpm = cfg->pnpm > 0 ? cfg->pnpm : default_pnpm(cfg->order);
  EXA_CUDA(cudaMalloc(&s->d_status, sizeof(unsigned)));
  EXA_CUDA(cudaMemset(s->d_status, 0, sizeof(unsigned)));
  *out = s.release();
  return EXA_OK;
}

int exa_solver_destroy(exa_solver* s) {
  if (!s) return EXA_OK;
  delete s;
  return EXA_OK;
}

int exa_solver_set_predictor_variant(exa_solver* s, int variant) {
  if (!s || variant < -1 || variant > 1) return fail(EXA_ERR_INVALID, "variant must be -1, 0 or 1");
  s->pred_variant = variant;
  return EXA_OK;
}

int exa_solver_set_update_variant(exa_solver* s, int variant) {
  if (!s || variant < -1 || variant > 1) return fail(EXA_ERR_INVALID, "variant must be -1, 0 or 1");
  s->upd_variant = variant;
  s->ops->riemann_variant = variant;
  return EXA_OK;
}

int exa_solver_predictor_variant(exa_solver* s, int* variant) {
  if (!s || !variant) return fail(EXA_ERR_INVALID, "null argument");
  *variant = s->pred_variant >= 0 ? s->pred_variant : s->ops->tuned_variant(s->cfg.precision == EXA_PREC_MIXED);
  return EXA_OK;
}

int exa_solver_sizes(const exa_solver* s, exa_sizes* o) {
  if (!s || !o) return fail(EXA_ERR_INVALID, "null argument");
  const exa::Ops& p = *s->ops;
  o->nvar = p.nvar;
  o->ndata = p.nvar + p.npar;
  o->nodes_per_cell = p.nd;
  o->nodes_per_face = p.nf;
  o->luh = p.sz_luh;
  o->lduh = p.sz_lduh;
  o->lQhbnd = p.sz_qhb;
  o->lFhbnd = p.sz_fhb;
  o->lQi = p.sz_lQi;
  o->lFi = p.sz_lFi;
  o->lQhi = p.sz_lQhi;
  o->lFhi = p.sz_lFhi;
  return EXA_OK;
}

int exa_solver_status(exa_solver* s, unsigned* bits) {
  if (!s || !bits) return fail(EXA_ERR_INVALID, "null argument");
  EXA_CUDA(cudaDeviceSynchronize());
  EXA_CUDA(cudaMemcpy(bits, s->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  EXA_CUDA(cudaMemset(s->d_status, 0, sizeof(unsigned)));
  return EXA_OK;
}

// ---- batched kernels ---------------------------------------------------------------------
static void set_uniform(exa::CellArgs& a, const exa_solver* s, const double* dx, double dt) {
  for (int d = 0; d < 3; d++) a.u_dx[d] = d < s->cfg.dim ? dx[d] : 1.0;
  a.u_dt = dt;
}

}  // extern "C"

static int fused_call(exa_solver* s, int ncells, const double* luh, double* lduh, double* lQhbnd, double* lFhbnd,
                      int* picard_sweeps, const double* dx, const double* centres, double t, double dt,
                      void* stream) {
  if (!s || ncells < 0 || (ncells > 0 && (!luh || !lduh || !lQhbnd || !lFhbnd || !dx)))
    return fail(EXA_ERR_INVALID, "null argument");
  if (s->ops->alg_source && !centres)
    return fail(EXA_ERR_INVALID, "an algebraic source needs the cells' centres: use the _x entry point");
  exa::CellArgs a = base_args(s, ncells);
  a.luh = luh;
  a.lduh = lduh;
  a.lQhbnd = lQhbnd;
  a.lFhbnd = lFhbnd;
  a.picard = picard_sweeps;
  a.centres = centres;
  a.u_t = t;
  set_uniform(a, s, dx, dt);
  EXA_CUDA(s->ops->reserve(ncells));
  EXA_CUDA(s->ops->predictor(a, (cudaStream_t)stream, s->cfg.precision == EXA_PREC_MIXED, s->pred_variant));
  return EXA_OK;
}

extern "C" {

int exa_fused_predictor_volume_integral(exa_solver* s, int ncells, const double* luh, double* lduh, double* lQhbnd,
                                        double* lFhbnd, int* picard_sweeps, const double* dx, double t, double dt,
                                        void* stream) {
  return fused_call(s, ncells, luh, lduh, lQhbnd, lFhbnd, picard_sweeps, dx, nullptr, t, dt, stream);
}

int exa_fused_predictor_volume_integral_x(exa_solver* s, int ncells, const double* luh, double* lduh,
                                          double* lQhbnd, double* lFhbnd, int* picard_sweeps, const double* dx,
                                          const double* centres, double t, double dt, void* stream) {
  if (ncells > 0 && !centres) return fail(EXA_ERR_INVALID, "null centres");
  return fused_call(s, ncells, luh, lduh, lQhbnd, lFhbnd, picard_sweeps, dx, centres, t, dt, stream);
}

static int check_faces(int nfaces) { return nfaces < 0 ? fail(EXA_ERR_INVALID, "nfaces < 0") : EXA_OK; }

}  // extern "C"

// the batched face entry points; dx (3 doubles, nullable) sets the faces' cell size, which a
// viscous flux needs
static int riemann_call(exa_solver* s, int nfaces, const int* left, const int* right, const signed char* dir,
                        const double* lQhbnd, double* lFhbnd, const double* dx, void* stream) {
  if (!s) return fail(EXA_ERR_INVALID, "null solver");
  if (int e = check_faces(nfaces)) return e;
  if (nfaces > 0 && (!left || !right || !dir || !lQhbnd || !lFhbnd)) return fail(EXA_ERR_INVALID, "null argument");
  if (s->ops->viscous && !dx) return fail(EXA_ERR_INVALID, "a viscous flux needs the cell size: use the _dx entry point");
  exa::FaceArgs f;
  memset(&f, 0, sizeof(f));
  f.nfaces = nfaces;
  f.left = left;
  f.right = right;
  f.dir = reinterpret_cast<const int8_t*>(dir);
  f.lQhbnd = lQhbnd;
  f.lFhbnd = lFhbnd;
  for (int d = 0; d < 3; d++) f.u_dx[d] = dx && d < s->cfg.dim ? dx[d] : 1.0;
  EXA_CUDA(s->ops->riemann(f, (cudaStream_t)stream));
  return EXA_OK;
}

static int boundary_call(exa_solver* s, int nfaces, const int* cell, const signed char* face, const double* lQhbnd,
                         double* lFhbnd, const double* dx, void* stream) {
  if (!s) return fail(EXA_ERR_INVALID, "null solver");
  if (int e = check_faces(nfaces)) return e;
  if (nfaces > 0 && (!cell || !face || !lQhbnd || !lFhbnd)) return fail(EXA_ERR_INVALID, "null argument");
  if (s->ops->viscous && !dx) return fail(EXA_ERR_INVALID, "a viscous flux needs the cell size: use the _dx entry point");
  exa::FaceArgs f;
  memset(&f, 0, sizeof(f));
  f.nfaces = nfaces;
  f.bcell = cell;
  f.bface = reinterpret_cast<const int8_t*>(face);
  f.lQhbnd = lQhbnd;
  f.lFhbnd = lFhbnd;
  for (int d = 0; d < 3; d++) f.u_dx[d] = dx && d < s->cfg.dim ? dx[d] : 1.0;
  EXA_CUDA(s->ops->boundary(f, (cudaStream_t)stream));
  return EXA_OK;
}

extern "C" {

int exa_riemann_solver_nonlinear(exa_solver* s, int nfaces, const int* left, const int* right, const signed char* dir,
                                 const double* lQhbnd, double* lFhbnd, void* stream) {
  return riemann_call(s, nfaces, left, right, dir, lQhbnd, lFhbnd, nullptr, stream);
}

int exa_riemann_solver_nonlinear_dx(exa_solver* s, int nfaces, const int* left, const int* right,
                                    const signed char* dir, const double* lQhbnd, double* lFhbnd, const double* dx,
                                    void* stream) {
  if (!dx) return fail(EXA_ERR_INVALID, "null dx");
  return riemann_call(s, nfaces, left, right, dir, lQhbnd, lFhbnd, dx, stream);
}

int exa_boundary_conditions_wall(exa_solver* s, int nfaces, const int* cell, const signed char* face,
                                 const double* lQhbnd, double* lFhbnd, void* stream) {
  return boundary_call(s, nfaces, cell, face, lQhbnd, lFhbnd, nullptr, stream);
}

int exa_boundary_conditions_wall_dx(exa_solver* s, int nfaces, const int* cell, const signed char* face,
                                    const double* lQhbnd, double* lFhbnd, const double* dx, void* stream) {
  if (!dx) return fail(EXA_ERR_INVALID, "null dx");
  return boundary_call(s, nfaces, cell, face, lQhbnd, lFhbnd, dx, stream);
}

int exa_surface_integral_and_update(exa_solver* s, int ncells, double* luh, const double* lduh, const double* lFhbnd,
                                    const double* dx, double dt, void* stream) {
  if (!s || ncells < 0 || (ncells > 0 && (!luh || !lduh || !lFhbnd || !dx)))
    return fail(EXA_ERR_INVALID, "null argument");
  exa::CellArgs a = base_args(s, ncells);
  a.luh = luh;
  a.luh_out = luh;
  a.lduh = const_cast<double*>(lduh);
  a.lFhbnd = const_cast<double*>(lFhbnd);
  set_uniform(a, s, dx, dt);
  EXA_CUDA(s->ops->update(a, true, true, (cudaStream_t)stream, s->upd_variant));
  return EXA_OK;
}

int exa_solution_update(exa_solver* s, int ncells, double* luh, const double* luhOld, const double* lduh, double dt,
                        void* stream) {
  if (!s || ncells < 0 || (ncells > 0 && (!luh || !luhOld || !lduh))) return fail(EXA_ERR_INVALID, "null argument");
  exa::CellArgs a = base_args(s, ncells);
  a.luh = luhOld;
  a.luh_out = luh;
  a.lduh = const_cast<double*>(lduh);
  double one[3] = {1.0, 1.0, 1.0};
  set_uniform(a, s, one, dt);
  EXA_CUDA(s->ops->update(a, false, true, (cudaStream_t)stream));
  return EXA_OK;
}

}  // extern "C"

// exa_stable_time_step_size with the solver's lock already held (the per-cell shim keeps it over
// its copies, so that no other thread can move the scratch in between)
static int stable_dt_locked(exa_solver* s, int ncells, const double* luh, const double* dx, double* cell_dt,
                            double* dt_min, cudaStream_t st) {
  exa::CellArgs a = base_args(s, ncells);
  a.luh = luh;
  a.cell_dt = cell_dt;
  set_uniform(a, s, dx, 0.0);
  if (dt_min) {
    if (!s->d_scratch) {
      EXA_CUDA(cudaMalloc(&s->d_scratch, 1024 * sizeof(double)));
      s->scratch_doubles = 1024;
    }
    exa::fill_kernel<<<1, 32, 0, st>>>(1, s->d_scratch, INFINITY);
    a.grid_dt_next = s->d_scratch;
  }
  EXA_CUDA(s->ops->update(a, false, false, st));
  if (dt_min) {
    EXA_CUDA(cudaMemcpyAsync(dt_min, s->d_scratch, sizeof(double), cudaMemcpyDeviceToHost, st));
    EXA_CUDA(cudaStreamSynchronize(st));
  }
  return EXA_OK;
}

extern "C" {

int exa_stable_time_step_size(exa_solver* s, int ncells, const double* luh, const double* dx, double* cell_dt,
                              double* dt_min, void* stream) {
  if (!s || ncells < 0 || (ncells > 0 && (!luh || !dx))) return fail(EXA_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  return stable_dt_locked(s, ncells, luh, dx, cell_dt, dt_min, (cudaStream_t)stream);
}

// ---- per-cell shims on host pointers ---------------------------------------------------------
static int shim_scratch(exa_solver* s, size_t doubles) {
  if (s->scratch_doubles >= doubles && s->d_scratch) return EXA_OK;
  cudaFree(s->d_scratch);
  s->d_scratch = nullptr;
  s->scratch_doubles = 0;
  EXA_CUDA(cudaMalloc(&s->d_scratch, doubles * sizeof(double)));
  s->scratch_doubles = doubles;
  if (!s->d_iscratch) EXA_CUDA(cudaMalloc(&s->d_iscratch, 64 * sizeof(int)));
  return EXA_OK;
}

int exa_spaceTimePredictorNonlinear(exa_solver* s, double* lQhbnd, double* lFhbnd, double* lQi, double* lFi,
                                    double* lQhi, double* lFhi, const double* luh, const double* cellCenter,
                                    const double* invDx, double t, double dt) {
  if (!s || !lQhbnd || !lFhbnd || !luh || !invDx || (s->ops->alg_source && !cellCenter)) {
    fail(EXA_ERR_INVALID, "null argument");
    return -1;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  const exa::Ops& o = *s->ops;
  const size_t total = o.sz_luh + o.sz_lduh + o.sz_qhb + o.sz_fhb + o.sz_lQi + o.sz_lFi + o.sz_lQhi + o.sz_lFhi + 3;
  if (shim_scratch(s, total)) return -1;
  double* d = s->d_scratch;
  double *d_luh = d, *d_lduh = d_luh + o.sz_luh, *d_qhb = d_lduh + o.sz_lduh, *d_fhb = d_qhb + o.sz_qhb;
  double *d_lQi = d_fhb + o.sz_fhb, *d_lFi = d_lQi + o.sz_lQi, *d_lQhi = d_lFi + o.sz_lFi, *d_lFhi = d_lQhi + o.sz_lQhi;
  double* d_centre = d_lFhi + o.sz_lFhi;
  if (cudaMemcpy(d_luh, luh, o.sz_luh * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
  // the cell's position and time reach an algebraic source (:339-345)
  double centre[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < s->cfg.dim && cellCenter; k++) centre[k] = cellCenter[k];
  if (cudaMemcpy(d_centre, centre, sizeof(centre), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
  exa::CellArgs a = base_args(s, 1);
  a.centres = d_centre;
  a.u_t = t;
  a.luh = d_luh;
  a.lduh = d_lduh;
  a.lQhbnd = d_qhb;
  a.lFhbnd = d_fhb;
  a.picard = s->d_iscratch;
  a.ex_lQi = d_lQi;
  a.ex_lFi = d_lFi;
  a.ex_lQhi = d_lQhi;
  a.ex_lFhi = d_lFhi;
  double dx[3] = {1.0, 1.0, 1.0};
  for (int k = 0; k < s->cfg.dim; k++) dx[k] = 1.0 / invDx[k];
  set_uniform(a, s, dx, dt);
  cudaError_t e = s->ops->reserve(1);
  if (e == cudaSuccess) e = s->ops->predictor(a, 0, s->cfg.precision == EXA_PREC_MIXED, s->pred_variant);
  if (e != cudaSuccess) {
    cuda_fail(e, "predictor");
    return -1;
  }
  int sweeps = 0;
  if (cudaMemcpy(&sweeps, s->d_iscratch, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  cudaMemcpy(lQhbnd, d_qhb, o.sz_qhb * sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(lFhbnd, d_fhb, o.sz_fhb * sizeof(double), cudaMemcpyDeviceToHost);
  if (lQi) cudaMemcpy(lQi, d_lQi, o.sz_lQi * sizeof(double), cudaMemcpyDeviceToHost);
  if (lFi) cudaMemcpy(lFi, d_lFi, o.sz_lFi * sizeof(double), cudaMemcpyDeviceToHost);
  if (lQhi) cudaMemcpy(lQhi, d_lQhi, o.sz_lQhi * sizeof(double), cudaMemcpyDeviceToHost);
  if (lFhi) cudaMemcpy(lFhi, d_lFhi, o.sz_lFhi * sizeof(double), cudaMemcpyDeviceToHost);
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  // the reference's return value (3d/...:408-412 breaks at the converging index; 2d/...:303-305
  // reports MaxIterations+2 on convergence)
  const int maxIter = s->cfg.max_picard > 0 ? s->cfg.max_picard : 2 * (s->cfg.order + 1);
  const bool converged = s->cfg.max_picard <= 0 && sweeps < maxIter ? true : false;
  if (s->cfg.max_picard > 0) return maxIter;
  if (s->cfg.dim == 2) return converged ? maxIter + 2 : maxIter;
  return converged ? sweeps - 1 : maxIter;
}

// one cell's volume / surface / face integral on the device (cell_integral_kernel)
static int shim_cell_integral(exa_solver* s, int mode, double* lduh, const double* in, size_t in_doubles,
                              int direction, int orientation, const double* dx) {
  std::lock_guard<std::mutex> lk(s->mu);
  const exa::Ops& o = *s->ops;
  if (int e = shim_scratch(s, o.sz_lduh + in_doubles)) return e;
  double* d_du = s->d_scratch;
  double* d_in = d_du + o.sz_lduh;
  if (mode != 0) EXA_CUDA(cudaMemcpy(d_du, lduh, o.sz_lduh * sizeof(double), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(d_in, in, in_doubles * sizeof(double), cudaMemcpyHostToDevice));
  double d3[3] = {1.0, 1.0, 1.0};
  for (int d = 0; d < o.dim; d++) d3[d] = dx[d];
  EXA_CUDA(s->ops->cell_integral(mode, d_du, d_in, direction, orientation, d3, 0));
  EXA_CUDA(cudaMemcpy(lduh, d_du, o.sz_lduh * sizeof(double), cudaMemcpyDeviceToHost));
  return EXA_OK;
}

int exa_volumeIntegralNonlinear(exa_solver* s, double* lduh, const double* lFhi, const double* dx) {
  if (!s || !lduh || !lFhi || !dx) return fail(EXA_ERR_INVALID, "null argument");
  return shim_cell_integral(s, 0, lduh, lFhi, s->ops->sz_lFhi, 0, 0, dx);
}

int exa_faceIntegralNonlinear(exa_solver* s, double* lduh, const double* lFhbnd, int direction, int orientation,
                              const double* dx) {
  if (!s || !lduh || !lFhbnd || !dx) return fail(EXA_ERR_INVALID, "null argument");
  if (direction < 0 || direction >= s->ops->dim || (orientation != 0 && orientation != 1))
    return fail(EXA_ERR_INVALID, "bad face");
  return shim_cell_integral(s, 2, lduh, lFhbnd, (size_t)s->ops->nf * s->ops->nvar, direction, orientation, dx);
}

int exa_riemannSolverNonlinear(exa_solver* s, double* FL, double* FR, const double* QL, const double* QR, double t,
                               double dt, const double* dx, int direction) {
  (void)t; (void)dt;
  if (!s || !FL || !FR || !QL || !QR || !dx) return fail(EXA_ERR_INVALID, "null argument");
  if (direction < 0 || direction >= s->cfg.dim) return fail(EXA_ERR_INVALID, "direction out of range");
  std::lock_guard<std::mutex> lk(s->mu);
  const exa::Ops& o = *s->ops;
  // two one-cell blocks: cell 0 holds QL/FL on face 2d+1, cell 1 holds QR/FR on face 2d
  const size_t total = 2 * (o.sz_qhb + o.sz_fhb);
  if (int e = shim_scratch(s, total)) return e;
  double* qhb = s->d_scratch;
  double* fhb = qhb + 2 * o.sz_qhb;
  const size_t fq = o.sz_qhb / (2 * o.dim), ff = o.sz_fhb / (2 * o.dim);
  EXA_CUDA(cudaMemcpy(qhb + (2 * direction + 1) * fq, QL, fq * sizeof(double), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(qhb + o.sz_qhb + (2 * direction) * fq, QR, fq * sizeof(double), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(fhb + (2 * direction + 1) * ff, FL, ff * sizeof(double), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(fhb + o.sz_fhb + (2 * direction) * ff, FR, ff * sizeof(double), cudaMemcpyHostToDevice));
  int* idx = s->d_iscratch;
  int h[3] = {0, 1, 0};
  int8_t dd = (int8_t)direction;
  EXA_CUDA(cudaMemcpy(idx, h, 2 * sizeof(int), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(idx + 2, &dd, 1, cudaMemcpyHostToDevice));
  exa::FaceArgs f;
  memset(&f, 0, sizeof(f));
  f.nfaces = 1;
  f.left = idx;
  f.right = idx + 1;
  f.dir = reinterpret_cast<const int8_t*>(idx + 2);
  f.lQhbnd = qhb;
  f.lFhbnd = fhb;
  for (int d = 0; d < 3; d++) f.u_dx[d] = d < o.dim ? dx[d] : 1.0;  // a viscous flux's Rusanov speed
  EXA_CUDA(s->ops->riemann(f, 0));
  EXA_CUDA(cudaMemcpy(FL, fhb + (2 * direction + 1) * ff, ff * sizeof(double), cudaMemcpyDeviceToHost));
  EXA_CUDA(cudaMemcpy(FR, fhb + o.sz_fhb + (2 * direction) * ff, ff * sizeof(double), cudaMemcpyDeviceToHost));
  return EXA_OK;
}

int exa_surfaceIntegralNonlinear(exa_solver* s, double* lduh, const double* lFhbnd, const double* dx) {
  if (!s || !lduh || !lFhbnd || !dx) return fail(EXA_ERR_INVALID, "null argument");
  return shim_cell_integral(s, 1, lduh, lFhbnd, s->ops->sz_fhb, 0, 0, dx);
}

int exa_solutionUpdate(exa_solver* s, double* luh, const double* luhOld, const double* lduh, double dt) {
  if (!s || !luh || !luhOld || !lduh) return fail(EXA_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  const exa::Ops& o = *s->ops;
  if (int e = shim_scratch(s, 2 * o.sz_luh + o.sz_lduh)) return e;
  double* d_old = s->d_scratch;
  double* d_new = d_old + o.sz_luh;
  double* d_du = d_new + o.sz_luh;
  EXA_CUDA(cudaMemcpy(d_old, luhOld, o.sz_luh * sizeof(double), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(d_new, luhOld, o.sz_luh * sizeof(double), cudaMemcpyHostToDevice));
  EXA_CUDA(cudaMemcpy(d_du, lduh, o.sz_lduh * sizeof(double), cudaMemcpyHostToDevice));
  exa::CellArgs a = base_args(s, 1);
  a.luh = d_old;
  a.luh_out = d_new;
  a.lduh = d_du;
  double one[3] = {1.0, 1.0, 1.0};
  set_uniform(a, s, one, dt);
  EXA_CUDA(s->ops->update(a, false, true, 0));
  // parameters are not touched by solutionUpdate: keep the caller's luh entries for them
  std::vector<double> tmp(o.sz_luh);
  EXA_CUDA(cudaMemcpy(tmp.data(), d_new, o.sz_luh * sizeof(double), cudaMemcpyDeviceToHost));
  const int D = o.nvar + o.npar;
  for (int p = 0; p < o.nd; p++)
    for (int m = 0; m < o.nvar; m++) luh[p * D + m] = tmp[p * D + m];
  return EXA_OK;
}

int exa_stableTimeStepSize(exa_solver* s, const double* luh, const double* dx, double* dt) {
  if (!s || !luh || !dx || !dt) return fail(EXA_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  // scratch: the cell's dt in entry 0, its luh from entry 8 on
  if (int e = shim_scratch(s, s->ops->sz_luh + 8)) return e;
  double* d_luh = s->d_scratch + 8;
  EXA_CUDA(cudaMemcpy(d_luh, luh, s->ops->sz_luh * sizeof(double), cudaMemcpyHostToDevice));
  if (int r = stable_dt_locked(s, 1, d_luh, dx, s->d_scratch, nullptr, 0)) return r;
  EXA_CUDA(cudaMemcpy(dt, s->d_scratch, sizeof(double), cudaMemcpyDeviceToHost));
  return EXA_OK;
}

// ---- mesh levels and the limiter ------------------------------------------------------------
static int amr_call(exa_solver* s, bool face, int mode, double* fQ, double* fF, double* cQ, double* cF, long long nfine,
                    long long ncoarse, int njobs, const int* jobs, int ngroups, const int* group_ptr, cudaStream_t st) {
  if (!s) return fail(EXA_ERR_INVALID, "null solver");
  if (mode < EXA_AMR_PROLONGATE || mode > EXA_AMR_RESTRICT_FLUX || (mode == EXA_AMR_RESTRICT_FLUX && !face))
    return fail(EXA_ERR_INVALID, "bad mode");
  if (face && s->cfg.dim < 2) return fail(EXA_ERR_UNSUPPORTED, "faces of a 1D cell");
  if (njobs < 0 || nfine < 0 || ncoarse < 0 || ngroups < 0) return fail(EXA_ERR_INVALID, "negative size");
  if (mode != EXA_AMR_RESTRICT || !group_ptr) {
    group_ptr = nullptr;
    ngroups = njobs;
  }
  if (ngroups == 0) return EXA_OK;
  if (!jobs) return fail(EXA_ERR_INVALID, "null jobs");
  const bool needQ = mode != EXA_AMR_RESTRICT_FLUX;
  if ((needQ && (!fQ || !cQ)) || (face && (!fF || !cF))) return fail(EXA_ERR_INVALID, "null block array");
  exa::AmrArgs a;
  memset(&a, 0, sizeof(a));
  a.mode = mode;
  if (mode == EXA_AMR_PROLONGATE) {
    a.outQ = fQ, a.inQ = cQ, a.outF = fF, a.inF = cF;
  } else {
    a.outQ = cQ, a.inQ = fQ, a.outF = cF, a.inF = fF;
  }
  a.nfine = nfine;
  a.ncoarse = ncoarse;
  a.ngroups = ngroups;
  a.ptr = group_ptr;
  a.njobs = njobs;
  a.jobs = jobs;
  a.status = s->d_status;
  EXA_CUDA(s->ops->amr(a, face, st));
  return EXA_OK;
}

int exa_amr_volume_unknowns(exa_solver* s, int mode, double* luhFine, double* luhCoarse, long long nfine,
                            long long ncoarse, int njobs, const int* jobs, int ngroups, const int* group_ptr,
                            void* stream) {
  return amr_call(s, false, mode, luhFine, nullptr, luhCoarse, nullptr, nfine, ncoarse, njobs, jobs, ngroups,
                  group_ptr, (cudaStream_t)stream);
}

int exa_amr_face_unknowns(exa_solver* s, int mode, double* lQhbndFine, double* lFhbndFine, double* lQhbndCoarse,
                          double* lFhbndCoarse, long long nfine, long long ncoarse, int njobs, const int* jobs,
                          int ngroups, const int* group_ptr, void* stream) {
  return amr_call(s, true, mode, lQhbndFine, lFhbndFine, lQhbndCoarse, lFhbndCoarse, nfine, ncoarse, njobs, jobs,
                  ngroups, group_ptr, (cudaStream_t)stream);
}

// one job on host arrays: the blocks are copied to the shim scratch, the job checked on the host
static int amr_shim(exa_solver* s, bool face, int mode, double* fQ, double* fF, double* cQ, double* cF, int levelDelta,
                    const int* index) {
  if (!s || !index) return fail(EXA_ERR_INVALID, "null argument");
  const int axes = face ? s->cfg.dim - 1 : s->cfg.dim;
  if (levelDelta < 1 || levelDelta > exa::kAmrMaxLevelDelta) return fail(EXA_ERR_INVALID, "level difference out of range");
  long long span = 1;
  for (int l = 0; l < levelDelta; l++) span *= 3;
  int job[6] = {0, 0, levelDelta, 0, 0, 0};
  for (int r = 0; r < axes; r++) {
    if (index[r] < 0 || index[r] >= span) return fail(EXA_ERR_INVALID, "subcell index out of range");
    job[3 + r] = index[r];
  }
  std::lock_guard<std::mutex> lk(s->mu);
  const exa::Ops& o = *s->ops;
  const size_t nq = face ? o.sz_qhb / (2 * o.dim) : o.sz_luh, nf = face ? o.sz_fhb / (2 * o.dim) : 0;
  if (int e = shim_scratch(s, 2 * (nq + nf))) return e;
  double *dfQ = s->d_scratch, *dcQ = dfQ + nq, *dfF = dcQ + nq, *dcF = dfF + nf;
  const bool needQ = mode != EXA_AMR_RESTRICT_FLUX;
  auto up = [&](double* d, const double* h, size_t k) { return cudaMemcpy(d, h, k * sizeof(double), cudaMemcpyHostToDevice); };
  auto down = [&](double* h, const double* d, size_t k) { return cudaMemcpy(h, d, k * sizeof(double), cudaMemcpyDeviceToHost); };
  if (needQ && (!fQ || !cQ)) return fail(EXA_ERR_INVALID, "null argument");
  if (face && (!fF || !cF)) return fail(EXA_ERR_INVALID, "null argument");
  if (mode == EXA_AMR_PROLONGATE) {
    EXA_CUDA(up(dcQ, cQ, nq));
    if (face) EXA_CUDA(up(dcF, cF, nf));
  } else {
    if (needQ) EXA_CUDA(up(dfQ, fQ, nq));
    if (needQ) EXA_CUDA(up(dcQ, cQ, nq));
    if (face) EXA_CUDA(up(dfF, fF, nf));
    if (face && mode == EXA_AMR_RESTRICT) EXA_CUDA(up(dcF, cF, nf));
  }
  EXA_CUDA(cudaMemcpy(s->d_iscratch, job, sizeof(job), cudaMemcpyHostToDevice));
  if (int e = amr_call(s, face, mode, needQ ? dfQ : nullptr, face ? dfF : nullptr, needQ ? dcQ : nullptr,
                       face ? dcF : nullptr, 1, 1, 1, s->d_iscratch, 1, nullptr, 0))
    return e;
  if (mode == EXA_AMR_PROLONGATE) {
    EXA_CUDA(down(fQ, dfQ, nq));
    if (face) EXA_CUDA(down(fF, dfF, nf));
  } else {
    if (needQ) EXA_CUDA(down(cQ, dcQ, nq));
    if (face) EXA_CUDA(down(cF, dcF, nf));
  }
  return EXA_OK;
}

int exa_volumeUnknownsProlongation(exa_solver* s, double* luhFine, const double* luhCoarse, int coarseGridLevel,
                                   int fineGridLevel, const int* subcellIndex) {
  return amr_shim(s, false, EXA_AMR_PROLONGATE, luhFine, nullptr, const_cast<double*>(luhCoarse), nullptr,
                  fineGridLevel - coarseGridLevel, subcellIndex);
}
int exa_volumeUnknownsRestriction(exa_solver* s, double* luhCoarse, const double* luhFine, int coarseGridLevel,
                                  int fineGridLevel, const int* subcellIndex) {
  return amr_shim(s, false, EXA_AMR_RESTRICT, const_cast<double*>(luhFine), nullptr, luhCoarse, nullptr,
                  fineGridLevel - coarseGridLevel, subcellIndex);
}
int exa_faceUnknownsProlongation(exa_solver* s, double* lQhbndFine, double* lFhbndFine, const double* lQhbndCoarse,
                                 const double* lFhbndCoarse, int coarseGridLevel, int fineGridLevel,
                                 const int* subfaceIndex) {
  return amr_shim(s, true, EXA_AMR_PROLONGATE, lQhbndFine, lFhbndFine, const_cast<double*>(lQhbndCoarse),
                  const_cast<double*>(lFhbndCoarse), fineGridLevel - coarseGridLevel, subfaceIndex);
}
int exa_faceUnknownsRestriction(exa_solver* s, double* lQhbndCoarse, double* lFhbndCoarse, const double* lQhbndFine,
                                const double* lFhbndFine, int coarseGridLevel, int fineGridLevel,
                                const int* subfaceIndex) {
  return amr_shim(s, true, EXA_AMR_RESTRICT, const_cast<double*>(lQhbndFine), const_cast<double*>(lFhbndFine),
                  lQhbndCoarse, lFhbndCoarse, fineGridLevel - coarseGridLevel, subfaceIndex);
}
int exa_faceFluxRestriction(exa_solver* s, double* lFhbndCoarse, const double* lFhbndFine, const int* subfaceIndex,
                            int levelDelta) {
  return amr_shim(s, true, EXA_AMR_RESTRICT_FLUX, nullptr, const_cast<double*>(lFhbndFine), nullptr, lFhbndCoarse,
                  levelDelta, subfaceIndex);
}

static int lim_patch(const exa_solver* s, int ghost) {
  const int E = 2 * s->cfg.order + 1 + 2 * ghost;
  return s->cfg.dim == 3 ? E * E * E : E * E;
}
static int lim_call(exa_solver* s, exa::LimArgs& a, cudaStream_t st) {
  if (!s) return fail(EXA_ERR_INVALID, "null solver");
  const int D = s->ops->nvar + s->ops->npar;
  if (a.ncells < 0) return fail(EXA_ERR_INVALID, "ncells < 0");
  if (a.ghost < 0 || a.ghost > 4) return fail(EXA_ERR_INVALID, "ghost layer width out of range");
  if (a.nobs < 0 || a.nobs > std::min(32, D)) return fail(EXA_ERR_INVALID, "observables out of range");
  if (a.ncells == 0) return EXA_OK;
  EXA_CUDA(s->ops->limiter(a, st));
  return EXA_OK;
}
static exa::LimArgs lim_args(int op, int ncells, int ghost, int nobs) {
  exa::LimArgs a;
  memset(&a, 0, sizeof(a));
  a.op = op;
  a.ncells = ncells;
  a.ghost = ghost;
  a.nobs = nobs;
  return a;
}

int exa_limiter_project_on_fv(exa_solver* s, int ncells, const double* luh, double* lim, int ghost, void* stream) {
  if (ncells > 0 && (!luh || !lim)) return fail(EXA_ERR_INVALID, "null argument");
  exa::LimArgs a = lim_args(0, ncells, ghost, 0);
  a.luh = luh;
  a.lim_out = lim;
  return lim_call(s, a, (cudaStream_t)stream);
}
int exa_limiter_project_on_dg(exa_solver* s, int ncells, const double* lim, double* luh, int ghost, void* stream) {
  if (ncells > 0 && (!luh || !lim)) return fail(EXA_ERR_INVALID, "null argument");
  exa::LimArgs a = lim_args(1, ncells, ghost, 0);
  a.lim = lim;
  a.luh_out = luh;
  return lim_call(s, a, (cudaStream_t)stream);
}
int exa_limiter_local_min_max(exa_solver* s, int ncells, const double* luh, int nobs, double* mn, double* mx,
                              void* stream) {
  if (ncells > 0 && nobs > 0 && (!luh || !mn || !mx)) return fail(EXA_ERR_INVALID, "null argument");
  exa::LimArgs a = lim_args(2, ncells, 0, nobs);
  a.luh = luh;
  a.mn = mn;
  a.mx = mx;
  return lim_call(s, a, (cudaStream_t)stream);
}
int exa_limiter_fv_min_max(exa_solver* s, int ncells, const double* lim, int ghost, int nobs, double* mn, double* mx,
                           void* stream) {
  if (ncells > 0 && nobs > 0 && (!lim || !mn || !mx)) return fail(EXA_ERR_INVALID, "null argument");
  exa::LimArgs a = lim_args(3, ncells, ghost, nobs);
  a.lim = lim;
  a.mn = mn;
  a.mx = mx;
  return lim_call(s, a, (cudaStream_t)stream);
}
int exa_limiter_dmp(exa_solver* s, int ncells, const double* luh, int nobs, double relax, double scale, double* bmin,
                    double* bmax, unsigned char* ok, void* stream) {
  if (ncells > 0 && (!luh || !ok || (nobs > 0 && (!bmin || !bmax)))) return fail(EXA_ERR_INVALID, "null argument");
  exa::LimArgs a = lim_args(4, ncells, 0, nobs);
  a.luh = luh;
  a.mn = bmin;
  a.mx = bmax;
  a.ok = ok;
  a.relax = relax;
  a.scale = scale;
  return lim_call(s, a, (cudaStream_t)stream);
}

// one cell on host arrays through the shim scratch: [luh][lim][mn][mx][ok]
static int lim_shim(exa_solver* s, int op, const double* luh_in, double* luh_out, const double* lim_in, double* lim_out,
                    int ghost, int nobs, double* mn, double* mx, double relax, double scale, int* ok) {
  if (!s) return fail(EXA_ERR_INVALID, "null solver");
  if (ghost < 0 || ghost > 4) return fail(EXA_ERR_INVALID, "ghost layer width out of range");
  const int D = s->ops->nvar + s->ops->npar;
  if (nobs < 0 || nobs > std::min(32, D)) return fail(EXA_ERR_INVALID, "observables out of range");
  std::lock_guard<std::mutex> lk(s->mu);
  const size_t nl = (size_t)s->ops->sz_luh, nm = (size_t)lim_patch(s, ghost) * D;
  const size_t nb = op == 4 ? (size_t)2 * s->cfg.dim * nobs : (size_t)nobs;
  if (int e = shim_scratch(s, nl + nm + 2 * nb + 1)) return e;
  double *d_luh = s->d_scratch, *d_lim = d_luh + nl, *d_mn = d_lim + nm, *d_mx = d_mn + nb;
  unsigned char* d_ok = reinterpret_cast<unsigned char*>(d_mx + nb);
  if (luh_in) EXA_CUDA(cudaMemcpy(d_luh, luh_in, nl * sizeof(double), cudaMemcpyHostToDevice));
  if (lim_in) EXA_CUDA(cudaMemcpy(d_lim, lim_in, nm * sizeof(double), cudaMemcpyHostToDevice));
  if (lim_out) EXA_CUDA(cudaMemcpy(d_lim, lim_out, nm * sizeof(double), cudaMemcpyHostToDevice));  // ghosts kept
  if (op == 4 && nb) {
    EXA_CUDA(cudaMemcpy(d_mn, mn, nb * sizeof(double), cudaMemcpyHostToDevice));
    EXA_CUDA(cudaMemcpy(d_mx, mx, nb * sizeof(double), cudaMemcpyHostToDevice));
  }
  exa::LimArgs a = lim_args(op, 1, ghost, nobs);
  a.luh = d_luh;
  a.luh_out = d_luh;
  a.lim = d_lim;
  a.lim_out = d_lim;
  a.mn = d_mn;
  a.mx = d_mx;
  a.ok = d_ok;
  a.relax = relax;
  a.scale = scale;
  if (int e = lim_call(s, a, 0)) return e;
  if (luh_out) EXA_CUDA(cudaMemcpy(luh_out, d_luh, nl * sizeof(double), cudaMemcpyDeviceToHost));
  if (lim_out) EXA_CUDA(cudaMemcpy(lim_out, d_lim, nm * sizeof(double), cudaMemcpyDeviceToHost));
  if (mn && nb) EXA_CUDA(cudaMemcpy(mn, d_mn, nb * sizeof(double), cudaMemcpyDeviceToHost));
  if (mx && nb) EXA_CUDA(cudaMemcpy(mx, d_mx, nb * sizeof(double), cudaMemcpyDeviceToHost));
  if (ok) {
    unsigned char v = 1;
    EXA_CUDA(cudaMemcpy(&v, d_ok, 1, cudaMemcpyDeviceToHost));
    *ok = v;
  }
  return EXA_OK;
}

int exa_projectOnFVLimiterSpace(exa_solver* s, const double* luh, double* lim, int ghost) {
  if (!luh || !lim) return fail(EXA_ERR_INVALID, "null argument");
  return lim_shim(s, 0, luh, nullptr, nullptr, lim, ghost, 0, nullptr, nullptr, 0.0, 0.0, nullptr);
}
int exa_projectOnDGSpace(exa_solver* s, const double* lim, double* luh, int ghost) {
  if (!luh || !lim) return fail(EXA_ERR_INVALID, "null argument");
  return lim_shim(s, 1, nullptr, luh, lim, nullptr, ghost, 0, nullptr, nullptr, 0.0, 0.0, nullptr);
}
int exa_findCellLocalMinAndMax(exa_solver* s, const double* luh, int nobs, double* mn, double* mx) {
  if (!luh || (nobs > 0 && (!mn || !mx))) return fail(EXA_ERR_INVALID, "null argument");
  return lim_shim(s, 2, luh, nullptr, nullptr, nullptr, 0, nobs, mn, mx, 0.0, 0.0, nullptr);
}
int exa_findCellLocalLimiterMinAndMax(exa_solver* s, const double* lim, int ghost, int nobs, double* mn, double* mx) {
  if (!lim || (nobs > 0 && (!mn || !mx))) return fail(EXA_ERR_INVALID, "null argument");
  return lim_shim(s, 3, nullptr, nullptr, lim, nullptr, ghost, nobs, mn, mx, 0.0, 0.0, nullptr);
}
int exa_discreteMaximumPrincipleAndMinAndMaxSearch(exa_solver* s, const double* luh, int nobs, double relax,
                                                   double scale, double* bmin, double* bmax, int* ok) {
  if (!luh || !ok || (nobs > 0 && (!bmin || !bmax))) return fail(EXA_ERR_INVALID, "null argument");
  return lim_shim(s, 4, luh, nullptr, nullptr, nullptr, 0, nobs, bmin, bmax, relax, scale, ok);
}

int exa_amr_limiter_projectors(int order, double* fine, double* dg2fv, double* fv2dg, double* leg2lob) {
  if (order < 1 || order > 9) return fail(EXA_ERR_INVALID, "order out of range");
  const int n = order + 1, P = 2 * order + 1;
  const double* t = exa::h_amr_lim[order];
  if (fine) std::copy_n(t, 3 * n * n, fine);
  t += 3 * n * n;
  if (dg2fv) std::copy_n(t, n * P, dg2fv);
  t += n * P;
  if (fv2dg) std::copy_n(t, P * n, fv2dg);
  t += P * n;
  if (leg2lob) std::copy_n(t, n * n, leg2lob);
  return EXA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// device-resident patches
// ------------------------------------------------------------------------------------------
struct exa_patch {
  exa_solver* s = nullptr;
  std::vector<exa_grid_desc> grids;
  long long ncells = 0;
  std::vector<long long> grid_first;
  double *luh = nullptr, *lduh = nullptr, *lQhbnd = nullptr, *lFhbnd = nullptr;
  int* picard = nullptr;
  int* cell_grid = nullptr;
  double *grid_dx = nullptr, *grid_t = nullptr, *grid_dt = nullptr, *grid_dt_next = nullptr;
  long long* steps = nullptr;
  int *fL = nullptr, *fR = nullptr;
  int8_t* fdir = nullptr;
  int nfaces = 0;
  int nhalo_faces = 0;  // the last nhalo_faces of the face list touch a ghost cell
  int* bcell = nullptr;
  int8_t* bface = nullptr;
  int nbfaces = 0;
  unsigned* status = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph_cfl = nullptr, graph_fixed = nullptr;
  bool track_picard = false;
  double fixed_dt = -1.0;
  double* grid_geo = nullptr;       // [grid][6]: lower corner, cells per axis
  long long* grid_first_d = nullptr; // [grid] first cell
  double* src = nullptr;            // point source parameters (8 doubles), nullptr when unset
  // the source's slot table (Ops::source_slots) and its values per slot, time node and node
  int* src_slot = nullptr;
  int* src_cells = nullptr;
  double* src_vals = nullptr;
  int nsrc = 0;
  int8_t* btype = nullptr;          // boundary type of every domain face
  // halo (slab decomposition): ghost cells appended after the real cells, face traces only
  long long nghost = 0;      // 2 * layer cells, or 0
  int halo_axis = -1;        // axis with EXA_BC_HALO
  bool has_user_bc = false;  // some domain face is EXA_BC_USER
  long long layer = 0;       // cells per layer normal to the halo axis
  long long halo_lo_first = 0, halo_hi_first = 0;  // first real cell of the low / high boundary layer
  // discrete adjoint workspace (allocated on the first exa_patch_adjoint_step)
  double *adjQ = nullptr, *adjF = nullptr, *adj_iter = nullptr;
  // halo patches: lambda of the real cells and, after them, of the ghost cells (the neighbours'
  // boundary layers), which the transposed halo faces read
  double* adj_lam = nullptr;
  bool adj_forward_done = false;  // EXA_ADJ_FORWARD ran and EXA_ADJ_REVERSE has not yet
  // host-buffer steps: copy stream and per-chunk events (created on the first exa_patch_step_host)
  cudaStream_t copy_stream = nullptr, d2h_stream = nullptr;
  std::vector<cudaEvent_t> ev_in, ev_upd, ev_out;
  cudaEvent_t ev_begin = nullptr;
};

static void patch_free(exa_patch* p) {
  if (p->graph_cfl) cudaGraphExecDestroy(p->graph_cfl);
  if (p->graph_fixed) cudaGraphExecDestroy(p->graph_fixed);
  void* ptrs[] = {p->luh, p->lduh, p->lQhbnd, p->lFhbnd, p->picard, p->cell_grid, p->grid_dx, p->grid_t,
                  p->grid_dt, p->grid_dt_next, p->steps, p->fL, p->fR, p->fdir, p->bcell, p->bface, p->status,
                  p->grid_geo, p->grid_first_d, p->src, p->src_slot, p->src_cells, p->src_vals, p->btype, p->adjQ, p->adjF, p->adj_iter, p->adj_lam};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (cudaEvent_t e : p->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : p->ev_out) cudaEventDestroy(e);
  for (cudaEvent_t e : p->ev_upd) cudaEventDestroy(e);
  if (p->ev_begin) cudaEventDestroy(p->ev_begin);
  if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
  if (p->d2h_stream) cudaStreamDestroy(p->d2h_stream);
  if (p->stream) cudaStreamDestroy(p->stream);
}

static exa::CellArgs patch_args(exa_patch* p) {
  exa::CellArgs a = base_args(p->s, (int)p->ncells);
  a.status = p->status;
  a.luh = p->luh;
  a.luh_out = p->luh;
  a.lduh = p->lduh;
  a.lQhbnd = p->lQhbnd;
  a.lFhbnd = p->lFhbnd;
  a.picard = p->picard;
  a.cell_grid = p->grids.size() > 1 ? p->cell_grid : nullptr;
  a.grid_dx = p->grid_dx;
  a.grid_dt = p->grid_dt;
  a.grid_t = p->grid_t;
  a.grid_geo = p->grid_geo;
  a.grid_first = p->grid_first_d;
  a.src = p->src;
  if (p->src && p->src_slot) {
    a.src_slot = p->src_slot;
    a.src_cells = p->src_cells;
    a.src_vals = p->src_vals;
    a.nsrc = p->nsrc;
  }
  return a;
}

static exa::FaceArgs patch_faces(exa_patch* p) {
  exa::FaceArgs f;
  memset(&f, 0, sizeof(f));
  f.nfaces = p->nfaces;
  f.left = p->fL;
  f.right = p->fR;
  f.dir = p->fdir;
  f.lQhbnd = p->lQhbnd;
  f.lFhbnd = p->lFhbnd;
  f.bcell = p->bcell;
  f.bface = p->bface;
  f.btype = p->btype;
  f.status = p->status;
  f.cell_grid = p->grids.size() > 1 ? p->cell_grid : nullptr;
  f.grid_dx = p->grid_dx;
  f.grid_geo = p->grid_geo;
  f.grid_first = p->grid_first_d;
  f.grid_t = p->grid_t;
  f.grid_dt = p->grid_dt;
  return f;
}

// enqueue one step on p->stream (used for capture)
static int patch_enqueue_step(exa_patch* p, bool cfl) {
  exa::CellArgs a = patch_args(p);
  EXA_CUDA(p->s->ops->predictor(a, p->stream, p->s->cfg.precision == EXA_PREC_MIXED, p->s->pred_variant));
  exa::FaceArgs f = patch_faces(p);
  EXA_CUDA(p->s->ops->riemann(f, p->stream));
  if (p->nbfaces > 0) {
    exa::FaceArgs b = f;
    b.nfaces = p->nbfaces;
    EXA_CUDA(p->s->ops->boundary(b, p->stream));
  }
  exa::CellArgs u = patch_args(p);
  if (cfl) u.grid_dt_next = p->grid_dt_next;
  EXA_CUDA(p->s->ops->update(u, true, true, p->stream, p->s->upd_variant));
  const int ng = (int)p->grids.size();
  if (cfl) {
    exa::advance_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_t, p->grid_dt, p->grid_dt_next, p->steps);
  } else {
    // fixed dt: t += dt, dt unchanged
    exa::advance_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_t, p->grid_dt, nullptr, p->steps);
  }
  EXA_CUDA(cudaGetLastError());
  return EXA_OK;
}

static int patch_graph(exa_patch* p, bool cfl, cudaGraphExec_t* out) {
  if (*out) return EXA_OK;
  cudaGraph_t g = nullptr;
  EXA_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
  int r = patch_enqueue_step(p, cfl);
  cudaError_t e = cudaStreamEndCapture(p->stream, &g);
  if (r != EXA_OK) {
    if (g) cudaGraphDestroy(g);
    return r;
  }
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(out, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  return EXA_OK;
}

namespace {
struct FaceBuild {
  long long ncells = 0, nghost = 0, layer = 0;
  int halo_axis = -1;
  int nhalo_faces = 0;  // faces that touch a ghost cell, at the end of fL / fR / fd
  std::vector<int> cell_grid, fL, fR, bc;
  std::vector<int8_t> fd, bf, bt;
  std::vector<double> dx;
  std::vector<long long> first;
};

// Face lists of a batch of uniform grids: interior faces (left cell, right cell, axis), domain
// faces with a wall (cell, face 2*axis+orientation), and, for EXA_BC_HALO on the last axis of a
// single grid, faces joining the boundary layers to ghost cells appended after the real cells
// (low ghost layer first, then the high one; cell index within a layer as in the grid).
int build_faces(int dim, int ngrids, const exa_grid_desc* grids, FaceBuild& fb) {
  fb.dx.assign(3 * ngrids, 1.0);
  long long c0 = 0;
  for (int g = 0; g < ngrids; g++) {
    const exa_grid_desc& G = grids[g];
    int nc[3] = {G.ncell[0], G.ncell[1], dim == 3 ? G.ncell[2] : 1};
    for (int d = 0; d < dim; d++) {
      if (nc[d] <= 0 || !(G.size[d] > 0)) return fail(EXA_ERR_INVALID, "grid extents must be positive");
      if (G.bc[d] != EXA_BC_PERIODIC && G.bc[d] != EXA_BC_WALL && G.bc[d] != EXA_BC_HALO &&
          G.bc[d] != EXA_BC_OUTFLOW && G.bc[d] != EXA_BC_USER)
        return fail(EXA_ERR_INVALID, "unknown boundary");
      if (G.bc[d] == EXA_BC_HALO && (d != dim - 1 || ngrids != 1))
        return fail(EXA_ERR_INVALID, "EXA_BC_HALO is supported on the last axis of a single-grid patch");
      fb.dx[3 * g + d] = G.size[d] / nc[d];
    }
    const long long n = (long long)nc[0] * nc[1] * nc[2];
    fb.first.push_back(c0);
    c0 += n;
  }
  fb.ncells = c0;
  const bool halo = grids[0].bc[dim - 1] == EXA_BC_HALO;
  if (halo) {
    fb.halo_axis = dim - 1;
    fb.layer = dim == 3 ? (long long)grids[0].ncell[0] * grids[0].ncell[1] : grids[0].ncell[0];
    fb.nghost = 2 * fb.layer;
  }
  if (fb.ncells + fb.nghost > 0x7fffffffLL) return fail(EXA_ERR_INVALID, "too many cells for 32-bit face indices");
  for (int g = 0; g < ngrids; g++) {
    const exa_grid_desc& G = grids[g];
    const long long c0g = fb.first[g];
    int nc[3] = {G.ncell[0], G.ncell[1], dim == 3 ? G.ncell[2] : 1};
    auto idx = [&](int x, int y, int z) { return c0g + ((long long)z * nc[1] + y) * nc[0] + x; };
    auto lidx = [&](int x, int y) { return dim == 3 ? (long long)y * nc[0] + x : (long long)x; };
    for (int d = 0; d < dim; d++)
      for (int z = 0; z < nc[2]; z++)
        for (int y = 0; y < nc[1]; y++)
          for (int x = 0; x < nc[0]; x++) {
            int j[3] = {x, y, z};
            const int i_d = j[d];
            j[d] += 1;
            const long long c = idx(x, y, z);
            if (j[d] == nc[d]) {
              if (G.bc[d] == EXA_BC_PERIODIC) {
                j[d] = 0;
              } else if (G.bc[d] == EXA_BC_WALL || G.bc[d] == EXA_BC_OUTFLOW || G.bc[d] == EXA_BC_USER) {
                fb.bc.push_back((int)c);
                fb.bf.push_back((int8_t)(2 * d + 1));
                fb.bt.push_back((int8_t)G.bc[d]);
              } else {  // halo: the high ghost cell of this column is the right cell
                fb.fL.push_back((int)c);
                fb.fR.push_back((int)(fb.ncells + fb.layer + lidx(x, y)));
                fb.fd.push_back((int8_t)d);
              }
            }
            if (j[d] < nc[d]) {
              fb.fL.push_back((int)c);
              fb.fR.push_back((int)idx(j[0], j[1], j[2]));
              fb.fd.push_back((int8_t)d);
            }
            if (i_d == 0 && (G.bc[d] == EXA_BC_WALL || G.bc[d] == EXA_BC_OUTFLOW || G.bc[d] == EXA_BC_USER)) {
              fb.bc.push_back((int)c);
              fb.bf.push_back((int8_t)(2 * d));
              fb.bt.push_back((int8_t)G.bc[d]);
            }
            if (i_d == 0 && G.bc[d] == EXA_BC_HALO) {  // the low ghost cell is the left cell
              fb.fL.push_back((int)(fb.ncells + lidx(x, y)));
              fb.fR.push_back((int)c);
              fb.fd.push_back((int8_t)d);
            }
          }
    if (ngrids > 1) fb.cell_grid.insert(fb.cell_grid.end(), (size_t)(nc[0] * (long long)nc[1] * nc[2]), g);
  }
  // faces that touch a ghost cell go last (stable), so that the faces between real cells can run
  // while the ghosts' traces are still being exchanged
  if (fb.nghost > 0) {
    std::vector<int> L, R;
    std::vector<int8_t> Dd;
    for (int pass = 0; pass < 2; pass++)
      for (size_t k = 0; k < fb.fL.size(); k++) {
        const bool ghost = fb.fL[k] >= fb.ncells || fb.fR[k] >= fb.ncells;
        if (ghost != (pass == 1)) continue;
        L.push_back(fb.fL[k]);
        R.push_back(fb.fR[k]);
        Dd.push_back(fb.fd[k]);
        if (ghost) fb.nhalo_faces++;
      }
    fb.fL.swap(L);
    fb.fR.swap(R);
    fb.fd.swap(Dd);
  }
  return EXA_OK;
}
}  // namespace

extern "C" int exa_build_face_lists(int dim, int ngrids, const exa_grid_desc* grids, exa_face_lists* out) {
  if (!grids || !out || ngrids <= 0 || (dim != 2 && dim != 3)) return fail(EXA_ERR_INVALID, "bad argument");
  FaceBuild fb;
  if (int r = build_faces(dim, ngrids, grids, fb)) return r;
  const bool fill = out->left != nullptr;
  if (fill && (out->nfaces < (int)fb.fL.size() || out->nbfaces < (int)fb.bc.size()))
    return fail(EXA_ERR_INVALID, "face arrays too small");
  out->ncells = fb.ncells;
  out->nghost = fb.nghost;
  out->nfaces = (int)fb.fL.size();
  out->nbfaces = (int)fb.bc.size();
  if (fill) {
    std::copy(fb.fL.begin(), fb.fL.end(), out->left);
    std::copy(fb.fR.begin(), fb.fR.end(), out->right);
    std::copy(fb.fd.begin(), fb.fd.end(), reinterpret_cast<int8_t*>(out->dir));
    if (out->bcell) std::copy(fb.bc.begin(), fb.bc.end(), out->bcell);
    if (out->bface) std::copy(fb.bf.begin(), fb.bf.end(), reinterpret_cast<int8_t*>(out->bface));
  }
  return EXA_OK;
}

extern "C" {

int exa_patch_create(exa_solver* s, int ngrids, const exa_grid_desc* grids, exa_patch** out) {
  if (!s || !grids || !out || ngrids <= 0) return fail(EXA_ERR_INVALID, "bad argument");
  *out = nullptr;
  const int dim = s->cfg.dim;
  std::unique_ptr<exa_patch> p(new exa_patch());
  p->s = s;
  p->grids.assign(grids, grids + ngrids);
  FaceBuild fb;
  if (int r = build_faces(dim, ngrids, grids, fb)) return r;
  for (int8_t t : fb.bt) {
    if (t == EXA_BC_USER && !s->ops->user_bc_ok)
      return fail(EXA_ERR_UNSUPPORTED, "EXA_BC_USER needs a PDE functor with boundary_values");
    if (t == EXA_BC_USER) p->has_user_bc = true;
  }
  std::vector<int>& hcell_grid = fb.cell_grid;
  std::vector<int>& fL = fb.fL;
  std::vector<int>& fR = fb.fR;
  std::vector<int>& bc = fb.bc;
  std::vector<int8_t>& fd = fb.fd;
  std::vector<int8_t>& bf = fb.bf;
  std::vector<double>& hdx = fb.dx;
  p->grid_first = fb.first;
  p->ncells = fb.ncells;
  p->nghost = fb.nghost;
  p->halo_axis = fb.halo_axis;
  p->layer = fb.layer;
  if (fb.halo_axis >= 0) {
    p->halo_lo_first = 0;
    p->halo_hi_first = fb.ncells - fb.layer;
  }
  p->nfaces = (int)fL.size();
  p->nhalo_faces = fb.nhalo_faces;
  p->nbfaces = (int)bc.size();
  exa::Ops& o = *s->ops;
  const long long nc = p->ncells;
  auto alloc = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 8);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    return EXA_OK;
  };
  int r = EXA_OK;
#define EXA_ALLOC(ptr, bytes)                          \
  if ((r = alloc((void**)&(ptr), (bytes))) != EXA_OK) { \
    patch_free(p.get());                               \
    return r;                                          \
  }
  EXA_ALLOC(p->luh, nc * o.sz_luh * sizeof(double));
  EXA_ALLOC(p->lduh, nc * o.sz_lduh * sizeof(double));
  EXA_ALLOC(p->lQhbnd, (nc + p->nghost) * o.sz_qhb * sizeof(double));
  EXA_ALLOC(p->lFhbnd, (nc + p->nghost) * o.sz_fhb * sizeof(double));
  EXA_ALLOC(p->picard, nc * sizeof(int));
  EXA_ALLOC(p->grid_dx, 3 * ngrids * sizeof(double));
  EXA_ALLOC(p->grid_t, ngrids * sizeof(double));
  EXA_ALLOC(p->grid_dt, ngrids * sizeof(double));
  EXA_ALLOC(p->grid_dt_next, ngrids * sizeof(double));
  EXA_ALLOC(p->steps, sizeof(long long));
  EXA_ALLOC(p->status, sizeof(unsigned));
  EXA_ALLOC(p->fL, fL.size() * sizeof(int));
  EXA_ALLOC(p->fR, fR.size() * sizeof(int));
  EXA_ALLOC(p->fdir, fd.size());
  EXA_ALLOC(p->bcell, bc.size() * sizeof(int));
  EXA_ALLOC(p->bface, bf.size());
  if (ngrids > 1) EXA_ALLOC(p->cell_grid, hcell_grid.size() * sizeof(int));
  EXA_ALLOC(p->grid_geo, 6 * ngrids * sizeof(double));
  EXA_ALLOC(p->grid_first_d, ngrids * sizeof(long long));
  EXA_ALLOC(p->btype, fb.bt.size() + 1);
#undef EXA_ALLOC
  cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    patch_free(p.get());
    return cuda_fail(e, "cudaStreamCreate");
  }
  std::vector<double> zeros(ngrids, 0.0);
  std::vector<double> geo(6 * ngrids);
  for (int g = 0; g < ngrids; g++)
    for (int k = 0; k < 3; k++) {
      geo[6 * g + k] = grids[g].offset[k];
      geo[6 * g + 3 + k] = (k < dim) ? grids[g].ncell[k] : 1;
    }
  bool ok = cudaMemcpy(p->grid_geo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(p->grid_first_d, fb.first.data(), ngrids * sizeof(long long), cudaMemcpyHostToDevice) ==
                cudaSuccess &&
            (fb.bt.empty() || cudaMemcpy(p->btype, fb.bt.data(), fb.bt.size(), cudaMemcpyHostToDevice) == cudaSuccess);
  ok = ok && cudaMemcpy(p->grid_dx, hdx.data(), hdx.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(p->grid_t, zeros.data(), ngrids * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemcpy(p->grid_dt, zeros.data(), ngrids * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
            cudaMemset(p->steps, 0, sizeof(long long)) == cudaSuccess &&
            cudaMemset(p->status, 0, sizeof(unsigned)) == cudaSuccess &&
            cudaMemset(p->luh, 0, nc * o.sz_luh * sizeof(double)) == cudaSuccess &&
            cudaMemset(p->picard, 0, nc * sizeof(int)) == cudaSuccess &&
            (fL.empty() || (cudaMemcpy(p->fL, fL.data(), fL.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
                            cudaMemcpy(p->fR, fR.data(), fR.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
                            cudaMemcpy(p->fdir, fd.data(), fd.size(), cudaMemcpyHostToDevice) == cudaSuccess)) &&
            (bc.empty() || (cudaMemcpy(p->bcell, bc.data(), bc.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
                            cudaMemcpy(p->bface, bf.data(), bf.size(), cudaMemcpyHostToDevice) == cudaSuccess)) &&
            (ngrids == 1 || cudaMemcpy(p->cell_grid, hcell_grid.data(), hcell_grid.size() * sizeof(int),
                                       cudaMemcpyHostToDevice) == cudaSuccess);
  if (!ok) {
    patch_free(p.get());
    return cuda_fail(cudaGetLastError(), "patch upload");
  }
  // the streamed predictor's scratch must exist before a step is captured into a graph
  e = o.reserve(p->ncells);
  if (e != cudaSuccess) {
    patch_free(p.get());
    return cuda_fail(e, "predictor scratch");
  }
  *out = p.release();
  return EXA_OK;
}

int exa_patch_destroy(exa_patch* p) {
  if (!p) return EXA_OK;
  cudaStreamSynchronize(p->stream);
  patch_free(p);
  delete p;
  return EXA_OK;
}

long long exa_patch_num_cells(const exa_patch* p) { return p ? p->ncells : -1; }
double* exa_patch_luh(exa_patch* p) { return p ? p->luh : nullptr; }
void* exa_patch_stream(exa_patch* p) { return p ? (void*)p->stream : nullptr; }

static int patch_initial_dt(exa_patch* p) {
  const int ng = (int)p->grids.size();
  exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_dt, INFINITY);
  exa::CellArgs a = patch_args(p);
  a.grid_dt_next = p->grid_dt;
  EXA_CUDA(p->s->ops->update(a, false, false, p->stream));
  exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_dt_next, INFINITY);
  EXA_CUDA(cudaGetLastError());
  return EXA_OK;
}

int exa_patch_set_solution(exa_patch* p, const double* luh, int on_device) {
  if (!p || !luh) return fail(EXA_ERR_INVALID, "null argument");
  const size_t bytes = (size_t)p->ncells * p->s->ops->sz_luh * sizeof(double);
  EXA_CUDA(cudaMemcpyAsync(p->luh, luh, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                           p->stream));
  int r = patch_initial_dt(p);
  if (r) return r;
  // grid_dt now holds the CFL step of the new state: a following fixed-dt step must refill it
  p->fixed_dt = -1.0;
  // first state on this device: time the predictor variants on it (halo patches: real cells only)
  if (p->s->pred_variant < 0) {
    exa::CellArgs a = patch_args(p);
    EXA_CUDA(p->s->ops->tune(a, p->stream, p->s->cfg.precision == EXA_PREC_MIXED));
  }
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

int exa_patch_get_solution(exa_patch* p, double* luh, int on_device) {
  if (!p || !luh) return fail(EXA_ERR_INVALID, "null argument");
  const size_t bytes = (size_t)p->ncells * p->s->ops->sz_luh * sizeof(double);
  EXA_CUDA(cudaMemcpyAsync(luh, p->luh, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           p->stream));
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

int exa_patch_step(exa_patch* p, int nsteps, double fixed_dt) {
  if (!p || nsteps < 0) return fail(EXA_ERR_INVALID, "bad argument");
  if (p->halo_axis >= 0)
    return fail(EXA_ERR_INVALID, "a patch with EXA_BC_HALO steps through exa_patch_step_phase and a halo exchange");
  const bool cfl = !(fixed_dt > 0);
  if (!cfl && fixed_dt != p->fixed_dt) {
    const int ng = (int)p->grids.size();
    exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_dt, fixed_dt);
    EXA_CUDA(cudaGetLastError());
    p->fixed_dt = fixed_dt;
  }
  if (cfl && p->fixed_dt > 0) {
    // back from fixed steps: recompute the CFL dt of the current state
    if (int r = patch_initial_dt(p)) return r;
    p->fixed_dt = -1.0;
  }
  cudaGraphExec_t* g = cfl ? &p->graph_cfl : &p->graph_fixed;
  if (int r = patch_graph(p, cfl, g)) return r;
  for (int i = 0; i < nsteps; i++) EXA_CUDA(cudaGraphLaunch(*g, p->stream));
  return EXA_OK;
}

int exa_patch_sync(exa_patch* p) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

int exa_patch_time(exa_patch* p, double* t, double* dt) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  const size_t ng = p->grids.size();
  if (t) EXA_CUDA(cudaMemcpyAsync(t, p->grid_t, ng * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  if (dt) EXA_CUDA(cudaMemcpyAsync(dt, p->grid_dt, ng * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

int exa_patch_track_picard(exa_patch* p, int on) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  p->track_picard = on != 0;
  return EXA_OK;
}

int exa_patch_stats_get(exa_patch* p, exa_patch_stats* st) {
  if (!p || !st) return fail(EXA_ERR_INVALID, "null argument");
  memset(st, 0, sizeof(*st));
  EXA_CUDA(cudaMemcpyAsync(&st->steps, p->steps, sizeof(long long), cudaMemcpyDeviceToHost, p->stream));
  std::vector<int> pic((size_t)p->ncells);
  EXA_CUDA(cudaMemcpyAsync(pic.data(), p->picard, pic.size() * sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  double sum = 0;
  for (int v : pic) {
    sum += v;
    st->picard_hist[std::min(std::max(v, 0), 31)]++;
  }
  st->picard_mean = pic.empty() ? 0.0 : sum / pic.size();
  return EXA_OK;
}

int exa_patch_status(exa_patch* p, unsigned* bits) {
  if (!p || !bits) return fail(EXA_ERR_INVALID, "null argument");
  EXA_CUDA(cudaMemcpyAsync(bits, p->status, sizeof(unsigned), cudaMemcpyDeviceToHost, p->stream));
  EXA_CUDA(cudaMemsetAsync(p->status, 0, sizeof(unsigned), p->stream));
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// step phases and halo exchange support (slab decomposition across devices)
// ------------------------------------------------------------------------------------------
extern "C" {

int exa_patch_step_phase(exa_patch* p, int phase, double fixed_dt) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  const bool cfl = !(fixed_dt > 0);
  const int ng = (int)p->grids.size();
  if (!cfl && fixed_dt != p->fixed_dt) {
    exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_dt, fixed_dt);
    EXA_CUDA(cudaGetLastError());
    p->fixed_dt = fixed_dt;
  }
  switch (phase) {
    case EXA_PHASE_PREDICTOR: {
      exa::CellArgs a = patch_args(p);
      EXA_CUDA(p->s->ops->predictor(a, p->stream, p->s->cfg.precision == EXA_PREC_MIXED, p->s->pred_variant));
      return EXA_OK;
    }
    case EXA_PHASE_FACES:
    case EXA_PHASE_FACES_INTERIOR:
    case EXA_PHASE_FACES_HALO: {
      exa::FaceArgs f = patch_faces(p);
      const int ninner = p->nfaces - p->nhalo_faces;
      if (phase == EXA_PHASE_FACES_INTERIOR) f.nfaces = ninner;
      if (phase == EXA_PHASE_FACES_HALO) {
        f.nfaces = p->nhalo_faces;
        f.left += ninner;
        f.right += ninner;
        f.dir += ninner;
      }
      EXA_CUDA(p->s->ops->riemann(f, p->stream));
      if (p->nbfaces > 0 && phase != EXA_PHASE_FACES_HALO) {
        exa::FaceArgs b = patch_faces(p);
        b.nfaces = p->nbfaces;
        EXA_CUDA(p->s->ops->boundary(b, p->stream));
      }
      return EXA_OK;
    }
    case EXA_PHASE_UPDATE: {
      exa::CellArgs u = patch_args(p);
      if (cfl) u.grid_dt_next = p->grid_dt_next;
      EXA_CUDA(p->s->ops->update(u, true, true, p->stream, p->s->upd_variant));
      return EXA_OK;
    }
    case EXA_PHASE_ADVANCE: {
      exa::advance_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_t, p->grid_dt,
                                                                   cfl ? p->grid_dt_next : nullptr, p->steps);
      EXA_CUDA(cudaGetLastError());
      return EXA_OK;
    }
    default:
      return fail(EXA_ERR_INVALID, "unknown phase");
  }
}

long long exa_patch_halo_doubles(const exa_patch* p) {
  if (!p || p->halo_axis < 0) return 0;
  const exa::Ops& o = *p->s->ops;
  const int nfaces = 2 * o.dim;
  return p->layer * (long long)(o.sz_qhb / nfaces + o.sz_fhb / nfaces);
}

// one side's face traces: [Q of every layer cell][F of every layer cell]; 2D-pitched copies
static int halo_copy(exa_patch* p, long long first_cell, int face, double* buf, bool to_buf) {
  const exa::Ops& o = *p->s->ops;
  const size_t fq = o.sz_qhb / (2 * o.dim), ff = o.sz_fhb / (2 * o.dim);
  double* q = p->lQhbnd + first_cell * o.sz_qhb + face * fq;
  double* f = p->lFhbnd + first_cell * o.sz_fhb + face * ff;
  double* bq = buf;
  double* bfl = buf + p->layer * fq;
  if (to_buf) {
    EXA_CUDA(cudaMemcpy2DAsync(bq, fq * sizeof(double), q, o.sz_qhb * sizeof(double), fq * sizeof(double),
                               (size_t)p->layer, cudaMemcpyDeviceToDevice, p->stream));
    EXA_CUDA(cudaMemcpy2DAsync(bfl, ff * sizeof(double), f, o.sz_fhb * sizeof(double), ff * sizeof(double),
                               (size_t)p->layer, cudaMemcpyDeviceToDevice, p->stream));
  } else {
    EXA_CUDA(cudaMemcpy2DAsync(q, o.sz_qhb * sizeof(double), bq, fq * sizeof(double), fq * sizeof(double),
                               (size_t)p->layer, cudaMemcpyDeviceToDevice, p->stream));
    EXA_CUDA(cudaMemcpy2DAsync(f, o.sz_fhb * sizeof(double), bfl, ff * sizeof(double), ff * sizeof(double),
                               (size_t)p->layer, cudaMemcpyDeviceToDevice, p->stream));
  }
  return EXA_OK;
}

int exa_patch_halo_pack(exa_patch* p, double* send_lo, double* send_hi) {
  if (!p || p->halo_axis < 0) return fail(EXA_ERR_INVALID, "patch has no halo");
  if (!send_lo || !send_hi) return fail(EXA_ERR_INVALID, "null buffer");
  const int a = p->halo_axis;
  // low real layer, its low face 2a; high real layer, its high face 2a+1
  if (int r = halo_copy(p, p->halo_lo_first, 2 * a, send_lo, true)) return r;
  return halo_copy(p, p->halo_hi_first, 2 * a + 1, send_hi, true);
}

int exa_patch_halo_unpack(exa_patch* p, const double* recv_lo, const double* recv_hi) {
  if (!p || p->halo_axis < 0) return fail(EXA_ERR_INVALID, "patch has no halo");
  if (!recv_lo || !recv_hi) return fail(EXA_ERR_INVALID, "null buffer");
  const int a = p->halo_axis;
  // recv_lo: the lower neighbour's high layer (face 2a+1) -> low ghost cells, face 2a+1
  // recv_hi: the upper neighbour's low layer (face 2a)    -> high ghost cells, face 2a
  if (int r = halo_copy(p, p->ncells, 2 * a + 1, const_cast<double*>(recv_lo), false)) return r;
  return halo_copy(p, p->ncells + p->layer, 2 * a, const_cast<double*>(recv_hi), false);
}

int exa_patch_set_point_source(exa_patch* p, const exa_point_source* src) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  if (!src) {
    EXA_CUDA(cudaStreamSynchronize(p->stream));
    if (p->src) cudaFree(p->src);
    p->src = nullptr;
  } else {
    if (src->variable < 0 || src->variable >= p->s->ops->nvar) return fail(EXA_ERR_INVALID, "source variable");
    if (!(src->width > 0)) return fail(EXA_ERR_INVALID, "source width must be positive");
    if (!p->src) EXA_CUDA(cudaMalloc(&p->src, 8 * sizeof(double)));
    const double h[8] = {src->x[0], src->x[1], src->x[2], src->f0, src->t0, src->amplitude, src->width,
                         (double)src->variable};
    // ordered after any step still running on the patch's stream
    EXA_CUDA(cudaMemcpyAsync(p->src, h, sizeof(h), cudaMemcpyHostToDevice, p->stream));
    // the cells the source reaches, and room for its values at their nodes
    exa::Ops& o = *p->s->ops;
    if (!p->src_slot) {
      EXA_CUDA(cudaMalloc(&p->src_slot, (size_t)std::max<long long>(p->ncells, 1) * sizeof(int)));
      EXA_CUDA(cudaMalloc(&p->src_cells, (size_t)std::max<long long>(p->ncells, 1) * sizeof(int) + sizeof(int)));
    }
    int* d_count = p->src_cells + std::max<long long>(p->ncells, 1);
    EXA_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), p->stream));
    exa::CellArgs a = patch_args(p);
    EXA_CUDA(o.source_slots(a, p->src_slot, p->src_cells, d_count, p->stream));
    int nsrc = 0;
    EXA_CUDA(cudaMemcpyAsync(&nsrc, d_count, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    EXA_CUDA(cudaStreamSynchronize(p->stream));
    const size_t per = (size_t)o.nd * (o.order + 1);
    if (nsrc > p->nsrc || !p->src_vals) {
      if (p->src_vals) cudaFree(p->src_vals);
      p->src_vals = nullptr;
      EXA_CUDA(cudaMalloc(&p->src_vals, (size_t)std::max(nsrc, 1) * per * sizeof(double)));
    }
    p->nsrc = nsrc;
  }
  // the captured step graphs hold the old pointer: rebuild them on the next step
  if (p->graph_cfl) cudaGraphExecDestroy(p->graph_cfl);
  if (p->graph_fixed) cudaGraphExecDestroy(p->graph_fixed);
  p->graph_cfl = p->graph_fixed = nullptr;
  return EXA_OK;
}

int exa_patch_adjust_solution(exa_patch* p) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  if (!p->s->ops->adjust_ok) return fail(EXA_ERR_UNSUPPORTED, "the PDE functor has no adjust_point_solution");
  exa::CellArgs a = patch_args(p);
  a.luh_out = p->luh;
  EXA_CUDA(p->s->ops->adjust(a, p->stream));
  if (int r = patch_initial_dt(p)) return r;
  p->fixed_dt = -1.0;
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

int exa_patch_dt_copy(exa_patch* p, double* dev_buf, int to_patch) {
  if (!p || !dev_buf) return fail(EXA_ERR_INVALID, "null argument");
  const size_t bytes = p->grids.size() * sizeof(double);
  if (to_patch)
    EXA_CUDA(cudaMemcpyAsync(p->grid_dt, dev_buf, bytes, cudaMemcpyDeviceToDevice, p->stream));
  else
    EXA_CUDA(cudaMemcpyAsync(dev_buf, p->grid_dt, bytes, cudaMemcpyDeviceToDevice, p->stream));
  return EXA_OK;
}

int exa_patch_dt_next_copy(exa_patch* p, double* dev_buf, int to_patch) {
  if (!p || !dev_buf) return fail(EXA_ERR_INVALID, "null argument");
  const size_t bytes = p->grids.size() * sizeof(double);
  if (to_patch)
    EXA_CUDA(cudaMemcpyAsync(p->grid_dt_next, dev_buf, bytes, cudaMemcpyDeviceToDevice, p->stream));
  else
    EXA_CUDA(cudaMemcpyAsync(dev_buf, p->grid_dt_next, bytes, cudaMemcpyDeviceToDevice, p->stream));
  return EXA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Allocation-free CFL time step (exa_stable_time_step_size_noalloc). No counterpart in the
// reference. Its scratch -- the per-cell time steps, the minimum and a status word -- lives in
// one file-scope device array instead of memory obtained from cudaMalloc. Every GPU that loads
// this library holds the array (8 MiB + 256 B) until the process exits.
// ------------------------------------------------------------------------------------------
namespace {

constexpr int kNoallocHead = 32;  // doubles before the per-cell area: [0] minimum, [1] status bits
static __device__ __align__(256) double g_exa_cfl_scratch[kNoallocHead + EXA_NOALLOC_MAX_CELLS];
// device address of g_exa_cfl_scratch per device ordinal, looked up on the first call on a device
std::atomic<double*> g_cfl_scratch_addr[64];

int noalloc_scratch(double** out) {
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(EXA_ERR_INVALID, "device ordinal >= 64 not supported by the scratch table");
  double* p = g_cfl_scratch_addr[dev].load();
  if (!p) {
    // the host-side name g_exa_cfl_scratch is only a stand-in: the kernels need the device address
    void* addr = nullptr;
    EXA_CUDA(cudaGetSymbolAddress(&addr, g_exa_cfl_scratch));
    p = static_cast<double*>(addr);
    g_cfl_scratch_addr[dev].store(p);
  }
  *out = p;
  return EXA_OK;
}

}  // namespace

extern "C" int exa_stable_time_step_size_noalloc(const exa_solver_config* cfg, int ncells, const double* luh,
                                                 const double* dx, double* cell_dt, double* dt_min, void* stream) {
  if (!cfg || !dx || (ncells > 0 && !luh)) return fail(EXA_ERR_INVALID, "null argument");
  if (ncells < 0) return fail(EXA_ERR_INVALID, "ncells < 0");
  if (ncells > EXA_NOALLOC_MAX_CELLS)
    return fail(EXA_ERR_INVALID, "ncells = " + std::to_string(ncells) +
                                     " exceeds EXA_NOALLOC_MAX_CELLS = " + std::to_string(EXA_NOALLOC_MAX_CELLS) +
                                     "; use exa_stable_time_step_size for larger batches");
  if (cfg->dim != 2 && cfg->dim != 3) return fail(EXA_ERR_INVALID, "dim must be 2 or 3");
  exa::Ops* ops = exa::find_ops(cfg->pde, cfg->dim, cfg->order, cfg->npar);
  if (!ops) return fail(EXA_ERR_UNSUPPORTED, "no kernel instantiation for this configuration");
  double* scratch = nullptr;
  if (int e = noalloc_scratch(&scratch)) return e;
  cudaStream_t st = (cudaStream_t)stream;
  double* d_min = scratch;
  unsigned* d_status = reinterpret_cast<unsigned*>(scratch + 1);
  double* d_cell = scratch + kNoallocHead;
  // the array keeps the previous call's contents: reset the minimum and the status word
  exa::fill_kernel<<<1, 32, 0, st>>>(1, d_min, INFINITY);
  exa::fill_kernel<<<1, 32, 0, st>>>(1, scratch + 1, 0.0);
  EXA_CUDA(cudaGetLastError());
  if (ncells > 0) {
    exa::CellArgs a;
    memset(&a, 0, sizeof(a));
    a.ncells = ncells;
    a.luh = luh;
    a.cell_dt = d_cell;
    a.grid_dt_next = d_min;  // every cell counts as grid 0: per-cell minima atomic-min into d_min
    a.status = d_status;
    a.pnpm = cfg->pnpm > 0 ? cfg->pnpm : default_pnpm(cfg->order);
    a.cfl_pnpm = (cfg->cfl > 0 ? cfg->cfl : 0.9) * a.pnpm;
    for (int d = 0; d < 3; d++) a.u_dx[d] = d < cfg->dim ? dx[d] : 1.0;
    EXA_CUDA(ops->update(a, false, false, st));
    if (cell_dt) EXA_CUDA(cudaMemcpyAsync(cell_dt, d_cell, sizeof(double) * ncells, cudaMemcpyDeviceToDevice, st));
  }
  unsigned bits = 0;
  if (dt_min) {
    EXA_CUDA(cudaMemcpyAsync(dt_min, d_min, sizeof(double), cudaMemcpyDeviceToHost, st));
    EXA_CUDA(cudaMemcpyAsync(&bits, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    EXA_CUDA(cudaStreamSynchronize(st));
    if (bits) return fail(EXA_ERR_NUMERICS, "non-finite state or non-positive dt (status bits " +
                                                std::to_string(bits) + ")");
  }
  return EXA_OK;
}

// ------------------------------------------------------------------------------------------
// discrete adjoint of one step (linear acoustic / elastic systems)
// ------------------------------------------------------------------------------------------
extern "C" {

int exa_patch_set_time(exa_patch* p, double t) {
  if (!p) return fail(EXA_ERR_INVALID, "null patch");
  const int ng = (int)p->grids.size();
  exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_t, t);
  EXA_CUDA(cudaGetLastError());
  return EXA_OK;
}

}  // extern "C"

// checks and workspace of an adjoint step; the face-trace adjoints cover the ghost cells too
static int adjoint_prepare(exa_patch* p, double dt) {
  exa::Ops& o = *p->s->ops;
  if (!o.adjoint_ok) return fail(EXA_ERR_UNSUPPORTED, "the adjoint is built for the acoustic and elastic systems");
  const int S = p->s->cfg.max_picard;
  if (S <= 0) return fail(EXA_ERR_UNSUPPORTED, "the adjoint needs a fixed Picard sweep count (max_picard > 0)");
  if (p->s->cfg.precision != EXA_PREC_FP64) return fail(EXA_ERR_UNSUPPORTED, "the adjoint runs in FP64");
  if (p->has_user_bc) return fail(EXA_ERR_UNSUPPORTED, "the adjoint supports periodic, wall and outflow faces");
  if (!(dt > 0)) return fail(EXA_ERR_INVALID, "the adjoint needs the fixed time step of the forward step");
  const size_t nc = (size_t)p->ncells, nt = nc + (size_t)p->nghost;
  if (!p->adjQ) EXA_CUDA(cudaMalloc(&p->adjQ, nt * o.sz_qhb * sizeof(double)));
  if (!p->adjF) EXA_CUDA(cudaMalloc(&p->adjF, nt * o.sz_fhb * sizeof(double)));
  if (!p->adj_iter) EXA_CUDA(cudaMalloc(&p->adj_iter, nc * (size_t)S * o.sz_lQi / (o.nvar + o.npar) * o.nvar * sizeof(double)));
  if (p->nghost > 0 && !p->adj_lam) EXA_CUDA(cudaMalloc(&p->adj_lam, nt * o.sz_luh * sizeof(double)));
  const int ng = (int)p->grids.size();
  if (dt != p->fixed_dt) {
    exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_dt, dt);
    EXA_CUDA(cudaGetLastError());
    p->fixed_dt = dt;
  }
  return EXA_OK;
}

// forward predictor at u_k: the face traces the Rusanov adjoint linearises around, and the Picard
// iterates the reverse sweeps need (written into the adjoint scratch)
static int adjoint_forward(exa_patch* p) {
  exa::CellArgs c = patch_args(p);
  c.ex_iter = p->adj_iter;
  EXA_CUDA(p->s->ops->predictor(c, p->stream, false, p->s->pred_variant));
  return EXA_OK;
}

// transposed faces (interior, halo and domain) and transposed predictors; lam holds the real
// cells' lambda, followed by the ghost cells' on a halo patch
static int adjoint_reverse(exa_patch* p, double* lam) {
  exa::AdjArgs a;
  a.c = patch_args(p);
  a.f = patch_faces(p);
  a.fb = a.f;
  a.fb.nfaces = p->nbfaces;
  a.lam = lam;
  a.adjQ = p->adjQ;
  a.adjF = p->adjF;
  a.iter = p->adj_iter;
  a.sweeps = p->s->cfg.max_picard;
  a.have_iter = 1;
  EXA_CUDA(p->s->ops->adjoint(a, p->stream));
  return EXA_OK;
}

extern "C" {

int exa_patch_adjoint_step(exa_patch* p, double* lambda, double dt) {
  if (!p || !lambda) return fail(EXA_ERR_INVALID, "null argument");
  if (p->halo_axis >= 0)
    return fail(EXA_ERR_INVALID, "a patch with EXA_BC_HALO runs the adjoint through exa_patch_adjoint_phase "
                                 "and a halo exchange");
  if (int r = adjoint_prepare(p, dt)) return r;
  if (int r = adjoint_forward(p)) return r;
  return adjoint_reverse(p, lambda);
}

int exa_patch_adjoint_phase(exa_patch* p, int phase, double* lambda, double dt) {
  if (!p || !lambda) return fail(EXA_ERR_INVALID, "null argument");
  const exa::Ops& o = *p->s->ops;
  const size_t bytes = (size_t)p->ncells * o.sz_luh * sizeof(double);
  if (phase == EXA_ADJ_FORWARD) {
    if (int r = adjoint_prepare(p, dt)) return r;
    if (int r = adjoint_forward(p)) return r;
    if (p->nghost > 0) {
      EXA_CUDA(cudaMemcpyAsync(p->adj_lam, lambda, bytes, cudaMemcpyDeviceToDevice, p->stream));
      // the ghost cells' lambda is zero until exa_patch_adjoint_halo_unpack delivers the neighbours'
      EXA_CUDA(cudaMemsetAsync(p->adj_lam + (size_t)p->ncells * o.sz_luh, 0,
                               (size_t)p->nghost * o.sz_luh * sizeof(double), p->stream));
    }
    p->adj_forward_done = true;
    return EXA_OK;
  }
  if (phase != EXA_ADJ_REVERSE) return fail(EXA_ERR_INVALID, "unknown adjoint phase");
  if (!p->adj_forward_done) return fail(EXA_ERR_INVALID, "EXA_ADJ_REVERSE needs EXA_ADJ_FORWARD first");
  if (dt != p->fixed_dt) return fail(EXA_ERR_INVALID, "EXA_ADJ_REVERSE needs the time step of EXA_ADJ_FORWARD");
  p->adj_forward_done = false;
  if (p->nghost == 0) return adjoint_reverse(p, lambda);
  if (int r = adjoint_reverse(p, p->adj_lam)) return r;
  EXA_CUDA(cudaMemcpyAsync(lambda, p->adj_lam, bytes, cudaMemcpyDeviceToDevice, p->stream));
  return EXA_OK;
}

long long exa_patch_adjoint_halo_doubles(const exa_patch* p) {
  if (!p || p->halo_axis < 0) return 0;
  return p->layer * (long long)p->s->ops->sz_luh;
}

int exa_patch_adjoint_halo_pack(exa_patch* p, double* send_lo, double* send_hi) {
  if (!p || p->halo_axis < 0) return fail(EXA_ERR_INVALID, "patch has no halo");
  if (!send_lo || !send_hi) return fail(EXA_ERR_INVALID, "null buffer");
  if (!p->adj_forward_done) return fail(EXA_ERR_INVALID, "pack lambda between EXA_ADJ_FORWARD and EXA_ADJ_REVERSE");
  const size_t blk = (size_t)p->s->ops->sz_luh, bytes = (size_t)p->layer * blk * sizeof(double);
  // the low and the high layer of real cells: lambda of u_{k+1}, as EXA_ADJ_FORWARD took it
  EXA_CUDA(cudaMemcpyAsync(send_lo, p->adj_lam + (size_t)p->halo_lo_first * blk, bytes, cudaMemcpyDeviceToDevice,
                           p->stream));
  EXA_CUDA(cudaMemcpyAsync(send_hi, p->adj_lam + (size_t)p->halo_hi_first * blk, bytes, cudaMemcpyDeviceToDevice,
                           p->stream));
  return EXA_OK;
}

int exa_patch_adjoint_halo_unpack(exa_patch* p, const double* recv_lo, const double* recv_hi) {
  if (!p || p->halo_axis < 0) return fail(EXA_ERR_INVALID, "patch has no halo");
  if (!recv_lo || !recv_hi) return fail(EXA_ERR_INVALID, "null buffer");
  if (!p->adj_forward_done) return fail(EXA_ERR_INVALID, "unpack lambda between EXA_ADJ_FORWARD and EXA_ADJ_REVERSE");
  const size_t blk = (size_t)p->s->ops->sz_luh, bytes = (size_t)p->layer * blk * sizeof(double);
  // recv_lo: the lower neighbour's high layer -> low ghost cells; recv_hi: the upper one's low layer
  EXA_CUDA(cudaMemcpyAsync(p->adj_lam + (size_t)p->ncells * blk, recv_lo, bytes, cudaMemcpyDeviceToDevice,
                           p->stream));
  EXA_CUDA(cudaMemcpyAsync(p->adj_lam + ((size_t)p->ncells + p->layer) * blk, recv_hi, bytes,
                           cudaMemcpyDeviceToDevice, p->stream));
  return EXA_OK;
}

}  // extern "C"

extern "C" {

int exa_checkpoint_schedule(int steps, int snaps, exa_ck_action* out, int capacity, int* count,
                            long long* forward_steps) {
  if (steps < 1 || snaps < 1 || !count) return fail(EXA_ERR_INVALID, "steps and snaps must be >= 1");
  if (steps > 8192) return fail(EXA_ERR_INVALID, "at most 8192 steps per schedule (chain schedules for more)");
  const int free_slots = std::min(snaps - 1, steps);
  exa_ck::Planner plan(steps, free_slots);
  const std::vector<exa_ck::Action> acts = plan.schedule();
  *count = (int)acts.size();
  long long fw = 0;
  for (const auto& x : acts)
    if (x.action == exa_ck::ADVANCE) fw += x.b - x.a;
  if (forward_steps) *forward_steps = fw;
  if (!out) return EXA_OK;
  if (capacity < (int)acts.size()) return fail(EXA_ERR_INVALID, "capacity below the schedule length");
  for (size_t i = 0; i < acts.size(); i++) {
    out[i].action = acts[i].action;
    out[i].a = acts[i].a;
    out[i].b = acts[i].b;
  }
  return EXA_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// one step from and to host memory, copies overlapped with the cell kernels
// ------------------------------------------------------------------------------------------
extern "C" {

int exa_patch_run_host(exa_patch* p, const double* luh_in, double* luh_out, int nsteps, double fixed_dt) {
  if (!p || !luh_in || !luh_out || nsteps < 0) return fail(EXA_ERR_INVALID, "bad argument");
  if (p->halo_axis >= 0) return fail(EXA_ERR_INVALID, "a patch with EXA_BC_HALO steps through exa_patch_step_phase");
  if (nsteps == 0) return EXA_OK;
  exa::Ops& o = *p->s->ops;
  const int ng = (int)p->grids.size();
  const bool cfl = !(fixed_dt > 0);
  const long long nc = p->ncells;
  const int K = (int)std::max<long long>(1, std::min<long long>(kHostChunks, nc));
  if (!p->copy_stream) {
    EXA_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    EXA_CUDA(cudaStreamCreateWithFlags(&p->d2h_stream, cudaStreamNonBlocking));
    EXA_CUDA(cudaEventCreateWithFlags(&p->ev_begin, cudaEventDisableTiming));
  }
  while ((int)p->ev_in.size() < K) {
    cudaEvent_t a, b, c;
    EXA_CUDA(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    EXA_CUDA(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    EXA_CUDA(cudaEventCreateWithFlags(&c, cudaEventDisableTiming));
    p->ev_in.push_back(a);
    p->ev_upd.push_back(b);
    p->ev_out.push_back(c);
  }
  auto first = [&](int j) { return (long long)((nc * j) / K); };
  const size_t per = o.sz_luh;
  // the copies wait for whatever the patch stream still has in flight
  EXA_CUDA(cudaEventRecord(p->ev_begin, p->stream));
  EXA_CUDA(cudaStreamWaitEvent(p->copy_stream, p->ev_begin, 0));
  EXA_CUDA(cudaStreamWaitEvent(p->d2h_stream, p->ev_begin, 0));
  for (int k = 0; k < nsteps; k++) {
    const double* src = k == 0 ? luh_in : luh_out;
    // uploads: chunk j of step k > 0 is the host copy step k-1 wrote back
    for (int j = 0; j < K; j++) {
      const long long c0 = first(j), c1 = first(j + 1);
      if (k > 0) EXA_CUDA(cudaStreamWaitEvent(p->copy_stream, p->ev_out[j], 0));
      EXA_CUDA(cudaMemcpyAsync(p->luh + c0 * per, src + c0 * per, (size_t)(c1 - c0) * per * sizeof(double),
                               cudaMemcpyHostToDevice, p->copy_stream));
      EXA_CUDA(cudaEventRecord(p->ev_in[j], p->copy_stream));
    }
    if (k == 0 && !cfl && fixed_dt != p->fixed_dt) {
      exa::fill_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_dt, fixed_dt);
      EXA_CUDA(cudaGetLastError());
      p->fixed_dt = fixed_dt;
    }
    if (k == 0 && cfl && p->fixed_dt > 0) {
      // back from fixed steps: the CFL step of the uploaded state needs all of it first
      EXA_CUDA(cudaStreamWaitEvent(p->stream, p->ev_in[K - 1], 0));
      if (int r = patch_initial_dt(p)) return r;
      p->fixed_dt = -1.0;
    }
    // predictor + volume integral chunk by chunk as the chunks arrive
    for (int j = 0; j < K; j++) {
      EXA_CUDA(cudaStreamWaitEvent(p->stream, p->ev_in[j], 0));
      exa::CellArgs a = patch_args(p);
      a.cell_begin = (int)first(j);
      a.ncells = (int)first(j + 1);
      EXA_CUDA(o.predictor(a, p->stream, p->s->cfg.precision == EXA_PREC_MIXED, p->s->pred_variant));
    }
    exa::FaceArgs f = patch_faces(p);
    EXA_CUDA(o.riemann(f, p->stream));
    if (p->nbfaces > 0) {
      exa::FaceArgs b = f;
      b.nfaces = p->nbfaces;
      EXA_CUDA(o.boundary(b, p->stream));
    }
    // surface integral + update (+ CFL of the new state) chunk by chunk; each chunk goes back to
    // the host as soon as it is final, on its own stream (the link carries both directions)
    for (int j = 0; j < K; j++) {
      const long long c0 = first(j), c1 = first(j + 1);
      exa::CellArgs u = patch_args(p);
      u.cell_begin = (int)c0;
      u.ncells = (int)c1;
      if (cfl) u.grid_dt_next = p->grid_dt_next;
      EXA_CUDA(o.update(u, true, true, p->stream, p->s->upd_variant));
      EXA_CUDA(cudaEventRecord(p->ev_upd[j], p->stream));
      EXA_CUDA(cudaStreamWaitEvent(p->d2h_stream, p->ev_upd[j], 0));
      EXA_CUDA(cudaMemcpyAsync(luh_out + c0 * per, p->luh + c0 * per, (size_t)(c1 - c0) * per * sizeof(double),
                               cudaMemcpyDeviceToHost, p->d2h_stream));
      EXA_CUDA(cudaEventRecord(p->ev_out[j], p->d2h_stream));
    }
    exa::advance_kernel<<<(ng + 127) / 128, 128, 0, p->stream>>>(ng, p->grid_t, p->grid_dt,
                                                                 cfl ? p->grid_dt_next : nullptr, p->steps);
    EXA_CUDA(cudaGetLastError());
  }
  EXA_CUDA(cudaStreamSynchronize(p->d2h_stream));
  EXA_CUDA(cudaStreamSynchronize(p->copy_stream));
  EXA_CUDA(cudaStreamSynchronize(p->stream));
  return EXA_OK;
}

int exa_patch_step_host(exa_patch* p, const double* luh_in, double* luh_out, double fixed_dt) {
  return exa_patch_run_host(p, luh_in, luh_out, 1, fixed_dt);
}

}  // extern "C"
