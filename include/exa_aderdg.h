/* exa_aderdg.h -- C ABI of the B200 ADER-DG cell update (libexa_aderdg.so).
 *
 * Drop-in for ExaHyPE's generic nonlinear ADER-DG kernels (kernels::aderdg::generic::c, declared
 * in ExaHyPE/kernels/aderdg/generic/Kernels.h:59-287) and for the generated solver glue that calls
 * them (Toolkit/exahype/toolkit/templates/solvers/AbstractGenericADERDGSolverImplementation.template
 * :104-361). Plain C types only: no torch, no C++ in the signatures.
 *
 * Data layouts are the reference's, per cell (row-major, last index fastest), n = Order+1,
 * D = NumberOfVariables + NumberOfParameters, V = NumberOfVariables:
 *   luh     [cell][z][y][x][D]        (2D: [cell][y][x][D])
 *   lduh    [cell][z][y][x][V]
 *   lQhbnd  [cell][2*DIM][a][b][D]    face 2*dir+orientation; (a,b) tangential, slower axis first
 *   lFhbnd  [cell][2*DIM][a][b][V]
 * Batched entry points take DEVICE pointers to arrays of `ncells` such blocks stored one after
 * another, and a CUDA stream (cudaStream_t passed as void*; NULL = legacy default stream).
 * They are asynchronous unless stated otherwise.
 *
 * Errors: every function returns an exa_status. Numerical trouble found on the device
 * (non-finite values, Picard cap reached, dt <= 0) is accumulated in a device status word that
 * exa_solver_status() / exa_patch_status() read and clear. The reference aborts or only logs
 * in these cases (AbstractGenericADERDGSolverImplementation.template:98-102, 2d/
 * spaceTimePredictorNonlinear.cpph:307-314); here they are reported, never trapped.
 */
#ifndef EXA_ADERDG_H
#define EXA_ADERDG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  EXA_OK = 0,
  EXA_ERR_INVALID = 1,     /* bad argument (null pointer, size, index) */
  EXA_ERR_UNSUPPORTED = 2, /* (pde, dim, order, npar, precision) not instantiated in this build */
  EXA_ERR_CUDA = 3,        /* a CUDA call failed; exa_last_error() has the message */
  EXA_ERR_NUMERICS = 4,    /* device status word non-zero (see exa_status_bits) */
  EXA_ERR_NOT_FOUND = 5
} exa_status;

/* bits of the device status word */
typedef enum {
  EXA_ST_NONFINITE_PREDICTOR = 1,
  EXA_ST_PICARD_CAP = 2,      /* some cell used all 2(N+1) Picard sweeps without converging */
  EXA_ST_NONFINITE_UPDATE = 4,
  EXA_ST_BAD_DT = 8,
  EXA_ST_TIMEOUT = 16,        /* a bounded device-side wait ran out; the launch's results are not valid */
  EXA_ST_BAD_JOB = 32         /* a mesh-level job named a block, level difference or subcell index out of range */
} exa_status_bits;

/* PDE systems compiled as device functors (the user hooks flux / eigenvalues /
 * nonConservativeProduct / boundaryValues of AbstractGenericADERDGSolverHeader.template:220-338). */
typedef enum {
  EXA_PDE_EULER = 0, /* compressible Euler, gamma 1.4, V=5 (Euler_ADERDG/EulerSolver_ADERDG.cpp:61-146) */
  EXA_PDE_SWE = 1,   /* shallow water h,hu,hv,b with NCP, V=4 (SWE_ADERDG/MySWESolver.cpp:103-152) */
  EXA_PDE_ACOUSTIC = 2, /* linear acoustics p,u,v,w with per-node rho,c (nPar=2), flux form; new */
  EXA_PDE_ELASTIC = 3   /* linear elasticity v,sigma (V=9) with per-node rho,cp,cs (nPar=3), flux form; new */
} exa_pde;

/* Application PDE systems: ids from EXA_PDE_USER_BASE up. An application compiles its functor into
 * its own shared library with include/exa_aderdg_user.cuh (EXA_REGISTER_PDE); loading that library
 * registers every (dim, order, npar) it instantiates, after which exa_solver_create accepts the id
 * like a built-in one. Replaces the toolkit-generated Abstract<App>Solver_ADERDG binding of the
 * user's solver class (AbstractGenericADERDGSolverHeader.template:34-68, 220-338). */
#define EXA_PDE_USER_BASE 64
/* called by EXA_REGISTER_PDE at load time: ops is the instantiation's launcher object (an
 * exa::Ops*, see exahype-engine_b200/csrc/exa_ops.cuh). Ids below EXA_PDE_USER_BASE, a mismatch
 * between the arguments and the object, or a second registration of the same key are refused. */
int exa_register_pde(int pde, int dim, int order, int npar, void* ops);
/* 1 if kernels for (pde, dim, order, npar) are available (built in or registered), else 0 */
int exa_pde_available(int pde, int dim, int order, int npar);

typedef enum {
  EXA_PREC_FP64 = 0,  /* every sweep in FP64 (generic-kernel semantics, parity 1e-12) */
  EXA_PREC_MIXED = 1  /* early Picard sweeps in FP32, final sweep + residual test + update in FP64 */
} exa_precision;

/* EXA_BC_HALO (last axis of a single-grid patch only): the two boundary layers face ghost
 * cells whose face traces a neighbouring subdomain supplies (slab decomposition, see
 * exa_patch_halo_pack / exa_patch_halo_unpack). */
/* EXA_BC_OUTFLOW: the ghost state is the inner state (boundaryValues copying stateIn), which
 * lets waves leave the domain (the absorbing boundary of the elastic configuration). */
/* EXA_BC_USER: the PDE functor's boundary_values hook gives the outer state and its normal flux
 * at every face node (the user's boundaryValues, 3d/boundaryConditions.cpph:29-122); only for
 * functors that define it (include/exa_aderdg_user.cuh). */
typedef enum { EXA_BC_PERIODIC = 0, EXA_BC_WALL = 1, EXA_BC_HALO = 2, EXA_BC_OUTFLOW = 3, EXA_BC_USER = 4 } exa_bc;

/* Compile-time constants of the reference's generated solver (AbstractGenericADERDGSolverHeader
 * .template:34-68), here runtime fields of a solver handle. */
typedef struct {
  int dim;            /* 2 or 3 (DIMENSIONS) */
  int order;          /* Order */
  int npar;           /* NumberOfParameters */
  exa_pde pde;
  double cfl;         /* CFL safety factor; <= 0 selects 0.9 (the toolkit default) */
  double pnpm;        /* PNPM; <= 0 selects the toolkit's table (solverController.py:17) */
  int max_picard;     /* 0: residual test with 2(N+1) cap (UseMaxPicardIterations=false);
                         > 0: exactly this many sweeps (UseMaxPicardIterations=true) */
  exa_precision precision;
} exa_solver_config;

typedef struct exa_solver exa_solver;
typedef struct exa_patch exa_patch;

/* per-cell array sizes in doubles */
typedef struct {
  int nvar, ndata, nodes_per_cell, nodes_per_face;
  size_t luh, lduh, lQhbnd, lFhbnd;
  /* predictor internals in reference layout (exa_spaceTimePredictorNonlinear) */
  size_t lQi, lFi, lQhi, lFhi;
} exa_sizes;

const char* exa_last_error(void);
const char* exa_version(void);
/* Gauss-Legendre nodes and weights on [0,1] of the given order (order+1 values each; the
 * kernels::legendre tables of GaussLegendreBasis.csnippet), for host glue that evaluates user hooks
 * at node positions. Host only. */
int exa_quadrature(int order, double* nodes, double* weights);

/* ---- solver handle -------------------------------------------------------------------- */
int exa_solver_create(const exa_solver_config* cfg, exa_solver** out);
int exa_solver_destroy(exa_solver* s);
int exa_solver_sizes(const exa_solver* s, exa_sizes* out);
/* reads and clears the device status word (synchronises the device) */
int exa_solver_status(exa_solver* s, unsigned* bits);
/* Launch form of the predictor (no reference counterpart: a tuning knob of this implementation).
 * 0: one group of cells per CTA; 1: persistent CTAs, each fetching its next group's luh by bulk
 * copy while it computes the current one; -1 (the default): the form measured as faster for this
 * instantiation on this device. The measurement runs once per (instantiation, precision, device),
 * in the first exa_patch_set_solution, on (up to 65,536 cells of) the state it was given. */
int exa_solver_set_predictor_variant(exa_solver* s, int variant);
/* the form the solver's next predictor launch uses on the current device */
int exa_solver_predictor_variant(exa_solver* s, int* variant);
/* Launch form of the HBM-bound kernels of a step, the surface integral + update + CFL kernel and
 * the Rusanov kernel: 0 one cell group per CTA / one face per warp with per-thread loads; 1 or -1
 * (the default) persistent CTAs / warps that move whole cell and face blocks by bulk copy
 * (cp.async.bulk), double-buffered, where the block sizes are multiples of 16 bytes and the arrays
 * 16-byte aligned (otherwise the first form runs). The Rusanov form is a setting of the
 * instantiation, shared by its solvers. */
int exa_solver_set_update_variant(exa_solver* s, int variant);

/* ---- batched kernels on caller-owned device memory ------------------------------------
 * `dx` is the cell size (DIM doubles, host memory) shared by all `ncells` cells; `dt` a host
 * scalar. */

/* Replaces the glue's fusedSpaceTimePredictorVolumeIntegral (AbstractGenericADERDGSolver
 * Implementation.template:104-235, nonlinear branch :168-211, addVolumeIntegralResultToUpdate=true):
 * spaceTimePredictorNonlinear (3d/spaceTimePredictorNonlinear.cpph:816-864) followed by
 * volumeIntegralNonlinear (3d/volumeIntegralNonlinear.cpph:29-223) for every cell.
 * picard_sweeps (device, nullable): Picard sweeps executed per cell (the reference returns the
 * loop index instead; exa_spaceTimePredictorNonlinear reproduces that return value). */
int exa_fused_predictor_volume_integral(exa_solver* s, int ncells, const double* luh, double* lduh,
                                        double* lQhbnd, double* lFhbnd, int* picard_sweeps, const double* dx,
                                        double t, double dt, void* stream);
/* The same with the cells' centres (device, [cell][3]), which an application functor's
 * algebraic_source needs (the reference's algebraicSource at x = centre + dx (node - 0.5) and
 * t + node_i dt, 3d/spaceTimePredictorNonlinear.cpph:323-367); PDEs with an algebraic source refuse
 * the call without them. */
int exa_fused_predictor_volume_integral_x(exa_solver* s, int ncells, const double* luh, double* lduh,
                                          double* lQhbnd, double* lFhbnd, int* picard_sweeps, const double* dx,
                                          const double* centres, double t, double dt, void* stream);

/* Replaces riemannSolverNonlinear<useNCP,false> (3d/riemannSolverNonlinear.cpph:37-128) for a
 * list of interior faces: face f joins cell left[f] (its face 2*dir[f]+1) and cell right[f]
 * (its face 2*dir[f]); FL/FR are the two cells' lFhbnd blocks, updated in place as in the
 * reference (ADERDGSolver.cpp:1781-1785). left/right/dir are device arrays. */
int exa_riemann_solver_nonlinear(exa_solver* s, int nfaces, const int* left, const int* right,
                                 const signed char* dir, const double* lQhbnd, double* lFhbnd, void* stream);
/* The same with the cells' size dx (DIM doubles, host), which riemannSolverNonlinear<useNCP,true>
 * needs for the viscous term of the Rusanov speed (:73-87); PDEs with a viscous flux refuse the
 * call without dx. */
int exa_riemann_solver_nonlinear_dx(exa_solver* s, int nfaces, const int* left, const int* right,
                                    const signed char* dir, const double* lQhbnd, double* lFhbnd, const double* dx,
                                    void* stream);

/* Replaces boundaryConditions (3d/boundaryConditions.cpph:29-122) + the Riemann call of the
 * glue's boundaryConditions (...Implementation.template:307-350) with a reflective wall
 * (the SWE app's boundaryValues, MySWESolver.cpp:43-62) on faces face[f] of cells cell[f]. */
int exa_boundary_conditions_wall(exa_solver* s, int nfaces, const int* cell, const signed char* face,
                                 const double* lQhbnd, double* lFhbnd, void* stream);
int exa_boundary_conditions_wall_dx(exa_solver* s, int nfaces, const int* cell, const signed char* face,
                                    const double* lQhbnd, double* lFhbnd, const double* dx, void* stream);

/* Replaces surfaceIntegralNonlinear (3d/surfaceIntegralNonlinear.cpph:21-90) followed by
 * solutionUpdate (3d/solutionUpdate.cpph:28-67): luh += dt/w * (lduh - surface terms). lduh is
 * left unchanged. */
int exa_surface_integral_and_update(exa_solver* s, int ncells, double* luh, const double* lduh,
                                    const double* lFhbnd, const double* dx, double dt, void* stream);

/* Replaces solutionUpdate alone (3d/solutionUpdate.cpph:28-67): luh = luhOld + dt/w * lduh
 * (luh may alias luhOld). */
int exa_solution_update(exa_solver* s, int ncells, double* luh, const double* luhOld, const double* lduh,
                        double dt, void* stream);

/* Replaces stableTimeStepSize (3d/stableTimeStepSize.cpph:14-62) and the min-reduction over
 * cells (ADERDGSolver::updateAdmissibleTimeStepSize, ADERDGSolver.cpp:458-462). cell_dt
 * (device, nullable) receives every cell's value; *dt_min (host, nullable) the minimum --
 * requesting it synchronises the stream. Cells whose state is non-finite or gives dt <= 0 set
 * bits in the solver's status word (exa_solver_status) and count as +inf; unlike
 * exa_stable_time_step_size_noalloc, the call itself still returns EXA_OK, because the status
 * word also collects the bits of the solver's other kernels. */
int exa_stable_time_step_size(exa_solver* s, int ncells, const double* luh, const double* dx, double* cell_dt,
                              double* dt_min, void* stream);

/* Allocation-free variant of exa_stable_time_step_size. It has no counterpart in the reference.
 *
 * Who needs it: callers that cannot call cudaMalloc. One case is a host program whose device
 * memory is owned by another runtime, such as a framework allocator that has reserved the whole
 * pool. Another is a step loop that must not pay the device-wide synchronisation an allocation
 * can imply. exa_solver_create allocates (its status word), so this entry point takes the solver
 * configuration directly and needs no handle. It calls no cudaMalloc, cudaFree or other
 * allocating routine.
 *
 * Inputs and outputs belong to the caller, as in exa_stable_time_step_size: luh and cell_dt are
 * device arrays of ncells cells (cell_dt nullable); *dt_min is a host double (nullable;
 * requesting it synchronises the stream).
 * Its scratch -- every cell's time step, the minimum and a status word -- is one file-scope
 * device array of the library sized for EXA_NOALLOC_MAX_CELLS cells (8 MiB). Every GPU that loads
 * the library holds the array until the process exits.
 *   - ncells > EXA_NOALLOC_MAX_CELLS is rejected with EXA_ERR_INVALID before any device work.
 *   - The first call on a device looks up the array's device address (cudaGetSymbolAddress) and
 *     caches it for that device; make that first call before any stream capture.
 *   - With lazy module loading (the CUDA default), the call that first loads the library's
 *     module on a device is what places the array in device memory. A caller whose device memory
 *     another runtime reserves should make its first call per device (or set
 *     CUDA_MODULE_LOADING=EAGER) before that runtime reserves the pool.
 *   - The cached address is only valid for the context it was looked up in: after
 *     cudaDeviceReset the module is loaded again and the array may move, so do not call this
 *     entry point after a device reset in the same process.
 *   - All calls share the one array and each call resets what it reads, but calls that overlap
 *     on the GPU (other streams, other host threads) race on it: serialise them.
 * Returns EXA_ERR_NUMERICS when a cell's state is non-finite or gives dt <= 0 and dt_min was
 * requested (the call then reads the status word after synchronising). With dt_min == NULL the
 * call does not synchronise and reports no numerical status; such cells get +inf in cell_dt. */
#define EXA_NOALLOC_MAX_CELLS 1048576
int exa_stable_time_step_size_noalloc(const exa_solver_config* cfg, int ncells, const double* luh, const double* dx,
                                      double* cell_dt, double* dt_min, void* stream);

/* ---- per-cell compatibility shims: the exact generic-kernel signatures on HOST pointers ----
 * One cell per call, synchronous; for conformance tests and glue that has not been batched yet. */

/* spaceTimePredictorNonlinear<useSource=false,useFlux=true,useViscousFlux=false,useNCP,
 * noTimeAveraging=false> (3d/spaceTimePredictorNonlinear.cpph:816-823): fills lQhbnd, lFhbnd and
 * the internals lQi [z][y][x][t][D], lFi [t][z][y][x][DIM+1][V] (last sweep), lQhi, lFhi (reference
 * blocks); any internal may be NULL. Returns the reference's value: 3D the index of the converging
 * iteration, 2D MaxIterations+2 on convergence (2d/...:303-305); -1 on error. */
int exa_spaceTimePredictorNonlinear(exa_solver* s, double* lQhbnd, double* lFhbnd, double* lQi, double* lFi,
                                    double* lQhi, double* lFhi, const double* luh, const double* cellCenter,
                                    const double* invDx, double t, double dt);
/* volumeIntegralNonlinear, time-averaged branch (3d/volumeIntegralNonlinear.cpph:133-223). */
int exa_volumeIntegralNonlinear(exa_solver* s, double* lduh, const double* lFhi, const double* dx);
/* riemannSolverNonlinear (3d/riemannSolverNonlinear.cpph:37-128), in place on FL/FR. */
int exa_riemannSolverNonlinear(exa_solver* s, double* FL, double* FR, const double* QL, const double* QR,
                               double t, double dt, const double* dx, int direction);
/* surfaceIntegralNonlinear (3d/surfaceIntegralNonlinear.cpph:21-90). */
int exa_surfaceIntegralNonlinear(exa_solver* s, double* lduh, const double* lFhbnd, const double* dx);
/* faceIntegralNonlinear (3d/faceIntegralNonlinear.cpph:21-103): one face block lFhbnd ([a][b][V])
 * of face 2*direction+orientation, the per-face form the engine's glue calls (...Implementation
 * .template:247-285). */
int exa_faceIntegralNonlinear(exa_solver* s, double* lduh, const double* lFhbnd, int direction, int orientation,
                              const double* dx);
/* solutionUpdate (3d/solutionUpdate.cpph:28-67). */
int exa_solutionUpdate(exa_solver* s, double* luh, const double* luhOld, const double* lduh, double dt);
/* stableTimeStepSize (3d/stableTimeStepSize.cpph:14-62); returns the value in *dt. */
int exa_stableTimeStepSize(exa_solver* s, const double* luh, const double* dx, double* dt);

/* ---- mesh levels (AMR) ---------------------------------------------------------------------
 * A fine cell of the 3:1 refined mesh lies levelDelta = fineGridLevel - coarseGridLevel levels
 * below a coarse cell; its subcell index along each axis runs over 0 .. 3^levelDelta - 1.
 *
 * Batched forms, on device arrays and `stream`. jobs: device int[njobs][6] = {fine block, coarse
 * block, levelDelta (1..12), subcell index along x, y (, z)}; the unused last entries of a face job
 * are ignored. Volume blocks are cells of luh
 * (n^DIM nodes x (nVar + nPar)); face blocks are faces of lQhbnd / lFhbnd (block = cell * 2 DIM +
 * face: n^(DIM-1) nodes x (nVar + nPar) or nVar). nfine / ncoarse: blocks in the fine / coarse arrays.
 *   EXA_AMR_PROLONGATE: the fine block is the coarse data prolongated (3d/amrRoutines.cpph:48-143
 *     faceUnknownsProlongation, :369-444 volumeUnknownsProlongation); group_ptr is ignored.
 *   EXA_AMR_RESTRICT: the restriction of each fine block is added to its coarse block
 *     (faceUnknownsRestriction :248-334, volumeUnknownsRestriction :484-554). One CTA per group of
 *     jobs: group g = jobs [group_ptr[g], group_ptr[g+1]) (device int[ngroups + 1]), all naming one
 *     coarse block, added in job order; with group_ptr NULL every job is its own group (ngroups is
 *     then ignored), and no two jobs may then name the same coarse block.
 *   EXA_AMR_RESTRICT_FLUX (faces): the coarse lFhbnd block is replaced by the fine block's
 *     restriction (faceUnknownsRestriction :186-246); every job is its own group.
 * A job out of range is skipped and sets EXA_ST_BAD_JOB in the solver's status word. */
#define EXA_AMR_PROLONGATE 0
#define EXA_AMR_RESTRICT 1
#define EXA_AMR_RESTRICT_FLUX 2
int exa_amr_volume_unknowns(exa_solver* s, int mode, double* luhFine, double* luhCoarse, long long nfine,
                            long long ncoarse, int njobs, const int* jobs, int ngroups, const int* group_ptr,
                            void* stream);
int exa_amr_face_unknowns(exa_solver* s, int mode, double* lQhbndFine, double* lFhbndFine, double* lQhbndCoarse,
                          double* lFhbndCoarse, long long nfine, long long ncoarse, int njobs, const int* jobs,
                          int ngroups, const int* group_ptr, void* stream);

/* Per-call shims with the reference's signatures on host arrays of one cell (luh) or one face
 * (lQhbnd / lFhbnd of one face); subcellIndex: DIM ints, subfaceIndex: DIM - 1 ints. The
 * restrictions add to the coarse arrays (the reference's accumulate), except
 * exa_faceFluxRestriction, which overwrites lFhbndCoarse. */
int exa_volumeUnknownsProlongation(exa_solver* s, double* luhFine, const double* luhCoarse, int coarseGridLevel,
                                   int fineGridLevel, const int* subcellIndex);
int exa_volumeUnknownsRestriction(exa_solver* s, double* luhCoarse, const double* luhFine, int coarseGridLevel,
                                  int fineGridLevel, const int* subcellIndex);
int exa_faceUnknownsProlongation(exa_solver* s, double* lQhbndFine, double* lFhbndFine, const double* lQhbndCoarse,
                                 const double* lFhbndCoarse, int coarseGridLevel, int fineGridLevel,
                                 const int* subfaceIndex);
int exa_faceUnknownsRestriction(exa_solver* s, double* lQhbndCoarse, double* lFhbndCoarse, const double* lQhbndFine,
                                const double* lFhbndFine, int coarseGridLevel, int fineGridLevel,
                                const int* subfaceIndex);
int exa_faceFluxRestriction(exa_solver* s, double* lFhbndCoarse, const double* lFhbndFine, const int* subfaceIndex,
                            int levelDelta);

/* ---- a-posteriori subcell limiter (limiter/generic/c/Limiter.cpph) ------------------------------
 * The finite-volume patch of a cell has P = 2N+1 subcells per axis (the generated limiting
 * solver's default PatchSize) plus `ghost` layers (0..4; the FV scheme's GhostLayerWidth: 1
 * Godunov, 2 MUSCL-Hancock): lim is [(P + 2 ghost)^DIM][nVar + nPar] per cell. Only interior
 * subcells are read or written. DMP observables are the first nobs (0..min(32, nVar + nPar))
 * variables and the relaxation parameter is `relax` itself (the generated solver's defaults of
 * mapDiscreteMaximumPrincipleObservables / getDiscreteMaximumPrincipleRelaxationParameter).
 * Batched over ncells cells of device arrays on `stream`:
 *   project_on_fv   projectOnFVLimiterSpace (:43-78): the subcell means of the DG polynomial;
 *   project_on_dg   projectOnDGSpace (:80-116): the constrained least-squares DG reconstruction;
 *   local_min_max   findCellLocalMinAndMax (:121-164): per observable, over the nodes, the
 *                   Gauss-Lobatto nodes and the subcell means; mn / mx [cell][nobs];
 *   fv_min_max      findCellLocalLimiterMinAndMax (:166-199), over the interior subcells;
 *   dmp             discreteMaximumPrincipleAndMinAndMaxSearch (:201-255): bmin / bmax
 *                   [cell][2 DIM][nobs] hold the neighbours' min / max on entry; on return face
 *                   block 0 holds the cell's own min / max and block 1 the neighbours'; ok[cell] = 1
 *                   where the principle holds (relaxed by max((max - min) * scale, relax)) and
 *                   every extremum is finite. */
int exa_limiter_project_on_fv(exa_solver* s, int ncells, const double* luh, double* lim, int ghost, void* stream);
int exa_limiter_project_on_dg(exa_solver* s, int ncells, const double* lim, double* luh, int ghost, void* stream);
int exa_limiter_local_min_max(exa_solver* s, int ncells, const double* luh, int nobs, double* mn, double* mx,
                              void* stream);
int exa_limiter_fv_min_max(exa_solver* s, int ncells, const double* lim, int ghost, int nobs, double* mn, double* mx,
                           void* stream);
int exa_limiter_dmp(exa_solver* s, int ncells, const double* luh, int nobs, double relax, double scale, double* bmin,
                    double* bmax, unsigned char* ok, void* stream);
/* the same for one cell on host arrays, as the generated limiting solver calls them
 * (GenericLimiterSolverImplementation.template:40-62); exa_discreteMaximumPrincipleAndMinAndMaxSearch
 * sets *ok to the decision */
int exa_projectOnFVLimiterSpace(exa_solver* s, const double* luh, double* lim, int ghost);
int exa_projectOnDGSpace(exa_solver* s, const double* lim, double* luh, int ghost);
int exa_findCellLocalMinAndMax(exa_solver* s, const double* luh, int nobs, double* mn, double* mx);
int exa_findCellLocalLimiterMinAndMax(exa_solver* s, const double* lim, int ghost, int nobs, double* mn, double* mx);
int exa_discreteMaximumPrincipleAndMinAndMaxSearch(exa_solver* s, const double* luh, int nobs, double relax,
                                                   double scale, double* bmin, double* bmax, int* ok);
/* The projectors of order `order` (1..9), host arrays: fine [3][n][n] (phi_k((j + x_m)/3)), dg2fv
 * [n][P], fv2dg [P][n], leg2lob [n][n] (Gauss-Lobatto nodes descending, as the reference's
 * tables); any pointer may be NULL. */
int exa_amr_limiter_projectors(int order, double* fine, double* dg2fv, double* fv2dg, double* leg2lob);

/* ---- device-resident patches: the per-step chain as one CUDA graph ------------------------
 * A patch holds one or more uniform grids (all cells of all grids in one batch, cell-major, grid
 * after grid; inside a grid c = (iz*ny + iy)*nx + ix). Each grid keeps its own t and CFL dt
 * (global non-fused order of ADERDGSolver: dt = min CFL(luh) -> predictor + volume -> Riemann ->
 * surface + update; ADERDGSolver.cpp:369-416, 887-947, 1190-1258). */
typedef struct {
  int ncell[3];       /* cells per axis (ncell[2] ignored in 2D) */
  double offset[3];   /* lower corner */
  double size[3];     /* edge lengths */
  int bc[3];          /* per axis: EXA_BC_PERIODIC or EXA_BC_WALL (both sides) */
} exa_grid_desc;

typedef struct {
  long long steps;          /* steps taken since creation */
  double picard_mean;       /* mean Picard sweeps per cell of the last step */
  int picard_hist[32];      /* sweeps histogram of the last step (index = sweeps, capped at 31) */
} exa_patch_stats;

int exa_patch_create(exa_solver* s, int ngrids, const exa_grid_desc* grids, exa_patch** out);
int exa_patch_destroy(exa_patch* p);
long long exa_patch_num_cells(const exa_patch* p);
/* copy the reference-layout solution of all cells in (from host memory, or device memory
 * when on_device != 0) and compute every grid's first CFL dt. */
int exa_patch_set_solution(exa_patch* p, const double* luh, int on_device);
int exa_patch_get_solution(exa_patch* p, double* luh, int on_device);
/* device pointer of the patch's luh (ncells * luh doubles), valid until destroy */
double* exa_patch_luh(exa_patch* p);
/* advance every grid by nsteps steps; fixed_dt > 0 replaces the CFL dt. Asynchronous on the
 * patch's stream (exa_patch_sync waits). One CUDA graph launch per step. */
int exa_patch_step(exa_patch* p, int nsteps, double fixed_dt);
int exa_patch_sync(exa_patch* p);
int exa_patch_time(exa_patch* p, double* t, double* dt);   /* host arrays of ngrids (synchronises) */
int exa_patch_track_picard(exa_patch* p, int on);       /* kept for compatibility: sweeps are always recorded */
int exa_patch_stats_get(exa_patch* p, exa_patch_stats* st);
int exa_patch_status(exa_patch* p, unsigned* bits);       /* reads and clears (synchronises) */
void* exa_patch_stream(exa_patch* p);                     /* the cudaStream_t the patch runs on */

/* Point source of the patch: the user's algebraicSource hook evaluated at every node x and
 * time t + node_i*dt (3d/spaceTimePredictorNonlinear.cpph:323-337) as
 *   S_var(x, t) = amplitude * r(t - t0) * exp(-|x - xs|^2 / (2 width^2)) / ((2 pi)^(d/2) width^d),
 *   r(s) = (1 - 2 pi^2 f0^2 s^2) exp(-pi^2 f0^2 s^2)  (Ricker wavelet),
 * on variable `variable`. Only PDEs built with a source (acoustic, elastic) use it; cells farther
 * than 6 widths plus a cell diagonal from xs are skipped. NULL removes the source. */
typedef struct {
  double x[3];
  double f0, t0, amplitude, width;
  int variable;
} exa_point_source;
int exa_patch_set_point_source(exa_patch* p, const exa_point_source* src);

/* adjustPointSolution (3d/solutionAdjustment.cpph:17-58) on the device: the functor's
 * adjust_point_solution hook at every node x of every cell (x = cell centre + dx (node - 0.5)),
 * with each grid's current time and step, in place; then every grid's CFL step is recomputed.
 * EXA_ERR_UNSUPPORTED for functors without the hook. Synchronises the patch stream. */
int exa_patch_adjust_solution(exa_patch* p);

/* ---- one step in phases, for subdomains that exchange face traces ---------------------------
 * The reference exchanges the face data of cells next to a remote rank by MPI
 * (ADERDGSolver::sendDataToNeighbour / mergeWithNeighbourData, ADERDGSolver.cpp:1946-2010) and
 * reduces the admissible time step over ranks. Here a rank's patch carries EXA_BC_HALO on its last
 * axis; one step is
 *   PREDICTOR -> halo_pack -> (exchange with the two neighbours) -> halo_unpack -> FACES ->
 *   UPDATE -> (all-reduce min of dt_next, exa_patch_dt_next_copy) -> ADVANCE.
 * FACES splits into FACES_INTERIOR (faces between real cells and domain faces, which do not need
 * the neighbours' traces and can run while the exchange is in flight) and FACES_HALO (the faces
 * of the ghost cells, after halo_unpack):
 *   PREDICTOR -> halo_pack -> (start the exchange) -> FACES_INTERIOR -> (finish the exchange) ->
 *   halo_unpack -> FACES_HALO -> UPDATE -> ...
 * exa_patch_step refuses halo patches. All calls enqueue on the patch stream. */
enum {
  EXA_PHASE_PREDICTOR = 0,
  EXA_PHASE_FACES = 1,
  EXA_PHASE_UPDATE = 2,
  EXA_PHASE_ADVANCE = 3,
  EXA_PHASE_FACES_INTERIOR = 4,
  EXA_PHASE_FACES_HALO = 5
};
int exa_patch_step_phase(exa_patch* p, int phase, double fixed_dt);
/* doubles in one side's exchange buffer: [lQhbnd face blocks of the layer][lFhbnd face blocks] */
long long exa_patch_halo_doubles(const exa_patch* p);
/* send_lo: the low boundary layer's low faces; send_hi: the high layer's high faces (device) */
int exa_patch_halo_pack(exa_patch* p, double* send_lo, double* send_hi);
/* recv_lo: what the lower neighbour packed as send_hi; recv_hi: the upper neighbour's send_lo */
int exa_patch_halo_unpack(exa_patch* p, const double* recv_lo, const double* recv_hi);
/* copy the per-grid CFL minimum of the last UPDATE phase to (to_patch=0) or from (1) a device buffer */
int exa_patch_dt_next_copy(exa_patch* p, double* dev_buf, int to_patch);
/* the same for the time step in use (after exa_patch_set_solution: the local CFL minimum) */
int exa_patch_dt_copy(exa_patch* p, double* dev_buf, int to_patch);

/* Host-only (no device work): the face lists a patch of these grids uses. With out->left == NULL
 * only the counts are filled; otherwise the caller's arrays (nfaces / nbfaces entries, sizes given
 * in out->nfaces / out->nbfaces) receive the lists. Ghost cells of a halo axis are numbered after
 * the real cells: the low ghost layer, then the high one. */
typedef struct {
  long long ncells, nghost;
  int nfaces, nbfaces;
  int* left;
  int* right;
  signed char* dir;
  int* bcell;
  signed char* bface;
} exa_face_lists;
int exa_build_face_lists(int dim, int ngrids, const exa_grid_desc* grids, exa_face_lists* out);

/* ---- one step from and to host memory -----------------------------------------------------
 * Uploads luh_in (host, reference layout, all cells), runs one step, downloads the new state into
 * luh_out (may equal luh_in). The copies run on a second stream in cell chunks, overlapped with
 * the predictor (chunk j starts as soon as it has arrived) and with the update (chunk j is
 * downloaded as soon as it is final); pinned host buffers make the overlap real. The time step is
 * fixed_dt if > 0, else the patch's CFL step, which is the CFL step of luh_in when luh_in is the
 * state the patch last produced or was given (exa_patch_set_solution, a previous step). Returns
 * after luh_out is written. Patches with EXA_BC_HALO are refused. */
int exa_patch_step_host(exa_patch* p, const double* luh_in, double* luh_out, double fixed_dt);
/* nsteps such steps of a host-resident state: step 0 reads luh_in, every step writes its result to
 * luh_out, steps >= 1 read luh_out. The upload of a chunk for step k waits only for that chunk's
 * download of step k-1, so downloads and uploads run at the same time on the two copy directions
 * and both overlap the kernels. */
int exa_patch_run_host(exa_patch* p, const double* luh_in, double* luh_out, int nsteps, double fixed_dt);

/* ---- discrete adjoint (acoustic and elastic systems) -----------------------------------------
 * No reference counterpart: the reference has no adjoint. The forward step differentiated is
 * exa_patch_step(p, 1, dt) with a fixed dt and a solver created with max_picard > 0 (the
 * reference's UseMaxPicardIterations mode: a fixed Picard sweep count, no residual test), FP64,
 * on grids whose domain faces are periodic, reflective walls, outflow or halo slabs (EXA_BC_USER
 * faces are refused with EXA_ERR_UNSUPPORTED).
 *
 * exa_patch_adjoint_step: the patch's current solution is u_k at time t_k (exa_patch_set_time).
 * lambda (device, luh layout: D doubles per node) holds dJ/du_{k+1} on entry and
 * (d u_{k+1} / d u_k)^T lambda on exit. The material-parameter entries V..D-1 accumulate: their
 * entry value plus the step's parameter adjoint, so after the adjoint of step 0 they hold
 * dJ/d(parameters) per node. The patch's solution is left unchanged; the call enqueues on the
 * patch stream. */
int exa_patch_set_time(exa_patch* p, double t);
int exa_patch_adjoint_step(exa_patch* p, double* lambda, double dt);

/* The same adjoint step in two phases around two halo exchanges, for a rank's slab (EXA_BC_HALO;
 * on other patches the two phases equal exa_patch_adjoint_step). The transposed Rusanov flux of a
 * face between slabs needs the neighbour cell's lambda and trace as well as this rank's:
 *   EXA_ADJ_FORWARD   the forward predictor at u_k; takes lambda (this rank's cells) in;
 *   then exchange the face traces (exa_patch_halo_pack / _unpack, as in a forward step) and the
 *   boundary layers' lambda (exa_patch_adjoint_halo_pack / _unpack, the same ring: recv_lo is the
 *   lower neighbour's send_hi, recv_hi the upper neighbour's send_lo);
 *   EXA_ADJ_REVERSE   the transposed faces and predictors; writes the result into lambda.
 * Each rank writes only its own cells' adjoints, so the ranks' results together equal the
 * adjoint step of the whole grid. exa_patch_adjoint_halo_doubles: doubles per buffer (cells per
 * layer x nodes x D). The buffers are device memory. */
#define EXA_ADJ_FORWARD 0
#define EXA_ADJ_REVERSE 1
int exa_patch_adjoint_phase(exa_patch* p, int phase, double* lambda, double dt);
long long exa_patch_adjoint_halo_doubles(const exa_patch* p);
int exa_patch_adjoint_halo_pack(exa_patch* p, double* send_lo, double* send_hi);
int exa_patch_adjoint_halo_unpack(exa_patch* p, const double* recv_lo, const double* recv_hi);

/* ---- binomial checkpointing (host only) -------------------------------------------------------
 * A schedule that reverses `steps` time steps while holding at most `snaps` stored states (the
 * initial state included), with the fewest forward recomputations (Griewank's binomial
 * checkpointing, computed by dynamic programming over the split points). Actions, in order:
 *   EXA_CK_STORE   a=slot, b=step   store the current state (which is u_step) in slot a
 *   EXA_CK_RESTORE a=slot, b=step   make slot a's state (u_step) current
 *   EXA_CK_ADVANCE a=from, b=to     advance the current state from u_from to u_to
 *   EXA_CK_ADJOINT a=step           adjoint of step a (current state u_a)
 * The first action stores u_0 in slot 0. With out == NULL only *count and *forward_steps are
 * set; otherwise at most `capacity` actions are written (EXA_ERR_INVALID if too few). */
enum { EXA_CK_STORE = 0, EXA_CK_RESTORE = 1, EXA_CK_ADVANCE = 2, EXA_CK_ADJOINT = 3 };
typedef struct {
  int action, a, b;
} exa_ck_action;
int exa_checkpoint_schedule(int steps, int snaps, exa_ck_action* out, int capacity, int* count,
                            long long* forward_steps);

#ifdef __cplusplus
}
#endif
#endif /* EXA_ADERDG_H */
