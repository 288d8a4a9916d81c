"""Python binding of libexa_aderdg.so (include/exa_aderdg.h) over ctypes.

This mirrors the reference's generic-kernel interface for the tests and the benchmark:
``Solver`` plays the generated ``Abstract<App>Solver_ADERDG`` glue (fusedSpaceTimePredictor-
VolumeIntegral, riemannSolver, boundaryConditions, faceIntegral + addUpdateToSolution,
stableTimeStepSize; AbstractGenericADERDGSolverImplementation.template:104-361) on batches of
device-resident cells, and exposes the per-cell shims with the exact generic-kernel semantics.
``Patch`` is a device-resident set of uniform grids stepped by one CUDA graph per step.

Device arrays are torch CUDA tensors (float64, contiguous); torch is used only for device
memory and streams. There is no CPU fallback: constructing a Solver without the built library
or without a CUDA device raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libexa_aderdg.so")

EXA_OK = 0
PDE_EULER, PDE_SWE, PDE_ACOUSTIC, PDE_ELASTIC = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1
BC_PERIODIC, BC_WALL = 0, 1
ST_NONFINITE_PREDICTOR, ST_PICARD_CAP, ST_NONFINITE_UPDATE, ST_BAD_DT, ST_TIMEOUT, ST_BAD_JOB = 1, 2, 4, 8, 16, 32
# mesh-level operations (exa_amr_volume_unknowns / exa_amr_face_unknowns)
AMR_PROLONGATE, AMR_RESTRICT, AMR_RESTRICT_FLUX = 0, 1, 2
NVAR = {PDE_EULER: 5, PDE_SWE: 4, PDE_ACOUSTIC: 4, PDE_ELASTIC: 9}
NPAR = {PDE_EULER: 0, PDE_SWE: 0, PDE_ACOUSTIC: 2, PDE_ELASTIC: 3}


class ExaError(RuntimeError):
    pass


class _Config(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("order", ctypes.c_int), ("npar", ctypes.c_int), ("pde", ctypes.c_int),
                ("cfl", ctypes.c_double), ("pnpm", ctypes.c_double), ("max_picard", ctypes.c_int),
                ("precision", ctypes.c_int)]


class _Sizes(ctypes.Structure):
    _fields_ = [("nvar", ctypes.c_int), ("ndata", ctypes.c_int), ("nodes_per_cell", ctypes.c_int),
                ("nodes_per_face", ctypes.c_int), ("luh", ctypes.c_size_t), ("lduh", ctypes.c_size_t),
                ("lQhbnd", ctypes.c_size_t), ("lFhbnd", ctypes.c_size_t), ("lQi", ctypes.c_size_t),
                ("lFi", ctypes.c_size_t), ("lQhi", ctypes.c_size_t), ("lFhi", ctypes.c_size_t)]


class GridDesc(ctypes.Structure):
    _fields_ = [("ncell", ctypes.c_int * 3), ("offset", ctypes.c_double * 3), ("size", ctypes.c_double * 3),
                ("bc", ctypes.c_int * 3)]


class FaceLists(ctypes.Structure):
    _fields_ = [("ncells", ctypes.c_longlong), ("nghost", ctypes.c_longlong), ("nfaces", ctypes.c_int),
                ("nbfaces", ctypes.c_int), ("left", ctypes.c_void_p), ("right", ctypes.c_void_p),
                ("dir", ctypes.c_void_p), ("bcell", ctypes.c_void_p), ("bface", ctypes.c_void_p)]


PHASE_PREDICTOR, PHASE_FACES, PHASE_UPDATE, PHASE_ADVANCE = 0, 1, 2, 3
PHASE_FACES_INTERIOR, PHASE_FACES_HALO = 4, 5
ADJ_FORWARD, ADJ_REVERSE = 0, 1
BC_HALO, BC_OUTFLOW, BC_USER = 2, 3, 4
PDE_USER_BASE = 64


class PointSource(ctypes.Structure):
    _fields_ = [("x", ctypes.c_double * 3), ("f0", ctypes.c_double), ("t0", ctypes.c_double),
                ("amplitude", ctypes.c_double), ("width", ctypes.c_double), ("variable", ctypes.c_int)]


class CkAction(ctypes.Structure):
    _fields_ = [("action", ctypes.c_int), ("a", ctypes.c_int), ("b", ctypes.c_int)]


CK_STORE, CK_RESTORE, CK_ADVANCE, CK_ADJOINT = 0, 1, 2, 3


class _PatchStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_longlong), ("picard_mean", ctypes.c_double), ("picard_hist", ctypes.c_int * 32)]


_lib = None


def load_library(path=None):
    """Load libexa_aderdg.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ExaError("%s is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`" % path)
    lib = ctypes.CDLL(path)
    lib.exa_last_error.restype = ctypes.c_char_p
    lib.exa_version.restype = ctypes.c_char_p
    vp, i, d, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_double)
    ll = ctypes.c_longlong
    sigs = {
        "exa_solver_create": [ctypes.POINTER(_Config), ctypes.POINTER(vp)],
        "exa_solver_destroy": [vp],
        "exa_solver_sizes": [vp, ctypes.POINTER(_Sizes)],
        "exa_solver_set_predictor_variant": [vp, i],
        "exa_solver_predictor_variant": [vp, ctypes.POINTER(i)],
        "exa_solver_set_update_variant": [vp, i],
        "exa_solver_status": [vp, ctypes.POINTER(ctypes.c_uint)],
        "exa_fused_predictor_volume_integral": [vp, i, vp, vp, vp, vp, vp, dp, d, d, vp],
        "exa_fused_predictor_volume_integral_x": [vp, i, vp, vp, vp, vp, vp, dp, vp, d, d, vp],
        "exa_riemann_solver_nonlinear": [vp, i, vp, vp, vp, vp, vp, vp],
        "exa_boundary_conditions_wall": [vp, i, vp, vp, vp, vp, vp],
        "exa_riemann_solver_nonlinear_dx": [vp, i, vp, vp, vp, vp, vp, vp, vp],
        "exa_boundary_conditions_wall_dx": [vp, i, vp, vp, vp, vp, vp, vp],
        "exa_surface_integral_and_update": [vp, i, vp, vp, vp, dp, d, vp],
        "exa_solution_update": [vp, i, vp, vp, vp, d, vp],
        "exa_stable_time_step_size": [vp, i, vp, dp, vp, dp, vp],
        "exa_spaceTimePredictorNonlinear": [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, d, d],
        "exa_riemannSolverNonlinear": [vp, vp, vp, vp, vp, d, d, dp, i],
        "exa_solutionUpdate": [vp, vp, vp, vp, d],
        "exa_volumeIntegralNonlinear": [vp, vp, vp, dp],
        "exa_surfaceIntegralNonlinear": [vp, vp, vp, dp],
        "exa_faceIntegralNonlinear": [vp, vp, vp, i, i, dp],
        "exa_stableTimeStepSize": [vp, vp, dp, dp],
        "exa_patch_create": [vp, i, ctypes.POINTER(GridDesc), ctypes.POINTER(vp)],
        "exa_patch_destroy": [vp],
        "exa_patch_set_solution": [vp, vp, i],
        "exa_patch_get_solution": [vp, vp, i],
        "exa_patch_step": [vp, i, d],
        "exa_patch_sync": [vp],
        "exa_patch_time": [vp, dp, dp],
        "exa_patch_stats_get": [vp, ctypes.POINTER(_PatchStats)],
        "exa_patch_status": [vp, ctypes.POINTER(ctypes.c_uint)],
        "exa_patch_step_phase": [vp, i, d],
        "exa_patch_halo_pack": [vp, vp, vp],
        "exa_patch_halo_unpack": [vp, vp, vp],
        "exa_patch_dt_next_copy": [vp, vp, i],
        "exa_patch_dt_copy": [vp, vp, i],
        "exa_build_face_lists": [i, i, ctypes.POINTER(GridDesc), ctypes.POINTER(FaceLists)],
        "exa_patch_set_point_source": [vp, ctypes.POINTER(PointSource)],
        "exa_patch_set_time": [vp, d],
        "exa_patch_step_host": [vp, vp, vp, d],
        "exa_patch_run_host": [vp, vp, vp, i, d],
        "exa_patch_adjoint_step": [vp, vp, d],
        "exa_patch_adjoint_phase": [vp, i, vp, d],
        "exa_patch_adjoint_halo_pack": [vp, vp, vp],
        "exa_patch_adjoint_halo_unpack": [vp, vp, vp],
        "exa_patch_adjust_solution": [vp],
        "exa_register_pde": [i, i, i, i, vp],
        "exa_pde_available": [i, i, i, i],
        "exa_checkpoint_schedule": [i, i, ctypes.POINTER(CkAction), i, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_longlong)],
        "exa_amr_volume_unknowns": [vp, i, vp, vp, ll, ll, i, vp, i, vp, vp],
        "exa_amr_face_unknowns": [vp, i, vp, vp, vp, vp, ll, ll, i, vp, i, vp, vp],
        "exa_volumeUnknownsProlongation": [vp, vp, vp, i, i, vp],
        "exa_volumeUnknownsRestriction": [vp, vp, vp, i, i, vp],
        "exa_faceUnknownsProlongation": [vp, vp, vp, vp, vp, i, i, vp],
        "exa_faceUnknownsRestriction": [vp, vp, vp, vp, vp, i, i, vp],
        "exa_faceFluxRestriction": [vp, vp, vp, vp, i],
        "exa_limiter_project_on_fv": [vp, i, vp, vp, i, vp],
        "exa_limiter_project_on_dg": [vp, i, vp, vp, i, vp],
        "exa_limiter_local_min_max": [vp, i, vp, i, vp, vp, vp],
        "exa_limiter_fv_min_max": [vp, i, vp, i, i, vp, vp, vp],
        "exa_limiter_dmp": [vp, i, vp, i, d, d, vp, vp, vp, vp],
        "exa_projectOnFVLimiterSpace": [vp, vp, vp, i],
        "exa_projectOnDGSpace": [vp, vp, vp, i],
        "exa_findCellLocalMinAndMax": [vp, vp, i, vp, vp],
        "exa_findCellLocalLimiterMinAndMax": [vp, vp, i, i, vp, vp],
        "exa_discreteMaximumPrincipleAndMinAndMaxSearch": [vp, vp, i, d, d, vp, vp, ctypes.POINTER(i)],
        "exa_amr_limiter_projectors": [i, vp, vp, vp, vp],
    }
    for name, args in sigs.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.exa_patch_num_cells.argtypes = [vp]
    lib.exa_patch_num_cells.restype = ctypes.c_longlong
    lib.exa_patch_luh.argtypes = [vp]
    lib.exa_patch_luh.restype = ctypes.c_void_p
    lib.exa_patch_stream.argtypes = [vp]
    lib.exa_patch_stream.restype = ctypes.c_void_p
    lib.exa_patch_halo_doubles.argtypes = [vp]
    lib.exa_patch_halo_doubles.restype = ctypes.c_longlong
    lib.exa_patch_adjoint_halo_doubles.argtypes = [vp]
    lib.exa_patch_adjoint_halo_doubles.restype = ctypes.c_longlong
    _lib = lib
    return lib


def load_user_pde(path):
    """Load an application's PDE library (compiled with include/exa_aderdg_user.cuh, e.g. by
    build.build_user_pde); loading it registers its instantiations with libexa_aderdg.so."""
    load_library()
    if not os.path.exists(path):
        raise ExaError("%s is missing" % path)
    return ctypes.CDLL(path)


def pde_available(pde, dim, order, npar=0):
    return bool(load_library().exa_pde_available(int(pde), int(dim), int(order), int(npar)))


def _check(rc, what):
    if rc != EXA_OK:
        raise ExaError("%s failed (%d): %s" % (what, rc, _lib.exa_last_error().decode()))


def _ptr(t):
    """Device pointer of a contiguous torch CUDA tensor (or None)."""
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ExaError("expected a contiguous CUDA tensor")
    return ctypes.c_void_p(t.data_ptr())


def torch_float64():
    import torch
    return torch.float64


def _np_ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _dx3(dx, dim):
    a = (ctypes.c_double * 3)(1.0, 1.0, 1.0)
    v = np.broadcast_to(np.asarray(dx, dtype=float), (dim,))
    for k in range(dim):
        a[k] = float(v[k])
    return a


def _stream(stream):
    if stream is None:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    return ctypes.c_void_p(stream)


class Solver:
    """One (PDE, dim, order, nPar, precision) instantiation of the cell update."""

    def __init__(self, pde=PDE_EULER, dim=3, order=5, npar=0, cfl=0.9, pnpm=0.0, max_picard=0, precision=PREC_FP64):
        self.lib = load_library()
        cfg = _Config(dim, order, npar, pde, cfl, pnpm, max_picard, precision)
        h = ctypes.c_void_p()
        _check(self.lib.exa_solver_create(ctypes.byref(cfg), ctypes.byref(h)), "exa_solver_create")
        self.h = h
        self.dim, self.order, self.npar, self.pde = dim, order, npar, pde
        sz = _Sizes()
        _check(self.lib.exa_solver_sizes(self.h, ctypes.byref(sz)), "exa_solver_sizes")
        self.sizes = {k: getattr(sz, k) for k, _ in _Sizes._fields_}
        self.nvar, self.ndata = sz.nvar, sz.ndata

    def close(self):
        if getattr(self, "h", None):
            self.lib.exa_solver_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def status(self):
        bits = ctypes.c_uint(0)
        _check(self.lib.exa_solver_status(self.h, ctypes.byref(bits)), "exa_solver_status")
        return bits.value

    @property
    def predictor_variant(self):
        """0: one cell group per CTA, 1: persistent CTAs with a prefetched next group."""
        v = ctypes.c_int(0)
        _check(self.lib.exa_solver_predictor_variant(self.h, ctypes.byref(v)), "exa_solver_predictor_variant")
        return v.value

    def set_update_variant(self, v):
        """0: update kernel with per-thread loads; 1 / -1: bulk-copy form where possible."""
        _check(self.lib.exa_solver_set_update_variant(self.h, int(v)), "exa_solver_set_update_variant")

    @predictor_variant.setter
    def predictor_variant(self, v):
        """-1 selects the variant measured as faster on this device."""
        _check(self.lib.exa_solver_set_predictor_variant(self.h, int(v)), "exa_solver_set_predictor_variant")

    # ---- batched, device tensors -------------------------------------------------------
    def fused_predictor_volume_integral(self, luh, lduh, lQhbnd, lFhbnd, dx, dt, t=0.0, picard=None, stream=None,
                                        centres=None):
        """centres (CUDA float64 [cells][3]): the cells' centres, which an algebraic source needs."""
        ncells = luh.numel() // self.sizes["luh"]
        if centres is None:
            _check(self.lib.exa_fused_predictor_volume_integral(
                self.h, ncells, _ptr(luh), _ptr(lduh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(picard),
                _dx3(dx, self.dim), float(t), float(dt), _stream(stream)), "exa_fused_predictor_volume_integral")
        else:
            _check(self.lib.exa_fused_predictor_volume_integral_x(
                self.h, ncells, _ptr(luh), _ptr(lduh), _ptr(lQhbnd), _ptr(lFhbnd), _ptr(picard),
                _dx3(dx, self.dim), _ptr(centres), float(t), float(dt), _stream(stream)),
                "exa_fused_predictor_volume_integral_x")

    def riemann(self, left, right, direction, lQhbnd, lFhbnd, stream=None, dx=None):
        """dx (the cells' size) is needed by PDEs with a viscous flux."""
        if dx is None:
            _check(self.lib.exa_riemann_solver_nonlinear(self.h, left.numel(), _ptr(left), _ptr(right),
                                                         _ptr(direction), _ptr(lQhbnd), _ptr(lFhbnd),
                                                         _stream(stream)), "exa_riemann_solver_nonlinear")
        else:
            _check(self.lib.exa_riemann_solver_nonlinear_dx(self.h, left.numel(), _ptr(left), _ptr(right),
                                                            _ptr(direction), _ptr(lQhbnd), _ptr(lFhbnd),
                                                            _dx3(dx, self.dim), _stream(stream)),
                   "exa_riemann_solver_nonlinear_dx")

    def boundary_wall(self, cell, face, lQhbnd, lFhbnd, stream=None, dx=None):
        if dx is None:
            _check(self.lib.exa_boundary_conditions_wall(self.h, cell.numel(), _ptr(cell), _ptr(face), _ptr(lQhbnd),
                                                         _ptr(lFhbnd), _stream(stream)), "exa_boundary_conditions_wall")
        else:
            _check(self.lib.exa_boundary_conditions_wall_dx(self.h, cell.numel(), _ptr(cell), _ptr(face),
                                                            _ptr(lQhbnd), _ptr(lFhbnd), _dx3(dx, self.dim),
                                                            _stream(stream)), "exa_boundary_conditions_wall_dx")

    def surface_integral_and_update(self, luh, lduh, lFhbnd, dx, dt, stream=None):
        ncells = luh.numel() // self.sizes["luh"]
        _check(self.lib.exa_surface_integral_and_update(self.h, ncells, _ptr(luh), _ptr(lduh), _ptr(lFhbnd),
                                                        _dx3(dx, self.dim), float(dt), _stream(stream)),
               "exa_surface_integral_and_update")

    def solution_update(self, luh, luh_old, lduh, dt, stream=None):
        ncells = luh.numel() // self.sizes["luh"]
        _check(self.lib.exa_solution_update(self.h, ncells, _ptr(luh), _ptr(luh_old), _ptr(lduh), float(dt),
                                            _stream(stream)), "exa_solution_update")

    def stable_time_step_size(self, luh, dx, cell_dt=None, stream=None):
        ncells = luh.numel() // self.sizes["luh"]
        out = ctypes.c_double(0.0)
        _check(self.lib.exa_stable_time_step_size(self.h, ncells, _ptr(luh), _dx3(dx, self.dim), _ptr(cell_dt),
                                                  ctypes.byref(out), _stream(stream)), "exa_stable_time_step_size")
        return out.value

    # ---- per-cell shims, numpy host arrays ------------------------------------------------
    def space_time_predictor(self, luh, dx, dt, centre=None, t=0.0):
        s = self.sizes
        out = {k: np.zeros(s[k]) for k in ("lQhbnd", "lFhbnd", "lQi", "lFi", "lQhi", "lFhi")}
        inv = (ctypes.c_double * 3)(*(1.0 / np.broadcast_to(np.asarray(dx, float), (self.dim,))).tolist(),
                                    *([1.0] * (3 - self.dim)))
        c = np.zeros(3) if centre is None else np.ascontiguousarray(centre, dtype=float)
        luh = np.ascontiguousarray(luh, dtype=float)
        ret = self.lib.exa_spaceTimePredictorNonlinear(self.h, _np_ptr(out["lQhbnd"]), _np_ptr(out["lFhbnd"]),
                                                       _np_ptr(out["lQi"]), _np_ptr(out["lFi"]), _np_ptr(out["lQhi"]),
                                                       _np_ptr(out["lFhi"]), _np_ptr(luh), _np_ptr(c), inv, float(t),
                                                       float(dt))
        if ret < 0:
            raise ExaError("exa_spaceTimePredictorNonlinear: " + self.lib.exa_last_error().decode())
        out["ret"] = ret
        return out

    def riemann_cell(self, FL, FR, QL, QR, dx, direction):
        FL = np.ascontiguousarray(FL, dtype=float).copy()
        FR = np.ascontiguousarray(FR, dtype=float).copy()
        _check(self.lib.exa_riemannSolverNonlinear(self.h, _np_ptr(FL), _np_ptr(FR),
                                                   _np_ptr(np.ascontiguousarray(QL, dtype=float)),
                                                   _np_ptr(np.ascontiguousarray(QR, dtype=float)), 0.0, 0.0,
                                                   _dx3(dx, self.dim), int(direction)), "exa_riemannSolverNonlinear")
        return FL, FR

    def solution_update_cell(self, luh, lduh, dt):
        out = np.ascontiguousarray(luh, dtype=float).copy()
        _check(self.lib.exa_solutionUpdate(self.h, _np_ptr(out), _np_ptr(np.ascontiguousarray(luh, dtype=float)),
                                           _np_ptr(np.ascontiguousarray(lduh, dtype=float)), float(dt)),
               "exa_solutionUpdate")
        return out

    def volume_integral_cell(self, lFhi, dx):
        """volumeIntegralNonlinear of one cell from its reference lFhi blocks (host arrays)."""
        out = np.zeros(self.sizes["lduh"])
        _check(self.lib.exa_volumeIntegralNonlinear(self.h, _np_ptr(out), _np_ptr(np.ascontiguousarray(lFhi, dtype=float)),
                                                    _dx3(dx, self.dim)), "exa_volumeIntegralNonlinear")
        return out

    def surface_integral_cell(self, lduh, lFhbnd, dx):
        out = np.ascontiguousarray(lduh, dtype=float).copy()
        _check(self.lib.exa_surfaceIntegralNonlinear(self.h, _np_ptr(out), _np_ptr(np.ascontiguousarray(lFhbnd, dtype=float)),
                                                     _dx3(dx, self.dim)), "exa_surfaceIntegralNonlinear")
        return out

    def face_integral_cell(self, lduh, lFhbnd_face, direction, orientation, dx):
        out = np.ascontiguousarray(lduh, dtype=float).copy()
        _check(self.lib.exa_faceIntegralNonlinear(self.h, _np_ptr(out),
                                                  _np_ptr(np.ascontiguousarray(lFhbnd_face, dtype=float)),
                                                  int(direction), int(orientation), _dx3(dx, self.dim)),
               "exa_faceIntegralNonlinear")
        return out

    # ---- mesh levels and the limiter --------------------------------------------------------
    def amr_volume(self, mode, luh_fine, luh_coarse, jobs, group_ptr=None, stream=None):
        """Batched volume prolongation / restriction (AMR_PROLONGATE / AMR_RESTRICT) on device tensors;
        jobs: int32 [njobs][6] = (fine cell, coarse cell, levelDelta, subcell index x, y, z)."""
        s = self.sizes["luh"]
        _check(self.lib.exa_amr_volume_unknowns(
            self.h, int(mode), _ptr(luh_fine), _ptr(luh_coarse), luh_fine.numel() // s, luh_coarse.numel() // s,
            jobs.shape[0], _ptr(jobs), 0 if group_ptr is None else group_ptr.numel() - 1, _ptr(group_ptr),
            _stream(stream)), "exa_amr_volume_unknowns")

    def amr_face(self, mode, qf, ff, qc, fc, jobs, group_ptr=None, stream=None):
        """Batched face prolongation / restriction on lQhbnd / lFhbnd device tensors (blocks = cell * 2 DIM + face)."""
        nq = self.sizes["lQhbnd"] // (2 * self.dim)
        nfine = (qf.numel() // nq) if qf is not None else ff.numel() // (self.sizes["lFhbnd"] // (2 * self.dim))
        ncoarse = (qc.numel() // nq) if qc is not None else fc.numel() // (self.sizes["lFhbnd"] // (2 * self.dim))
        _check(self.lib.exa_amr_face_unknowns(
            self.h, int(mode), _ptr(qf), _ptr(ff), _ptr(qc), _ptr(fc), nfine, ncoarse, jobs.shape[0], _ptr(jobs),
            0 if group_ptr is None else group_ptr.numel() - 1, _ptr(group_ptr), _stream(stream)),
            "exa_amr_face_unknowns")

    def volume_prolongation_cell(self, luh_coarse, coarse_level, fine_level, subcell):
        out = np.zeros(self.sizes["luh"])
        idx = np.ascontiguousarray(subcell, dtype=np.int32)
        _check(self.lib.exa_volumeUnknownsProlongation(self.h, _np_ptr(out), _np_ptr(np.ascontiguousarray(luh_coarse, dtype=float)),
                                                       int(coarse_level), int(fine_level), _np_ptr(idx)),
               "exa_volumeUnknownsProlongation")
        return out

    def volume_restriction_cell(self, luh_coarse, luh_fine, coarse_level, fine_level, subcell):
        out = np.ascontiguousarray(luh_coarse, dtype=float).copy()
        idx = np.ascontiguousarray(subcell, dtype=np.int32)
        _check(self.lib.exa_volumeUnknownsRestriction(self.h, _np_ptr(out), _np_ptr(np.ascontiguousarray(luh_fine, dtype=float)),
                                                      int(coarse_level), int(fine_level), _np_ptr(idx)),
               "exa_volumeUnknownsRestriction")
        return out

    def face_prolongation_cell(self, q_coarse, f_coarse, coarse_level, fine_level, subface):
        q = np.zeros(self.sizes["lQhbnd"] // (2 * self.dim))
        f = np.zeros(self.sizes["lFhbnd"] // (2 * self.dim))
        idx = np.ascontiguousarray(subface, dtype=np.int32)
        _check(self.lib.exa_faceUnknownsProlongation(self.h, _np_ptr(q), _np_ptr(f),
                                                     _np_ptr(np.ascontiguousarray(q_coarse, dtype=float)),
                                                     _np_ptr(np.ascontiguousarray(f_coarse, dtype=float)),
                                                     int(coarse_level), int(fine_level), _np_ptr(idx)),
               "exa_faceUnknownsProlongation")
        return q, f

    def face_restriction_cell(self, q_coarse, f_coarse, q_fine, f_fine, coarse_level, fine_level, subface):
        q = np.ascontiguousarray(q_coarse, dtype=float).copy()
        f = np.ascontiguousarray(f_coarse, dtype=float).copy()
        idx = np.ascontiguousarray(subface, dtype=np.int32)
        _check(self.lib.exa_faceUnknownsRestriction(self.h, _np_ptr(q), _np_ptr(f),
                                                    _np_ptr(np.ascontiguousarray(q_fine, dtype=float)),
                                                    _np_ptr(np.ascontiguousarray(f_fine, dtype=float)),
                                                    int(coarse_level), int(fine_level), _np_ptr(idx)),
               "exa_faceUnknownsRestriction")
        return q, f

    def face_flux_restriction_cell(self, f_fine, subface, level_delta):
        f = np.zeros(self.sizes["lFhbnd"] // (2 * self.dim))
        idx = np.ascontiguousarray(subface, dtype=np.int32)
        _check(self.lib.exa_faceFluxRestriction(self.h, _np_ptr(f), _np_ptr(np.ascontiguousarray(f_fine, dtype=float)),
                                                _np_ptr(idx), int(level_delta)), "exa_faceFluxRestriction")
        return f

    def limiter_patch_size(self, ghost):
        return (2 * self.order + 1 + 2 * ghost) ** self.dim * self.ndata

    def project_on_fv_cell(self, luh, ghost, lim=None):
        out = np.zeros(self.limiter_patch_size(ghost)) if lim is None else np.ascontiguousarray(lim, dtype=float).copy()
        _check(self.lib.exa_projectOnFVLimiterSpace(self.h, _np_ptr(np.ascontiguousarray(luh, dtype=float)),
                                                    _np_ptr(out), int(ghost)), "exa_projectOnFVLimiterSpace")
        return out

    def project_on_dg_cell(self, lim, ghost):
        out = np.zeros(self.sizes["luh"])
        _check(self.lib.exa_projectOnDGSpace(self.h, _np_ptr(np.ascontiguousarray(lim, dtype=float)), _np_ptr(out),
                                             int(ghost)), "exa_projectOnDGSpace")
        return out

    def local_min_max_cell(self, luh, nobs):
        mn, mx = np.zeros(nobs), np.zeros(nobs)
        _check(self.lib.exa_findCellLocalMinAndMax(self.h, _np_ptr(np.ascontiguousarray(luh, dtype=float)), int(nobs),
                                                   _np_ptr(mn), _np_ptr(mx)), "exa_findCellLocalMinAndMax")
        return mn, mx

    def fv_min_max_cell(self, lim, ghost, nobs):
        mn, mx = np.zeros(nobs), np.zeros(nobs)
        _check(self.lib.exa_findCellLocalLimiterMinAndMax(self.h, _np_ptr(np.ascontiguousarray(lim, dtype=float)),
                                                          int(ghost), int(nobs), _np_ptr(mn), _np_ptr(mx)),
               "exa_findCellLocalLimiterMinAndMax")
        return mn, mx

    def dmp_cell(self, luh, nobs, relax, scale, bmin, bmax):
        """discreteMaximumPrincipleAndMinAndMaxSearch: returns (ok, bmin, bmax) with the rewritten blocks."""
        bmn = np.ascontiguousarray(bmin, dtype=float).copy()
        bmx = np.ascontiguousarray(bmax, dtype=float).copy()
        ok = ctypes.c_int(0)
        _check(self.lib.exa_discreteMaximumPrincipleAndMinAndMaxSearch(
            self.h, _np_ptr(np.ascontiguousarray(luh, dtype=float)), int(nobs), float(relax), float(scale),
            _np_ptr(bmn), _np_ptr(bmx), ctypes.byref(ok)), "exa_discreteMaximumPrincipleAndMinAndMaxSearch")
        return bool(ok.value), bmn, bmx

    def limiter_project_on_fv(self, luh, lim, ghost, stream=None):
        ncells = luh.numel() // self.sizes["luh"]
        _check(self.lib.exa_limiter_project_on_fv(self.h, ncells, _ptr(luh), _ptr(lim), int(ghost), _stream(stream)),
               "exa_limiter_project_on_fv")

    def limiter_project_on_dg(self, lim, luh, ghost, stream=None):
        ncells = luh.numel() // self.sizes["luh"]
        _check(self.lib.exa_limiter_project_on_dg(self.h, ncells, _ptr(lim), _ptr(luh), int(ghost), _stream(stream)),
               "exa_limiter_project_on_dg")

    def limiter_dmp(self, luh, nobs, relax, scale, bmin, bmax, ok, stream=None):
        ncells = luh.numel() // self.sizes["luh"]
        _check(self.lib.exa_limiter_dmp(self.h, ncells, _ptr(luh), int(nobs), float(relax), float(scale), _ptr(bmin),
                                        _ptr(bmax), _ptr(ok), _stream(stream)), "exa_limiter_dmp")

    def stable_time_step_size_cell(self, luh, dx):
        out = ctypes.c_double(0.0)
        _check(self.lib.exa_stableTimeStepSize(self.h, _np_ptr(np.ascontiguousarray(luh, dtype=float)),
                                               _dx3(dx, self.dim), ctypes.byref(out)), "exa_stableTimeStepSize")
        return out.value


def amr_limiter_projectors(order):
    """The mesh-level and limiter projectors of one order (host tables of the library): fine
    [3][n][n], dg2fv [n][P], fv2dg [P][n], leg2lob [n][n] with P = 2N+1."""
    lib = load_library()
    n, P = order + 1, 2 * order + 1
    out = dict(fine=np.zeros((3, n, n)), dg2fv=np.zeros((n, P)), fv2dg=np.zeros((P, n)), leg2lob=np.zeros((n, n)))
    _check(lib.exa_amr_limiter_projectors(int(order), _np_ptr(out["fine"]), _np_ptr(out["dg2fv"]),
                                          _np_ptr(out["fv2dg"]), _np_ptr(out["leg2lob"])), "exa_amr_limiter_projectors")
    return out


def grid_descs(grids):
    """ctypes array of exa_grid_desc from dicts {ncell, size, offset=0, bc=periodic (or per axis)}."""
    arr = (GridDesc * len(grids))()
    for g, spec in zip(arr, grids):
        nc = list(spec["ncell"]) + [1] * (3 - len(spec["ncell"]))
        sz = list(spec["size"]) + [1.0] * (3 - len(spec["size"]))
        off = list(spec.get("offset", [0.0] * 3)) + [0.0] * 3
        bc = spec.get("bc", BC_PERIODIC)
        bcs = list(bc) if hasattr(bc, "__len__") else [bc] * 3
        bcs = bcs + [BC_PERIODIC] * (3 - len(bcs))
        for k in range(3):
            g.ncell[k] = int(nc[k])
            g.size[k] = float(sz[k])
            g.offset[k] = float(off[k])
            g.bc[k] = int(bcs[k])
    return arr


def build_face_lists(dim, grids):
    """Host-only: the face lists exa_patch_create builds for these grids (numpy arrays)."""
    lib = load_library()
    arr = grid_descs(grids)
    fl = FaceLists()
    _check(lib.exa_build_face_lists(dim, len(grids), arr, ctypes.byref(fl)), "exa_build_face_lists")
    left = np.zeros(fl.nfaces, dtype=np.int32)
    right = np.zeros(fl.nfaces, dtype=np.int32)
    d = np.zeros(fl.nfaces, dtype=np.int8)
    bcell = np.zeros(max(fl.nbfaces, 1), dtype=np.int32)
    bface = np.zeros(max(fl.nbfaces, 1), dtype=np.int8)
    fl.left, fl.right, fl.dir = _np_ptr(left), _np_ptr(right), _np_ptr(d)
    fl.bcell, fl.bface = _np_ptr(bcell), _np_ptr(bface)
    _check(lib.exa_build_face_lists(dim, len(grids), arr, ctypes.byref(fl)), "exa_build_face_lists")
    return {"ncells": fl.ncells, "nghost": fl.nghost, "left": left, "right": right, "dir": d,
            "bcell": bcell[:fl.nbfaces], "bface": bface[:fl.nbfaces]}


def checkpoint_schedule(steps, snaps):
    """Host-only: the binomial checkpointing schedule (list of (action, a, b)) and its forward steps."""
    lib = load_library()
    cnt = ctypes.c_int(0)
    fw = ctypes.c_longlong(0)
    _check(lib.exa_checkpoint_schedule(int(steps), int(snaps), None, 0, ctypes.byref(cnt), ctypes.byref(fw)),
           "exa_checkpoint_schedule")
    arr = (CkAction * cnt.value)()
    _check(lib.exa_checkpoint_schedule(int(steps), int(snaps), arr, cnt.value, ctypes.byref(cnt), ctypes.byref(fw)),
           "exa_checkpoint_schedule")
    return [(x.action, x.a, x.b) for x in arr], int(fw.value)


class Patch:
    """Device-resident uniform grid(s); the step is one CUDA graph launch."""

    def __init__(self, solver, grids):
        """grids: list of dicts {ncell, size, offset=0, bc=periodic} (bc per axis)."""
        self.solver = solver
        self.lib = solver.lib
        arr = grid_descs(grids)
        h = ctypes.c_void_p()
        _check(self.lib.exa_patch_create(solver.h, len(grids), arr, ctypes.byref(h)), "exa_patch_create")
        self.h = h
        self.ngrids = len(grids)
        self.ncells = int(self.lib.exa_patch_num_cells(self.h))

    def step_phase(self, phase, fixed_dt=0.0):
        _check(self.lib.exa_patch_step_phase(self.h, int(phase), float(fixed_dt)), "exa_patch_step_phase")

    def halo_doubles(self):
        return int(self.lib.exa_patch_halo_doubles(self.h))

    def halo_pack(self, send_lo, send_hi):
        _check(self.lib.exa_patch_halo_pack(self.h, _ptr(send_lo), _ptr(send_hi)), "exa_patch_halo_pack")

    def halo_unpack(self, recv_lo, recv_hi):
        _check(self.lib.exa_patch_halo_unpack(self.h, _ptr(recv_lo), _ptr(recv_hi)), "exa_patch_halo_unpack")

    def dt_next_copy(self, buf, to_patch):
        _check(self.lib.exa_patch_dt_next_copy(self.h, _ptr(buf), int(to_patch)), "exa_patch_dt_next_copy")

    def adjust_solution(self):
        """The functor's adjust_point_solution at every node (device initial conditions)."""
        _check(self.lib.exa_patch_adjust_solution(self.h), "exa_patch_adjust_solution")

    def set_point_source(self, x, f0=0.0, t0=0.0, amplitude=0.0, width=1.0, variable=0):
        """Ricker point source on `variable` (acoustic / elastic solvers); x=None removes it."""
        if x is None:
            _check(self.lib.exa_patch_set_point_source(self.h, None), "exa_patch_set_point_source")
            return
        ps = PointSource((ctypes.c_double * 3)(*list(x) + [0.0] * (3 - len(x))), f0, t0, amplitude, width,
                         int(variable))
        _check(self.lib.exa_patch_set_point_source(self.h, ctypes.byref(ps)), "exa_patch_set_point_source")

    def dt_copy(self, buf, to_patch):
        _check(self.lib.exa_patch_dt_copy(self.h, _ptr(buf), int(to_patch)), "exa_patch_dt_copy")

    def step_host(self, luh_in, luh_out, fixed_dt=0.0, nsteps=1):
        """nsteps steps of a host-resident state (numpy arrays or CPU torch tensors, pinned for
        overlap): every step uploads, steps and downloads, copies pipelined with the kernels."""
        def hptr(x):
            if isinstance(x, np.ndarray):
                if x.dtype != np.float64 or not x.flags["C_CONTIGUOUS"]:
                    raise ExaError("expected a contiguous float64 array")
                return _np_ptr(x)
            if x.is_cuda or not x.is_contiguous() or x.dtype != torch_float64():
                raise ExaError("expected a contiguous float64 CPU tensor")
            return ctypes.c_void_p(x.data_ptr())
        _check(self.lib.exa_patch_run_host(self.h, hptr(luh_in), hptr(luh_out), int(nsteps), float(fixed_dt)),
               "exa_patch_run_host")

    def set_time(self, t):
        _check(self.lib.exa_patch_set_time(self.h, float(t)), "exa_patch_set_time")

    def adjoint_step(self, lam, dt):
        """lam (CUDA float64 tensor, luh layout): dJ/du_{k+1} in, dJ/du_k out (parameters accumulate)."""
        _check(self.lib.exa_patch_adjoint_step(self.h, _ptr(lam), float(dt)), "exa_patch_adjoint_step")

    def adjoint_phase(self, phase, lam, dt):
        """ADJ_FORWARD takes lam (this patch's cells) in; ADJ_REVERSE writes the result into it. A halo
        patch exchanges the face traces (halo_pack / halo_unpack) and the boundary layers' lambda
        (adjoint_halo_pack / adjoint_halo_unpack) in between."""
        _check(self.lib.exa_patch_adjoint_phase(self.h, int(phase), _ptr(lam), float(dt)), "exa_patch_adjoint_phase")

    def adjoint_halo_doubles(self):
        return int(self.lib.exa_patch_adjoint_halo_doubles(self.h))

    def adjoint_halo_pack(self, send_lo, send_hi):
        _check(self.lib.exa_patch_adjoint_halo_pack(self.h, _ptr(send_lo), _ptr(send_hi)),
               "exa_patch_adjoint_halo_pack")

    def adjoint_halo_unpack(self, recv_lo, recv_hi):
        _check(self.lib.exa_patch_adjoint_halo_unpack(self.h, _ptr(recv_lo), _ptr(recv_hi)),
               "exa_patch_adjoint_halo_unpack")

    def close(self):
        if getattr(self, "h", None):
            self.lib.exa_patch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def luh_ptr(self):
        return self.lib.exa_patch_luh(self.h)

    @property
    def stream(self):
        return self.lib.exa_patch_stream(self.h)

    def set_solution(self, luh):
        """luh: numpy host array (reference layout) or a CUDA tensor."""
        if isinstance(luh, np.ndarray):
            a = np.ascontiguousarray(luh, dtype=np.float64)
            _check(self.lib.exa_patch_set_solution(self.h, _np_ptr(a), 0), "exa_patch_set_solution")
        else:
            _check(self.lib.exa_patch_set_solution(self.h, _ptr(luh), 1), "exa_patch_set_solution")

    def get_solution(self, out=None):
        if out is None:
            out = np.zeros(self.ncells * self.solver.sizes["luh"])
            _check(self.lib.exa_patch_get_solution(self.h, _np_ptr(out), 0), "exa_patch_get_solution")
            return out
        if isinstance(out, np.ndarray):
            _check(self.lib.exa_patch_get_solution(self.h, _np_ptr(out), 0), "exa_patch_get_solution")
        else:
            _check(self.lib.exa_patch_get_solution(self.h, _ptr(out), 1), "exa_patch_get_solution")
        return out

    def step(self, nsteps=1, fixed_dt=0.0):
        _check(self.lib.exa_patch_step(self.h, int(nsteps), float(fixed_dt)), "exa_patch_step")

    def sync(self):
        _check(self.lib.exa_patch_sync(self.h), "exa_patch_sync")

    def time(self):
        t = np.zeros(self.ngrids)
        dt = np.zeros(self.ngrids)
        _check(self.lib.exa_patch_time(self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       dt.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "exa_patch_time")
        return t, dt

    def stats(self):
        st = _PatchStats()
        _check(self.lib.exa_patch_stats_get(self.h, ctypes.byref(st)), "exa_patch_stats_get")
        return {"steps": st.steps, "picard_mean": st.picard_mean, "picard_hist": list(st.picard_hist)}

    def status(self):
        bits = ctypes.c_uint(0)
        _check(self.lib.exa_patch_status(self.h, ctypes.byref(bits)), "exa_patch_status")
        return bits.value
