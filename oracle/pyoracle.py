"""ctypes bindings of the CPU checkers. TEST INFRASTRUCTURE ONLY.

``Oracle``    -- oracle/liboracle.so, the C restatement of the reference's generic kernels.
``RefKernels`` -- oracle/_ref/libexaref{2,3}d.so, the reference's OWN generic kernels compiled in
                 place behind a shim (present only where the reference checkout was available at
                 build time; the built libraries travel with the repository snapshot).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

PDE_EULER, PDE_SWE, PDE_ACOUSTIC, PDE_ELASTIC = 0, 1, 2, 3
# ADER-DG PNPM table by order (Toolkit/exahype/toolkit/solverController.py:17)
PNPM = [1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015]


class ExoCfg(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("order", ctypes.c_int), ("nvar", ctypes.c_int), ("npar", ctypes.c_int),
                ("pde", ctypes.c_int), ("use_ncp", ctypes.c_int), ("cfl", ctypes.c_double),
                ("pnpm", ctypes.c_double), ("max_picard", ctypes.c_int), ("has_src", ctypes.c_int),
                ("src", ctypes.c_double * 8)]

NVAR = {PDE_EULER: 5, PDE_SWE: 4, PDE_ACOUSTIC: 4, PDE_ELASTIC: 9}
NPAR = {PDE_EULER: 0, PDE_SWE: 0, PDE_ACOUSTIC: 2, PDE_ELASTIC: 3}


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """The C restatement, one configuration (dim, order, PDE) per instance."""

    def __init__(self, dim, order, pde=PDE_EULER, nvar=None, npar=None, cfl=0.9, max_picard=0, source=None):
        """source: (x, y, z, f0, t0, amplitude, width, variable) of the point source, or None."""
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run make -C oracle")
        self.lib = ctypes.CDLL(path)
        self.lib.exo_predictor.restype = ctypes.c_int
        self.lib.exo_dt.restype = ctypes.c_double
        if nvar is None:
            nvar = NVAR[pde]
        if npar is None:
            npar = NPAR[pde]
        src = (ctypes.c_double * 8)(*(list(source) if source is not None else [0.0] * 8))
        self.cfg = ExoCfg(dim, order, nvar, npar, pde, 1 if pde == PDE_SWE else 0, cfl, PNPM[order], max_picard,
                          1 if source is not None else 0, src)
        self.dim, self.n, self.v, self.D = dim, order + 1, nvar, nvar + npar
        self.nd = self.n ** dim
        self.nf = self.n ** (dim - 1)

    def tables(self):
        n = self.n
        t = {k: np.zeros(n) for k in ("nodes", "weights", "F0", "F1")}
        for k in ("Kxi", "iK1", "dudx"):
            t[k] = np.zeros((n, n))
        self.lib.exo_tables(n - 1, _p(t["nodes"]), _p(t["weights"]), _p(t["Kxi"]), _p(t["iK1"]), _p(t["dudx"]),
                            _p(t["F0"]), _p(t["F1"]))
        return t

    def _dx(self, dx):
        d = np.zeros(3)
        d[: self.dim] = dx[: self.dim] if np.ndim(dx) else dx
        return d

    def predictor(self, luh, dx, dt, centre=None, t=0.0):
        n, nd, D, v, dim = self.n, self.nd, self.D, self.v, self.dim
        out = dict(lQi=np.zeros(nd * n * D), lFi=np.zeros(n * nd * (dim + 1) * v), lQhi=np.zeros(nd * D),
                   lFhi=np.zeros((dim + 1) * nd * v), lQhbnd=np.zeros(2 * dim * self.nf * D),
                   lFhbnd=np.zeros(2 * dim * self.nf * v))
        sw = ctypes.c_int(0)
        c = np.zeros(3) if centre is None else _f64(centre)
        ret = self.lib.exo_predictor(ctypes.byref(self.cfg), _p(_f64(luh)), _p(c), _p(self._dx(dx)),
                                     ctypes.c_double(t), ctypes.c_double(dt), _p(out["lQi"]), _p(out["lFi"]),
                                     _p(out["lQhi"]), _p(out["lFhi"]), _p(out["lQhbnd"]), _p(out["lFhbnd"]),
                                     ctypes.byref(sw))
        out["ret"] = ret
        out["sweeps"] = sw.value
        return out

    def volume(self, lFhi, dx):
        lduh = np.zeros(self.nd * self.v)
        self.lib.exo_volume(ctypes.byref(self.cfg), _p(lduh), _p(_f64(lFhi)), _p(self._dx(dx)))
        return lduh

    def riemann(self, FL, FR, QL, QR, dx, direction):
        FL, FR = _f64(FL).copy(), _f64(FR).copy()
        self.lib.exo_riemann(ctypes.byref(self.cfg), _p(FL), _p(FR), _p(_f64(QL)), _p(_f64(QR)), _p(self._dx(dx)),
                             int(direction))
        return FL, FR

    def surface(self, lduh, lFhbnd, dx):
        lduh = _f64(lduh).copy()
        self.lib.exo_surface(ctypes.byref(self.cfg), _p(lduh), _p(_f64(lFhbnd)), _p(self._dx(dx)))
        return lduh

    def face(self, lduh, lFhbnd_face, direction, orientation, dx):
        lduh = _f64(lduh).copy()
        self.lib.exo_face(ctypes.byref(self.cfg), _p(lduh), _p(_f64(lFhbnd_face)), int(direction), int(orientation),
                          _p(self._dx(dx)))
        return lduh

    def update(self, luh, lduh, dt):
        out = _f64(luh).copy()
        self.lib.exo_update(ctypes.byref(self.cfg), _p(out), _p(_f64(luh)), _p(_f64(lduh)), ctypes.c_double(dt))
        return out

    def dt(self, luh, dx):
        return float(self.lib.exo_dt(ctypes.byref(self.cfg), _p(_f64(luh)), _p(self._dx(dx))))

    def flux(self, Q):
        F = np.zeros(self.dim * self.v)
        self.lib.exo_flux(ctypes.byref(self.cfg), _p(_f64(Q)), _p(F))
        return F.reshape(self.dim, self.v)

    def run(self, luh, ncell, size, nsteps, offset=(0.0, 0.0, 0.0), walls=False, t0=0.0, fixed_dt=0.0,
            nthreads=0, want_picard=False):
        """Advance a uniform patch in place; returns (t, dts, picard sweeps per step and cell).

        walls: False / 0 periodic, True / 1 reflective walls, 3 outflow on every domain face."""
        luh = np.ascontiguousarray(luh, dtype=np.float64)
        nc = int(np.prod(ncell))
        dts = np.zeros(nsteps)
        pic = np.zeros(nsteps * nc, dtype=np.int32) if want_picard else None
        t = ctypes.c_double(0.0)
        nce = np.array(list(ncell) + [1] * (3 - len(ncell)), dtype=np.int32)
        self.lib.exo_run(ctypes.byref(self.cfg), _p(nce), _p(self._dx(np.array(offset, dtype=float))),
                         _p(self._dx(np.array(size, dtype=float))), int(walls), _p(luh), int(nsteps),
                         ctypes.c_double(t0), ctypes.c_double(fixed_dt), ctypes.byref(t), _p(dts),
                         _p(pic) if pic is not None else None, int(nthreads))
        return t.value, dts, (pic.reshape(nsteps, nc) if pic is not None else None)


class RefKernels:
    """The reference's own generic kernels (oracle/_ref), one instantiation per instance."""

    def __init__(self, dim, order, pde="euler", npar=0, source=None):
        """source: point source (x, y, z, f0, t0, amplitude, width, variable) for the acoustic and
        elastic instantiations (process-wide setting of the library), or None. pde "acousticfixed"
        / "elasticfixed": the same systems with a fixed Picard count (UseMaxPicardIterations)."""
        path = os.path.join(HERE, "_ref", "libexaref%dd.so" % dim)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.prefix = "exaref%dd_%s_o%d_p%d" % (dim, pde, order, npar)
        if not hasattr(self.lib, self.prefix + "_predictor"):
            raise AttributeError("instantiation %s not built" % self.prefix)
        self.dim, self.n = dim, order + 1
        self.v = {"euler": 5, "swe": 4, "acoustic": 4, "elastic": 9, "acousticfixed": 4, "elasticfixed": 9,
                  "advdiff": 3, "advreact": 3}[pde]
        src = (ctypes.c_double * 8)(*(list(source) if source is not None else [0, 0, 0, 0, 0, 0, 1, 0]))
        self.lib.exaref_set_source(src, 1 if source is not None else 0)
        self.D = self.v + npar
        self.nd, self.nf = self.n ** dim, self.n ** (dim - 1)
        getattr(self.lib, self.prefix + "_predictor").restype = ctypes.c_int
        getattr(self.lib, self.prefix + "_dt").restype = ctypes.c_double

    def _f(self, name):
        return getattr(self.lib, self.prefix + "_" + name)

    def _dx(self, dx):
        d = np.zeros(3)
        d[: self.dim] = dx[: self.dim] if np.ndim(dx) else dx
        return d

    def predictor(self, luh, dx, dt, centre=None, t=0.0):
        n, nd, D, v, dim = self.n, self.nd, self.D, self.v, self.dim
        out = dict(lQi=np.zeros(nd * n * D), rhs=np.zeros(nd * n * D), lFi=np.zeros(n * nd * (dim + 1) * v),
                   gradQ=np.zeros(dim * v * nd), lQhi=np.zeros(nd * D), lFhi=np.zeros((dim + 1) * nd * v),
                   lQhbnd=np.zeros(2 * dim * self.nf * D), lFhbnd=np.zeros(2 * dim * self.nf * v))
        c = np.zeros(3) if centre is None else _f64(centre)
        out["ret"] = self._f("predictor")(_p(_f64(luh)), _p(c), _p(self._dx(dx)), ctypes.c_double(t),
                                          ctypes.c_double(dt), _p(out["lQi"]), _p(out["rhs"]), _p(out["lFi"]),
                                          _p(out["gradQ"]), _p(out["lQhi"]), _p(out["lFhi"]), _p(out["lQhbnd"]),
                                          _p(out["lFhbnd"]))
        return out

    def volume(self, lFhi, dx):
        lduh = np.zeros(self.nd * self.v)
        self._f("volume")(_p(lduh), _p(_f64(lFhi)), _p(self._dx(dx)))
        return lduh

    def riemann(self, FL, FR, QL, QR, dx, direction):
        FL, FR = _f64(FL).copy(), _f64(FR).copy()
        self._f("riemann")(_p(FL), _p(FR), _p(_f64(QL)), _p(_f64(QR)), ctypes.c_double(0.0), ctypes.c_double(0.0),
                           _p(self._dx(dx)), int(direction))
        return FL, FR

    def surface(self, lduh, lFhbnd, dx):
        lduh = _f64(lduh).copy()
        self._f("surface")(_p(lduh), _p(_f64(lFhbnd)), _p(self._dx(dx)))
        return lduh

    def face(self, lduh, lFhbnd_face, direction, orientation, dx):
        lduh = _f64(lduh).copy()
        self._f("face")(_p(lduh), _p(_f64(lFhbnd_face)), int(direction), int(orientation), _p(self._dx(dx)))
        return lduh

    def update(self, luh, lduh, dt):
        out = _f64(luh).copy()
        self._f("update")(_p(out), _p(_f64(luh)), _p(_f64(lduh)), ctypes.c_double(dt))
        return out

    def dt(self, luh, dx):
        return float(self._f("dt")(_p(_f64(luh)), _p(self._dx(dx))))

    def run(self, luh, ncell, size, nsteps, offset=(0.0, 0.0, 0.0), walls=False, t0=0.0, fixed_dt=0.0,
            nthreads=0, want_picard=False):
        luh = np.ascontiguousarray(luh, dtype=np.float64)
        nc = int(np.prod(ncell))
        dts = np.zeros(nsteps)
        pic = np.zeros(nsteps * nc, dtype=np.int32) if want_picard else None
        t = ctypes.c_double(0.0)
        nce = np.array(list(ncell) + [1] * (3 - len(ncell)), dtype=np.int32)
        self._f("run")(_p(nce), _p(self._dx(np.array(offset, dtype=float))), _p(self._dx(np.array(size, dtype=float))),
                       int(walls), _p(luh), int(nsteps), ctypes.c_double(t0), ctypes.c_double(fixed_dt),
                       ctypes.byref(t), _p(dts), _p(pic) if pic is not None else None, int(nthreads))
        return t.value, dts, (pic.reshape(nsteps, nc) if pic is not None else None)


class RefLinear:
    """The reference's linear generic kernels (Cauchy-Kowalewski predictor, linear Riemann solver,
    delta-distribution point source) with the PDE terms of its own linear applications: "elastic"
    (ElasticWave3D: v1 v2 v3 s11 s22 s33 s12 s13 s23 + rho cp cs) or "acoustic" (acousticwaveCPP:
    p, u1, u2, u3 with unit density and speed, u = minus the flux-form velocity). 3D, orders 3, 4."""

    def __init__(self, pde, order, source=None):
        """source: (x, y, z, f0, t0, amplitude, -, variable): a delta at (x, y, z) with amplitude
        times the Ricker wavelet of peak frequency f0 delayed by t0 on `variable`, or None."""
        path = os.path.join(HERE, "_ref", "libexaref3d.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.prefix = "exalin_%s_o%d" % (pde, order)
        if not hasattr(self.lib, self.prefix + "_run"):
            raise AttributeError("instantiation %s not built" % self.prefix)
        self.elastic = pde == "elastic"
        self.v, self.npar = (9, 3) if self.elastic else (4, 0)
        self.D, self.n = self.v + self.npar, order + 1
        src = (ctypes.c_double * 8)(*(list(source) if source is not None else [0, 0, 0, 0, 0, 0, 1, 0]))
        self.lib.exaref_set_source(src, 1 if source is not None else 0)

    def terms(self, Q, G):
        """M(Q) (F_d(G_d) + B_d(G)) for d = 0, 1, 2: the d-th term of -dQ/dt for a field with state Q
        (parameters included) and per-direction gradients G[d] of the variables."""
        out = np.zeros((3, self.v))
        fn = self.lib.exalin_elastic_terms if self.elastic else self.lib.exalin_acoustic_terms
        fn(_p(_f64(Q)), _p(_f64(np.asarray(G).reshape(3, self.v))), _p(out))
        return out

    def eigenvalues(self, Q):
        out = np.zeros(self.v)
        self.lib.exalin_eigenvalues(1 if self.elastic else 0, _p(_f64(Q)), _p(out))
        return out

    def run(self, luh, ncell, size, nsteps, offset=(0.0, 0.0, 0.0), t0=0.0, fixed_dt=0.0, nthreads=0):
        """Periodic uniform patch, luh [cells][n^3][D] updated in place; returns (t, dts)."""
        luh = np.ascontiguousarray(luh, dtype=np.float64)
        dts = np.zeros(nsteps)
        t = ctypes.c_double(0.0)
        nce = np.array(list(ncell), dtype=np.int32)
        self.lib[self.prefix + "_run"](_p(nce), _p(_f64(offset)), _p(_f64(size)), _p(luh), int(nsteps),
                                       ctypes.c_double(t0), ctypes.c_double(fixed_dt), ctypes.byref(t), _p(dts),
                                       int(nthreads))
        return t.value, dts


class RefAmrLimiter:
    """The reference's mesh-level (3d/amrRoutines.cpph) and limiter (limiter/generic/c/Limiter.cpph)
    kernels, 3D, for (order, nVar, nPar) in (3,5,0), (3,5,1), (5,5,0), (4,4,2), (4,9,3)
    (oracle/_ref/libexaref_amrlim3d.so). DMP observables: the first nVar variables."""

    def __init__(self, order, nvar, npar, dim=3):
        """dim 2: (order, nVar, nPar) in (3,5,0), (3,5,1), (4,4,0) (libexaref_amrlim2d.so)."""
        path = os.path.join(HERE, "_ref", "libexaref_amrlim%dd.so" % dim)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.order, self.nvar, self.npar, self.dim = order, nvar, npar, dim
        self.n, self.D, self.P = order + 1, nvar + npar, 2 * order + 1

    def _idx(self, idx):
        a = np.zeros(3, dtype=np.int32)
        a[: len(idx)] = idx
        return a

    def volume(self, mode, out, inp, coarse_level, fine_level, idx):
        """mode 0: out (fine luh) = prolongation of inp (coarse); 1: out (coarse) += restriction of inp."""
        out = _f64(out).copy()
        r = self.lib.exaamr_volume(self.order, self.nvar, self.npar, int(mode), _p(out), _p(_f64(inp)),
                                   int(coarse_level), int(fine_level), _p(self._idx(idx)))
        assert r == 0, "configuration not built"
        return out

    def face(self, mode, outQ, outF, inQ, inF, coarse_level, fine_level, idx):
        """mode 0 prolongation, 1 restriction (accumulating), 2 flux-only restriction (overwrite)."""
        outQ, outF = _f64(outQ).copy(), _f64(outF).copy()
        r = self.lib.exaamr_face(self.order, self.nvar, self.npar, int(mode), _p(outQ), _p(outF), _p(_f64(inQ)),
                                 _p(_f64(inF)), int(coarse_level), int(fine_level), _p(self._idx(idx)))
        assert r == 0, "configuration not built"
        return outQ, outF

    def limiter(self, op, a, ghost=0, out=None, mn=None, mx=None, relax=0.0, scale=0.0):
        """op 0 luh -> lim, 1 lim -> luh, 2 / 3 min and max (observables = the first nVar variables),
        4 discrete maximum principle (mn / mx [2 DIM][nVar] in/out); returns (result, out, mn, mx)."""
        out = None if out is None else _f64(out).copy()
        mn = None if mn is None else _f64(mn).copy()
        mx = None if mx is None else _f64(mx).copy()
        self.lib.exaamr_limiter.restype = ctypes.c_int
        r = self.lib.exaamr_limiter(self.order, self.nvar, self.npar, int(ghost), int(op), _p(_f64(a)),
                                    _p(out) if out is not None else None, _p(mn) if mn is not None else None,
                                    _p(mx) if mx is not None else None, ctypes.c_double(relax), ctypes.c_double(scale))
        assert r >= 0, "configuration not built"
        return r, out, mn, mx

    @staticmethod
    def tables(order):
        lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libexaref_amrlim3d.so"))
        n, P = order + 1, 2 * order + 1
        fine, d, v, l = np.zeros(3 * n * n), np.zeros(n * P), np.zeros(n * P), np.zeros(n * n)
        lib.exaamr_fine_grid_projector(int(order), _p(fine))
        lib.exaamr_limiter_projectors(int(order), _p(d), _p(v), _p(l))
        return dict(fine=fine.reshape(3, n, n), dg2fv=d.reshape(n, P), fv2dg=v.reshape(P, n), leg2lob=l.reshape(n, n))


class KGKernels:
    """The reference's generated optimised kernels (KernelGenerator, plain-loop mode) for the Euler
    application, 3D, order 3 or 5 (oracle/_ref/libkg_euler_o{3,5}.so, built by ``make -C oracle kg``)
    behind a uniform-patch driver with the generic glue's step order. Cubic cells only."""

    def __init__(self, order):
        path = os.path.join(HERE, "_ref", "libkg_euler_o%d.so" % order)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.kgref_run.restype = ctypes.c_int
        self.order = order

    def run(self, luh, ncell, size, nsteps, walls=False, fixed_dt=0.0, nthreads=0, want_picard=False):
        luh = np.ascontiguousarray(luh, dtype=np.float64)
        nc = int(np.prod(ncell))
        dts = np.zeros(nsteps)
        pic = np.zeros(nsteps * nc, dtype=np.int32) if want_picard else None
        t = ctypes.c_double(0.0)
        nce = np.array(list(ncell), dtype=np.int32)
        sz = np.array(list(size), dtype=np.float64)
        self.lib.kgref_run(_p(nce), _p(sz), int(walls), _p(luh), int(nsteps), ctypes.c_double(fixed_dt),
                           ctypes.byref(t), _p(dts), _p(pic) if pic is not None else None, int(nthreads))
        return t.value, dts, (pic.reshape(nsteps, nc) if pic is not None else None)
