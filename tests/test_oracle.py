"""Pins the CPU oracle (oracle/oracle.c) to the reference.

(a) against the reference's own known-answer arrays
    (ExaHyPE/exahype/tests/kernels/testdata/generic_euler_testdata.cpp -> tests/golden/*.npz),
    with the inputs the reference's tests build (tests/kernels/c/GenericEulerKernelTest{2D,3D}.cpp);
(b) against the reference's own generic kernels run on seeded NON-constant cells
    (tests/golden/picard_*.npz, written by tests/golden/make_golden.py through oracle/_ref);
(c) directly against oracle/_ref when that library is present (differential, random inputs).
"""
import os

import numpy as np
import pytest

from pyoracle import Oracle, RefKernels

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
EPS_REF = 1e-10  # the reference tests' tolerance (GenericEulerKernelTest.h:96)


def g3():
    return np.load(os.path.join(GOLD, "generic_euler_3d.npz"))


def g2():
    return np.load(os.path.join(GOLD, "generic_euler_2d.npz"))


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


def with_params(arr, nvar, npar):
    """Re-stride a [nodes][nVar] golden array to [nodes][nVar+nPar] (parameters zero)."""
    a = np.asarray(arr).reshape(-1, nvar)
    out = np.zeros((a.shape[0], nvar + npar))
    out[:, :nvar] = a
    return out.reshape(-1)


def strip_params(arr, nvar, npar):
    return np.asarray(arr).reshape(-1, nvar + npar)[:, :nvar].reshape(-1)


@pytest.mark.parametrize("order", [1, 3, 5, 7, 9])
def test_tables_match_reference_snippet(order):
    ref = np.load(os.path.join(GOLD, "gl_tables.npz"))
    t = Oracle(3, order).tables()
    for k, rk in (("nodes", "nodes"), ("weights", "weights"), ("Kxi", "Kxi"), ("iK1", "iK1"), ("dudx", "dudx"),
                  ("F0", "FCoeff0"), ("F1", "FCoeff1")):
        r = ref["%s_%d" % (rk, order)]
        assert np.max(np.abs(t[k] - r)) <= 4e-16 * max(1.0, np.max(np.abs(r))), (k, order)


# ---------------------------------------------------------------------------------------------
# 3D known-answer tests (GenericEulerKernelTest3D.cpp), Euler N=3, nVar=5, nPar=1
# ---------------------------------------------------------------------------------------------

def test_golden3d_riemann():
    g = g3()
    o = Oracle(3, 3, npar=1)
    FL = np.arange(1, 81, dtype=float)
    FR = np.arange(-1, 79, dtype=float)
    QL = with_params(g["testRiemannSolver.QL"], 5, 1)
    QR = with_params(g["testRiemannSolver.QR"], 5, 1)
    FLo, FRo = o.riemann(FL, FR, QL, QR, 0.5, 1)
    assert np.max(np.abs(FLo - g["testRiemannSolverNonlinear.FL"])) < EPS_REF
    assert np.max(np.abs(FRo - g["testRiemannSolverNonlinear.FR"])) < EPS_REF


def test_golden3d_surface_integral():
    g = g3()
    o = Oracle(3, 3, npar=1)
    lF = np.zeros(480)
    for i in range(0, 80, 5):
        lF[0 + i + 1] = lF[80 + i + 1] = 1.0
        lF[160 + i + 2] = lF[240 + i + 2] = 1.0
        lF[320 + i + 3] = lF[400 + i + 3] = 1.0
    lduh = np.arange(320) / 10.0
    out = o.surface(lduh, lF, 0.1)
    assert np.max(np.abs(out - g["testSurfaceIntegralNonlinear.lduh"])) < EPS_REF


def test_golden3d_solution_update():
    g = g3()
    o = Oracle(3, 3, npar=1)
    luh = np.zeros(6 * 64)
    luh[0::6] = 1.0
    luh[4::6] = 2.5
    lduh = np.arange(320, dtype=float)
    out = o.update(luh, lduh, 1.40831757919882352703e-03)
    # the reference test checks the first basisSize^2 nodes (GenericEulerKernelTest3D.cpp:495-503)
    ref = g["testSolutionUpdate.luh"]
    got = strip_params(out, 5, 1)
    assert np.max(np.abs(got[:80] - ref[:80])) < EPS_REF
    # every node: the fixture holds exactly the reference formula for all 64 nodes
    assert np.max(np.abs(got - ref)) < EPS_REF


def test_golden3d_predictor_constant_state():
    g = g3()
    o = Oracle(3, 3, npar=1)
    luh = with_params(g["testSpaceTimePredictorNonlinear.luh"], 5, 1)
    r = o.predictor(luh, [0.05, 0.05, 0.05], 1.083937460199773e-3)
    assert r["ret"] == 0  # constant state: converged in the first sweep
    assert np.max(np.abs(strip_params(r["lQi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQi"])) < EPS_REF
    lFi = r["lFi"].reshape(4, 64, 4, 5)[:, :, :3, :].reshape(-1)
    assert np.max(np.abs(lFi - g["testSpaceTimePredictorNonlinear.lFi"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhbnd"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhbnd"])) < EPS_REF
    assert np.max(np.abs(r["lFhbnd"] - g["testSpaceTimePredictorNonlinear.lFhbnd"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhi"])) < EPS_REF
    assert np.max(np.abs(r["lFhi"][:960] - g["testSpaceTimePredictorNonlinear.lFhi"])) < EPS_REF


# ---------------------------------------------------------------------------------------------
# 2D known-answer tests (GenericEulerKernelTest2D.cpp)
# ---------------------------------------------------------------------------------------------

def test_golden2d_riemann():
    g = g2()
    o = Oracle(2, 3, npar=1)
    for case, direction in ((1, 0), (2, 1)):
        QL = with_params(g["testRiemannSolverNonlinear.QL_%d_in" % case], 5, 1)
        QR = with_params(g["testRiemannSolverNonlinear.QR_%d_in" % case], 5, 1)
        FL, FR = o.riemann(g["testRiemannSolverNonlinear.FL_%d_in" % case],
                           g["testRiemannSolverNonlinear.FR_%d_in" % case], QL, QR, 0.5, direction)
        ref = g["testRiemannSolverNonlinear.F_%d_out" % case]
        assert np.max(np.abs(FL - ref)) < EPS_REF
        assert np.max(np.abs(FR - ref)) < EPS_REF


def test_golden2d_surface_integral():
    g = g2()
    o = Oracle(2, 3, npar=1)
    lF = np.zeros(80)
    for i in range(0, 20, 5):
        lF[i + 1] = lF[20 + i + 1] = 1.0
        lF[40 + i + 2] = lF[60 + i + 2] = 1.0
    out1 = o.surface(g["testSurfaceIntegral.lduh_in"], lF, 0.1)
    assert np.max(np.abs(out1 - g["testSurfaceIntegralNonlinear.lduh_1"])) < EPS_REF
    out2 = o.surface(g["testSurfaceIntegral.lduh_in"], g["testSurfaceIntegral.lFhbnd_in"], 0.1)
    assert np.max(np.abs(out2 - g["testSurfaceIntegralNonlinear.lduh_2"])) < EPS_REF


def test_golden2d_solution_update():
    g = g2()
    o = Oracle(2, 3, npar=1)
    luh = np.zeros(6 * 16)
    luh[0::6] = 1.0
    luh[4::6] = 2.5
    out = o.update(luh, g["testSolutionUpdate.lduh"], 1.40831757919882352703e-03)
    assert np.max(np.abs(strip_params(out, 5, 1) - g["testSolutionUpdate.luh"])) < EPS_REF


def test_golden2d_predictor_constant_state():
    g = g2()
    o = Oracle(2, 3, npar=1)
    luh = with_params(g["testSpaceTimePredictorNonlinear.luh"], 5, 1)
    r = o.predictor(luh, [0.05, 0.05], 1.686854344081342e-3)
    assert r["ret"] == 2 * 4 + 2  # 2D returns MaxIterations+2 on convergence (2d/...:303-305)
    assert np.max(np.abs(strip_params(r["lQi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQi"])) < EPS_REF
    lFi = r["lFi"].reshape(4, 16, 3, 5)[:, :, :2, :].reshape(-1)
    assert np.max(np.abs(lFi - g["testSpaceTimePredictorNonlinear.lFi"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhi"])) < EPS_REF
    assert np.max(np.abs(r["lFhi"][:160] - g["testSpaceTimePredictorNonlinear.lFhi"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhbnd"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhbnd"])) < EPS_REF
    assert np.max(np.abs(r["lFhbnd"] - g["testSpaceTimePredictorNonlinear.lFhbnd"])) < EPS_REF


# ---------------------------------------------------------------------------------------------
# Non-trivial Picard iteration: reference outputs on seeded non-constant cells
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("dim", [2, 3])
def test_picard_nontrivial_vs_reference_fixture(dim):
    fx = np.load(os.path.join(GOLD, "picard_euler%dd_o3.npz" % dim))
    o = Oracle(dim, 3)
    for c in range(int(fx["ncase"][0])):
        k = lambda s: fx["case%d.%s" % (c, s)]
        r = o.predictor(k("luh"), k("dx"), float(k("dt")[0]), centre=[0.3, 0.6, 0.2])
        assert r["ret"] == int(k("iters")[0])
        for key in ("lQi", "lQhi", "lFhi", "lQhbnd", "lFhbnd"):
            assert relerr(r[key], k(key)) < 1e-12, (c, key, relerr(r[key], k(key)))
        lduh = o.volume(r["lFhi"], k("dx"))
        assert relerr(lduh, k("lduh")) < 1e-12


# ---------------------------------------------------------------------------------------------
# Differential against the compiled reference kernels (only where oracle/_ref was built)
# ---------------------------------------------------------------------------------------------

def _ref_or_skip(dim, order, npar=0):
    try:
        return RefKernels(dim, order, npar=npar)
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)


def euler_cells(rng, ncells, nd, amp=0.1, dim=3):
    rho = 1.0 + amp * rng.uniform(-1, 1, (ncells, nd))
    u = 0.3 * rng.uniform(-1, 1, (ncells, nd, 3))
    if dim == 2:
        u[..., 2] = 0
    p = 1.0 + amp * rng.uniform(-1, 1, (ncells, nd))
    Q = np.zeros((ncells, nd, 5))
    Q[..., 0] = rho
    Q[..., 1:4] = rho[..., None] * u
    Q[..., 4] = p / 0.4 + 0.5 * rho * (u ** 2).sum(-1)
    return Q


@pytest.mark.parametrize("dim,order", [(3, 3), (3, 5), (2, 3), (2, 5)])
def test_differential_kernels_vs_ref(dim, order):
    ref = _ref_or_skip(dim, order)
    o = Oracle(dim, order)
    rng = np.random.default_rng(11 + order)
    n = order + 1
    nd, nf = n ** dim, n ** (dim - 1)
    dx = np.array([0.031, 0.027, 0.022])
    for trial in range(3):
        luh = euler_cells(rng, 1, nd, amp=0.05 * (trial + 1), dim=dim).reshape(-1)
        dt_r, dt_o = ref.dt(luh, dx), o.dt(luh, dx)
        assert abs(dt_r - dt_o) <= 1e-15 * dt_r
        a = ref.predictor(luh, dx, dt_r, centre=[0.1, 0.2, 0.3])
        b = o.predictor(luh, dx, dt_r, centre=[0.1, 0.2, 0.3])
        assert a["ret"] == b["ret"]
        for key in ("lQi", "lQhi", "lFhi", "lQhbnd", "lFhbnd"):
            assert relerr(b[key], a[key]) < 1e-13, key
        assert relerr(o.volume(b["lFhi"], dx), ref.volume(a["lFhi"], dx)) < 1e-13
        # Riemann on random faces in every direction
        for d in range(dim):
            QL = euler_cells(rng, 1, nf, dim=dim).reshape(-1)
            QR = euler_cells(rng, 1, nf, dim=dim).reshape(-1)
            FL = rng.normal(size=nf * 5)
            FR = rng.normal(size=nf * 5)
            ra = ref.riemann(FL, FR, QL, QR, dx, d)
            rb = o.riemann(FL, FR, QL, QR, dx, d)
            assert relerr(rb[0], ra[0]) < 1e-14 and relerr(rb[1], ra[1]) < 1e-14
        lduh = rng.normal(size=nd * 5)
        lF = rng.normal(size=2 * dim * nf * 5)
        assert relerr(o.surface(lduh, lF, dx), ref.surface(lduh, lF, dx)) < 1e-14
        for d in range(dim):
            for ori in (0, 1):
                face = lF[(2 * d + ori) * nf * 5:(2 * d + ori + 1) * nf * 5]
                assert relerr(o.face(lduh, face, d, ori, dx), ref.face(lduh, face, d, ori, dx)) < 1e-14
        assert relerr(o.update(luh, lduh, 1e-3), ref.update(luh, lduh, 1e-3)) < 1e-15


@pytest.mark.parametrize("dim,order,ncell,walls", [(3, 3, (3, 4, 2), False), (2, 3, (5, 4), False),
                                                    (2, 3, (4, 3), True), (3, 3, (2, 3, 2), True)])
def test_differential_patch_run_vs_ref(dim, order, ncell, walls):
    ref = _ref_or_skip(dim, order)
    o = Oracle(dim, order)
    rng = np.random.default_rng(5)
    nd = (order + 1) ** dim
    nc = int(np.prod(ncell))
    luh0 = euler_cells(rng, nc, nd, amp=0.03, dim=dim).reshape(-1)
    la, lb = luh0.copy(), luh0.copy()
    size = [1.0, 0.8, 0.9][:dim]
    ta, dta, _ = ref.run(la, ncell, size, 3, walls=walls)
    tb, dtb, _ = o.run(lb, ncell, size, 3, walls=walls)
    assert np.max(np.abs(dta - dtb) / dta) < 1e-13
    assert relerr(lb, la) < 1e-12


# ---------------------------------------------------------------------------------------------
# Linear waves with per-node material parameters, a point source (algebraicSource) and outflow
# boundaries: the restatement against the reference's kernels instantiated with useSource.
# ---------------------------------------------------------------------------------------------

LINEAR = [("acoustic", 4, 2, 0), ("elastic", 3, 3, 3)]  # name, order, npar, source variable


def _linear(name, order, npar, var, size):
    from exa_scenarios import ricker_source
    from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC
    src = ricker_source(3, size, f0=4.0, variable=var, width=0.1)
    src = src[:4] + (0.05,) + src[5:]  # source active from the first step
    try:
        ref = RefKernels(3, order, name, npar, source=src)
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)
    o = Oracle(3, order, {"acoustic": PDE_ACOUSTIC, "elastic": PDE_ELASTIC}[name], source=src)
    return o, ref, src


@pytest.mark.parametrize("name,order,npar,var", LINEAR)
def test_linear_source_predictor_vs_ref(name, order, npar, var):
    """One cell next to the source (source on) and one far from it (off), several times."""
    from exa_scenarios import layered_medium
    size = [1.0, 0.8, 1.2]
    o, ref, src = _linear(name, order, npar, var, size)
    luh_all = layered_medium(name, (5, 4, 6), size, order, seed=3)
    D = o.D
    nd = (order + 1) ** 3
    dx = np.array([0.2, 0.2, 0.2])
    # a seeded non-trivial state in the cell so that the flux part is exercised too
    rng = np.random.default_rng(4)
    luh = luh_all[:nd * D].copy().reshape(nd, D)
    luh[:, :o.v] = rng.normal(scale=0.1, size=(nd, o.v))
    luh = luh.reshape(-1)
    for centre in ([src[0] + 0.05, src[1] - 0.1, src[2]], [0.05, 0.05, 0.05]):
        for t in (0.0, 0.031, 0.2):
            dt = 0.5 * ref.dt(luh, dx)
            a = ref.predictor(luh, dx, dt, centre=centre, t=t)
            b = o.predictor(luh, dx, dt, centre=centre, t=t)
            assert a["ret"] == b["ret"]
            for key in ("lQhi", "lFhi", "lQhbnd", "lFhbnd"):
                assert relerr(b[key], a[key]) < 1e-13, key
            assert relerr(o.volume(b["lFhi"], dx), ref.volume(a["lFhi"], dx)) < 1e-13


@pytest.mark.parametrize("name,order,npar,var", LINEAR)
@pytest.mark.parametrize("walls", [0, 1, 3])
def test_linear_source_patch_run_vs_ref(name, order, npar, var, walls):
    """Periodic, reflective and outflow domains over a two-layer medium with the point source."""
    from exa_scenarios import layered_medium
    size = [1.0, 0.8, 1.2]
    o, ref, _ = _linear(name, order, npar, var, size)
    ncell = (5, 4, 6)
    luh0 = layered_medium(name, ncell, size, order, seed=2)
    la, lb = luh0.copy(), luh0.copy()
    ta, dta, pa = ref.run(la, ncell, size, 3, walls=walls, want_picard=True)
    tb, dtb, pb = o.run(lb, ncell, size, 3, walls=walls, want_picard=True)
    assert np.max(np.abs(dta - dtb) / dta) < 1e-13
    assert np.array_equal(pa + 1, pb)  # break index vs sweep count
    assert relerr(lb, la) < 1e-12
    assert np.abs(lb - luh0).max() > 1e-3  # the waves and the source did act


@pytest.mark.parametrize("name,order,npar,var", LINEAR)
def test_linear_fixed_picard_count_vs_ref(name, order, npar, var):
    """The reference's UseMaxPicardIterations mode (Order+1 sweeps, no residual test)."""
    from exa_scenarios import layered_medium, ricker_source
    from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC
    size = [1.0, 0.8, 1.2]
    src = ricker_source(3, size, f0=4.0, variable=var, width=0.1)
    src = src[:4] + (0.05,) + src[5:]
    try:
        ref = RefKernels(3, order, name + "fixed", npar, source=src)
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)
    o = Oracle(3, order, {"acoustic": PDE_ACOUSTIC, "elastic": PDE_ELASTIC}[name], source=src,
               max_picard=order + 1)
    ncell = (4, 3, 5)
    luh0 = layered_medium(name, ncell, size, order, seed=4)
    la, lb = luh0.copy(), luh0.copy()
    dt = 0.5 * ref.dt(luh0[:(order + 1) ** 3 * o.D], np.array(size) / np.array(ncell))
    ref.run(la, ncell, size, 3, walls=3, fixed_dt=dt)
    o.run(lb, ncell, size, 3, walls=3, fixed_dt=dt)
    assert relerr(lb, la) < 1e-12
    # single cell: every output of the predictor
    dx = np.array([0.2, 0.2, 0.2])
    luh = luh0[:(order + 1) ** 3 * o.D].copy()
    a = ref.predictor(luh, dx, dt, centre=[src[0], src[1], src[2]], t=0.01)
    b = o.predictor(luh, dx, dt, centre=[src[0], src[1], src[2]], t=0.01)
    for key in ("lQhi", "lFhi", "lQhbnd", "lFhbnd"):
        assert relerr(b[key], a[key]) < 1e-13, key


def test_elastic_order7_source_outflow_vs_ref():
    """The order-7 elastic configuration (8^3 nodes, 9 variables + 3 parameters)."""
    from exa_scenarios import layered_medium, ricker_source
    from pyoracle import PDE_ELASTIC
    size = [1.0, 1.0, 1.0]
    src = ricker_source(3, size, f0=4.0, variable=3, width=0.15)
    src = src[:4] + (0.05,) + src[5:]
    try:
        ref = RefKernels(3, 7, "elastic", 3, source=src)
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)
    o = Oracle(3, 7, PDE_ELASTIC, source=src)
    ncell = (2, 2, 3)
    luh0 = layered_medium("elastic", ncell, size, 7, seed=1)
    la, lb = luh0.copy(), luh0.copy()
    ta, dta, pa = ref.run(la, ncell, size, 2, walls=3, want_picard=True)
    tb, dtb, pb = o.run(lb, ncell, size, 2, walls=3, want_picard=True)
    assert np.max(np.abs(dta - dtb) / dta) < 1e-13
    assert np.array_equal(pa + 1, pb)
    assert relerr(lb, la) < 1e-12
    assert np.abs(lb - luh0).max() > 1e-4


# ---------------------------------------------------------------------------------------------
# Shallow water with bathymetry (NCP path): the restatement against the reference's kernels
# instantiated for the SWE app's solver (SWE_ADERDG/MySWESolver.cpp:43-62, 103-152). This pins
# the gradient of the old iterate (dudx, 2d/spaceTimePredictorNonlinear.cpph:95-140), the
# fusedSource sign S = -NCP (fusedMethods.cpph:65-80) and the Rusanov NCP split
# (2d/riemannSolverNonlinear.cpph:37-133).
# ---------------------------------------------------------------------------------------------

def _swe_ref_or_skip(order):
    try:
        return RefKernels(2, order, "swe")
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)


def swe_cells(rng, ncells, nd, vel=0.2):
    """h = 1 + bumps, velocities U[-vel, vel], smooth-ish random bathymetry (h, hu, hv, b)."""
    Q = np.zeros((ncells, nd, 4))
    Q[..., 0] = 1.0 + 0.3 * rng.uniform(0, 1, (ncells, nd))
    Q[..., 1] = Q[..., 0] * rng.uniform(-vel, vel, (ncells, nd))
    Q[..., 2] = Q[..., 0] * rng.uniform(-vel, vel, (ncells, nd))
    Q[..., 3] = 0.1 * rng.uniform(0, 1, (ncells, nd))
    return Q


@pytest.mark.parametrize("order", [2, 4])
def test_swe_predictor_vs_ref(order):
    from pyoracle import PDE_SWE
    ref = _swe_ref_or_skip(order)
    o = Oracle(2, order, PDE_SWE)
    rng = np.random.default_rng(40 + order)
    nd = (order + 1) ** 2
    dx = np.array([0.05, 0.04])
    for trial in range(4):
        luh = swe_cells(rng, 1, nd, vel=0.05 * (trial + 1)).reshape(-1)
        dt_r, dt_o = ref.dt(luh, dx), o.dt(luh, dx)
        assert abs(dt_r - dt_o) <= 1e-15 * dt_r
        a = ref.predictor(luh, dx, dt_r, centre=[0.4, 0.6])
        b = o.predictor(luh, dx, dt_r, centre=[0.4, 0.6])
        assert a["ret"] == b["ret"]
        for key in ("lQi", "lFi", "lQhi", "lFhi", "lQhbnd", "lFhbnd"):
            assert relerr(b[key], a[key]) < 1e-13, (key, relerr(b[key], a[key]))
        # the source slot of lFhi is the time-averaged -NCP: non-zero for a non-flat bottom
        assert np.abs(a["lFhi"][2 * nd * 4:]).max() > 1e-6
        assert relerr(o.volume(b["lFhi"], dx), ref.volume(a["lFhi"], dx)) < 1e-13


@pytest.mark.parametrize("order", [2, 4])
def test_swe_riemann_ncp_split_vs_ref(order):
    from pyoracle import PDE_SWE
    ref = _swe_ref_or_skip(order)
    o = Oracle(2, order, PDE_SWE)
    rng = np.random.default_rng(7 + order)
    nf = order + 1
    dx = np.array([0.05, 0.04])
    for d in range(2):
        for _ in range(3):
            QL = swe_cells(rng, 1, nf).reshape(-1)
            QR = swe_cells(rng, 1, nf).reshape(-1)
            FL = rng.normal(size=nf * 4)
            FR = rng.normal(size=nf * 4)
            ra = ref.riemann(FL, FR, QL, QR, dx, d)
            rb = o.riemann(FL, FR, QL, QR, dx, d)
            assert relerr(rb[0], ra[0]) < 1e-14 and relerr(rb[1], ra[1]) < 1e-14
            # the NCP makes the two sides differ (FL = F + ncp/2, FR = F - ncp/2)
            assert np.abs(ra[0] - ra[1]).max() > 1e-8


@pytest.mark.parametrize("order,ncell", [(4, (5, 4)), (2, (6, 5))])
def test_swe_wall_patch_run_vs_ref(order, ncell):
    """Four steps of a wall-bounded grid with bumps and bathymetry (the batched-SWE state)."""
    from exa_scenarios import swe_bumps_state
    from pyoracle import PDE_SWE
    ref = _swe_ref_or_skip(order)
    o = Oracle(2, order, PDE_SWE)
    luh0 = swe_bumps_state(ncell, order, np.random.default_rng(3))
    la, lb = luh0.copy(), luh0.copy()
    ta, dta, pa = ref.run(la, ncell, [1.0, 1.0], 4, walls=True, want_picard=True)
    tb, dtb, pb = o.run(lb, ncell, [1.0, 1.0], 4, walls=True, want_picard=True)
    assert np.max(np.abs(dta - dtb) / dta) < 1e-13
    # the 2D reference returns MaxIterations+2 when a cell converged (2d/...:303-305), else the cap
    n = order + 1
    assert np.all((pa == 2 * n + 2) | ((pa == 2 * n) & (pb == 2 * n)))
    assert pb.min() >= 2 and pb.max() <= 2 * n
    assert relerr(lb, la) < 1e-12
    assert np.abs(lb - luh0).max() > 1e-3  # the bumps moved


# ---------------------------------------------------------------------------------------------
# The reference's generated optimised kernels (KernelGenerator, plain-loop mode; oracle/_ref/
# libkg_euler_o{3,5}.so): the second CPU baseline, cross-checked against the generic kernels.
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("order,walls", [(3, 0), (3, 3), (5, 0), (5, 3)])
def test_kernelgenerator_kernels_vs_generic_reference(order, walls):
    import exa_scenarios as sc
    from pyoracle import KGKernels
    try:
        kg = KGKernels(order)
        ref = RefKernels(3, order)
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)
    ncell = (4, 3, 5)
    luh, _ = sc.euler_entropy_wave(ncell, order)
    a, b = luh.copy(), luh.copy()
    size = [n / 5.0 for n in ncell]  # cubic cells, as the generated kernels assume
    _, dta, pa = ref.run(a, ncell, size, 3, walls=walls, want_picard=True)
    _, dtb, pb = kg.run(b, ncell, size, 3, walls=walls, want_picard=True)
    assert np.max(np.abs(dta - dtb) / dta) < 1e-13
    assert np.array_equal(pa + 1, pb)  # generic: break index; generated: sweeps
    assert relerr(b, a) < 1e-13
