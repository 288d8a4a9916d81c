"""GPU parity: the sm_100a kernels through the C ABI against the CPU oracle and the reference's
golden arrays. FP64 form: 1e-12 relative (max |gpu - oracle| / max |oracle|) unless stated.
"""
import os

import numpy as np
import pytest

from conftest import REPO
from pyoracle import Oracle, PDE_SWE

GOLD = os.path.join(REPO, "tests", "golden")
TOL = 1e-12
EPS_REF = 1e-10

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


def with_params(arr, nvar, npar):
    a = np.asarray(arr).reshape(-1, nvar)
    out = np.zeros((a.shape[0], nvar + npar))
    out[:, :nvar] = a
    return out.reshape(-1)


def strip_params(arr, nvar, npar):
    return np.asarray(arr).reshape(-1, nvar + npar)[:, :nvar].reshape(-1)


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.fixture(scope="module")
def exa():
    import exa_aderdg
    return exa_aderdg


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


# ------------------------------------------------------------------------------------------
# known-answer arrays of the reference (GenericEulerKernelTest{2D,3D}.cpp)
# ------------------------------------------------------------------------------------------

def test_golden3d_predictor_riemann_update(exa):
    g = np.load(os.path.join(GOLD, "generic_euler_3d.npz"))
    s = exa.Solver(exa.PDE_EULER, 3, 3, npar=1)
    luh = with_params(g["testSpaceTimePredictorNonlinear.luh"], 5, 1)
    r = s.space_time_predictor(luh, 0.05, 1.083937460199773e-3)
    assert r["ret"] == 0
    assert np.max(np.abs(strip_params(r["lQi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQi"])) < EPS_REF
    lFi = r["lFi"].reshape(4, 64, 4, 5)[:, :, :3, :].reshape(-1)
    assert np.max(np.abs(lFi - g["testSpaceTimePredictorNonlinear.lFi"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhbnd"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhbnd"])) < EPS_REF
    assert np.max(np.abs(r["lFhbnd"] - g["testSpaceTimePredictorNonlinear.lFhbnd"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhi"])) < EPS_REF
    assert np.max(np.abs(r["lFhi"][:960] - g["testSpaceTimePredictorNonlinear.lFhi"])) < EPS_REF
    # Rusanov, direction 1
    FL, FR = s.riemann_cell(np.arange(1, 81, dtype=float), np.arange(-1, 79, dtype=float),
                            with_params(g["testRiemannSolver.QL"], 5, 1), with_params(g["testRiemannSolver.QR"], 5, 1),
                            0.5, 1)
    assert np.max(np.abs(FL - g["testRiemannSolverNonlinear.FL"])) < EPS_REF
    assert np.max(np.abs(FR - g["testRiemannSolverNonlinear.FR"])) < EPS_REF
    # solution update
    luh = np.zeros(6 * 64)
    luh[0::6] = 1.0
    luh[4::6] = 2.5
    out = s.solution_update_cell(luh, np.arange(320, dtype=float), 1.40831757919882352703e-03)
    assert np.max(np.abs(strip_params(out, 5, 1) - g["testSolutionUpdate.luh"])) < EPS_REF
    assert s.status() == 0


def test_cell_integrals_vs_golden_and_reference(exa):
    """The per-cell volume, surface and face integrals (the generic signatures on host pointers):
    the reference's surface-integral known answers (GenericEulerKernelTest3D.cpp:277-319), and the
    compiled reference kernels on random blocks, 3D N=3 and 5 and 2D N=3."""
    g = np.load(os.path.join(GOLD, "generic_euler_3d.npz"))
    s = exa.Solver(exa.PDE_EULER, 3, 3, npar=1)
    lF = np.zeros(480)
    for i in range(0, 80, 5):
        lF[0 + i + 1] = lF[80 + i + 1] = 1.0
        lF[160 + i + 2] = lF[240 + i + 2] = 1.0
        lF[320 + i + 3] = lF[400 + i + 3] = 1.0
    out = s.surface_integral_cell(np.arange(320) / 10.0, lF, 0.1)
    assert np.max(np.abs(out - g["testSurfaceIntegralNonlinear.lduh"])) < EPS_REF
    from pyoracle import RefKernels
    rng = np.random.default_rng(31)
    for dim, order in ((3, 3), (3, 5), (2, 3)):
        try:
            ref = RefKernels(dim, order)
        except (FileNotFoundError, AttributeError, OSError) as e:
            pytest.skip("reference kernels not built: %s" % e)
        s = exa.Solver(exa.PDE_EULER, dim, order)
        n = order + 1
        nd, nf = n ** dim, n ** (dim - 1)
        dx = np.array([0.031, 0.027, 0.022])[:dim]
        lFhi = rng.normal(size=(dim + 1) * nd * 5)
        assert rel(s.volume_integral_cell(lFhi, dx), ref.volume(lFhi, dx)) < 1e-14
        lduh = rng.normal(size=nd * 5)
        lFhbnd = rng.normal(size=2 * dim * nf * 5)
        assert rel(s.surface_integral_cell(lduh, lFhbnd, dx), ref.surface(lduh, lFhbnd, dx)) < 1e-14
        for d in range(dim):
            for ori in (0, 1):
                face = lFhbnd[(2 * d + ori) * nf * 5:(2 * d + ori + 1) * nf * 5]
                assert rel(s.face_integral_cell(lduh, face, d, ori, dx), ref.face(lduh, face, d, ori, dx)) < 1e-14


def test_golden2d_predictor_riemann_update(exa):
    g = np.load(os.path.join(GOLD, "generic_euler_2d.npz"))
    s = exa.Solver(exa.PDE_EULER, 2, 3, npar=1)
    luh = with_params(g["testSpaceTimePredictorNonlinear.luh"], 5, 1)
    r = s.space_time_predictor(luh, 0.05, 1.686854344081342e-3)
    assert r["ret"] == 2 * 4 + 2
    assert np.max(np.abs(strip_params(r["lQi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQi"])) < EPS_REF
    lFi = r["lFi"].reshape(4, 16, 3, 5)[:, :, :2, :].reshape(-1)
    assert np.max(np.abs(lFi - g["testSpaceTimePredictorNonlinear.lFi"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhi"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhi"])) < EPS_REF
    assert np.max(np.abs(r["lFhi"][:160] - g["testSpaceTimePredictorNonlinear.lFhi"])) < EPS_REF
    assert np.max(np.abs(strip_params(r["lQhbnd"], 5, 1) - g["testSpaceTimePredictorNonlinear.lQhbnd"])) < EPS_REF
    assert np.max(np.abs(r["lFhbnd"] - g["testSpaceTimePredictorNonlinear.lFhbnd"])) < EPS_REF
    for case, d in ((1, 0), (2, 1)):
        FL, FR = s.riemann_cell(g["testRiemannSolverNonlinear.FL_%d_in" % case],
                                g["testRiemannSolverNonlinear.FR_%d_in" % case],
                                with_params(g["testRiemannSolverNonlinear.QL_%d_in" % case], 5, 1),
                                with_params(g["testRiemannSolverNonlinear.QR_%d_in" % case], 5, 1), 0.5, d)
        ref = g["testRiemannSolverNonlinear.F_%d_out" % case]
        assert np.max(np.abs(FL - ref)) < EPS_REF and np.max(np.abs(FR - ref)) < EPS_REF
    luh = np.zeros(6 * 16)
    luh[0::6] = 1.0
    luh[4::6] = 2.5
    out = s.solution_update_cell(luh, g["testSolutionUpdate.lduh"], 1.40831757919882352703e-03)
    assert np.max(np.abs(strip_params(out, 5, 1) - g["testSolutionUpdate.luh"])) < EPS_REF


@pytest.mark.parametrize("dim", [2, 3])
def test_picard_nontrivial_vs_reference_fixture(exa, dim):
    """Reference outputs on non-constant cells (the Picard loop really iterates here)."""
    fx = np.load(os.path.join(GOLD, "picard_euler%dd_o3.npz" % dim))
    s = exa.Solver(exa.PDE_EULER, dim, 3)
    for c in range(int(fx["ncase"][0])):
        k = lambda name: fx["case%d.%s" % (c, name)]
        r = s.space_time_predictor(k("luh"), k("dx")[:dim], float(k("dt")[0]))
        assert r["ret"] == int(k("iters")[0])
        for key in ("lQi", "lQhi", "lFhi", "lQhbnd", "lFhbnd"):
            assert rel(r[key], k(key)) < TOL, (c, key, rel(r[key], k(key)))


# ------------------------------------------------------------------------------------------
# batched kernels vs the oracle
# ------------------------------------------------------------------------------------------

@pytest.mark.parametrize("dim,order", [(3, 5), (3, 3), (2, 3)])
def test_batched_predictor_volume_vs_oracle(exa, torch, dim, order):
    rng = np.random.default_rng(100 + order)
    n = order + 1
    nd, nf = n ** dim, n ** (dim - 1)
    ncells = 37
    luh = euler_cells(rng, ncells, nd, amp=0.05, dim=dim).reshape(-1)
    dx = np.array([0.02, 0.025, 0.03])[:dim]
    o = Oracle(dim, order)
    dt = min(o.dt(luh.reshape(ncells, -1)[c], dx) for c in range(ncells))
    s = exa.Solver(exa.PDE_EULER, dim, order)
    dev = torch.device("cuda")
    t_luh = torch.from_numpy(luh).to(dev)
    lduh = torch.zeros(ncells * nd * 5, dtype=torch.float64, device=dev)
    qhb = torch.zeros(ncells * 2 * dim * nf * 5, dtype=torch.float64, device=dev)
    fhb = torch.zeros_like(qhb)
    pic = torch.zeros(ncells, dtype=torch.int32, device=dev)
    s.fused_predictor_volume_integral(t_luh, lduh, qhb, fhb, dx, dt, picard=pic)
    torch.cuda.synchronize()
    lduh, qhb, fhb, pic = lduh.cpu().numpy(), qhb.cpu().numpy(), fhb.cpu().numpy(), pic.cpu().numpy()
    for c in range(ncells):
        r = o.predictor(luh.reshape(ncells, -1)[c], dx, dt)
        assert pic[c] == r["sweeps"]
        assert rel(qhb.reshape(ncells, -1)[c], r["lQhbnd"]) < TOL
        assert rel(fhb.reshape(ncells, -1)[c], r["lFhbnd"]) < TOL
        assert rel(lduh.reshape(ncells, -1)[c], o.volume(r["lFhi"], dx)) < TOL
    assert s.status() == 0


@pytest.mark.parametrize("dim,order", [(3, 5), (2, 3)])
def test_batched_riemann_surface_update_cfl_vs_oracle(exa, torch, dim, order):
    rng = np.random.default_rng(7)
    n = order + 1
    nd, nf = n ** dim, n ** (dim - 1)
    ncells = 12
    o = Oracle(dim, order)
    s = exa.Solver(exa.PDE_EULER, dim, order)
    dev = torch.device("cuda")
    qhb = np.concatenate([euler_cells(rng, 2 * dim, nf, dim=dim).reshape(-1) for _ in range(ncells)])
    fhb = rng.normal(size=ncells * 2 * dim * nf * 5)
    left = np.array([0, 3, 5, 7, 11, 2], dtype=np.int32)
    right = np.array([1, 4, 6, 8, 10, 9], dtype=np.int32)
    dirs = np.array([0, 1, dim - 1, 0, 1, dim - 1], dtype=np.int8)
    t_q = torch.from_numpy(qhb).to(dev)
    t_f = torch.from_numpy(fhb.copy()).to(dev)
    s.riemann(torch.from_numpy(left).to(dev), torch.from_numpy(right).to(dev), torch.from_numpy(dirs).to(dev), t_q, t_f)
    got = t_f.cpu().numpy().reshape(ncells, 2 * dim, nf * 5)
    exp = fhb.copy().reshape(ncells, 2 * dim, nf * 5)
    qq = qhb.reshape(ncells, 2 * dim, nf * 5)
    for L, R, d in zip(left, right, dirs):
        FL, FR = o.riemann(exp[L, 2 * d + 1], exp[R, 2 * d], qq[L, 2 * d + 1], qq[R, 2 * d], 1.0, d)
        exp[L, 2 * d + 1], exp[R, 2 * d] = FL, FR
    assert rel(got, exp) < TOL
    # surface integral + update, then CFL of the updated state
    luh = euler_cells(rng, ncells, nd, dim=dim).reshape(-1)
    lduh = rng.normal(size=ncells * nd * 5) * 0.01
    dx = np.array([0.1, 0.07, 0.05])[:dim]
    t_luh = torch.from_numpy(luh.copy()).to(dev)
    s.surface_integral_and_update(t_luh, torch.from_numpy(lduh).to(dev), torch.from_numpy(fhb * 0.01).to(dev), dx, 1e-3)
    new = t_luh.cpu().numpy().reshape(ncells, -1)
    for c in range(ncells):
        du = o.surface(lduh.reshape(ncells, -1)[c], (fhb * 0.01).reshape(ncells, -1)[c], dx)
        ref = o.update(luh.reshape(ncells, -1)[c], du, 1e-3)
        assert rel(new[c], ref) < TOL
    cell_dt = torch.zeros(ncells, dtype=torch.float64, device=dev)
    dtmin = s.stable_time_step_size(t_luh, dx, cell_dt=cell_dt)
    ref_dt = np.array([o.dt(new[c], dx) for c in range(ncells)])
    assert rel(cell_dt.cpu().numpy(), ref_dt) < 1e-15
    assert dtmin == ref_dt.min()


def test_per_cell_shims_from_many_host_threads(exa):
    """The per-cell shims on one solver from eight host threads at once, as the reference's TBB jobs
    call its kernels on different cells (ADERDGSolver.cpp:726-729, 769-773): every result equals the
    one-thread result bit for bit and the oracle's at 1e-12 (the per-cell CFL step at 1e-15). The
    shims serialise on the solver's lock; exa_stableTimeStepSize keeps it over its copies, so no
    other thread can move the shared scratch between its upload and its kernel."""
    import concurrent.futures
    rng = np.random.default_rng(11)
    dim, order, ncells = 3, 3, 48
    nd = (order + 1) ** dim
    o = Oracle(dim, order)
    s = exa.Solver(exa.PDE_EULER, dim, order)
    cells = euler_cells(rng, ncells, nd).reshape(ncells, -1)
    lduh = rng.normal(size=(ncells, nd * 5)) * 0.01
    dx = np.array([0.1, 0.07, 0.05])

    def work(c):
        r = s.space_time_predictor(cells[c], dx, 1e-3)
        return (r["lQhbnd"], r["lFhbnd"], s.volume_integral_cell(r["lFhi"], dx),
                s.solution_update_cell(cells[c], lduh[c], 1e-3), s.stable_time_step_size_cell(cells[c], dx))

    with concurrent.futures.ThreadPoolExecutor(8) as ex:
        got = list(ex.map(work, range(ncells)))
    for c in range(ncells):
        for a, b in zip(got[c], work(c)):
            assert np.array_equal(a, b), c
        r = o.predictor(cells[c], dx, 1e-3)
        assert rel(got[c][0], r["lQhbnd"]) < TOL and rel(got[c][1], r["lFhbnd"]) < TOL
        assert rel(got[c][2], o.volume(r["lFhi"], dx)) < TOL
        assert rel(got[c][3], o.update(cells[c], lduh[c], 1e-3)) < TOL
        assert abs(got[c][4] - o.dt(cells[c], dx)) <= 1e-15 * o.dt(cells[c], dx)
    assert s.status() == 0


# ------------------------------------------------------------------------------------------
# whole steps on device-resident patches vs the oracle's patch driver
# ------------------------------------------------------------------------------------------

@pytest.mark.parametrize("dim,order,ncell,steps,walls", [
    (2, 3, (27, 27), 20, False),      # 2D Euler entropy wave, the parity workload
    (3, 3, (5, 4, 3), 4, False),
    (3, 5, (4, 3, 3), 3, False),
    (2, 3, (6, 5), 5, True),
    (3, 3, (3, 3, 4), 3, True),
])
def test_patch_steps_vs_oracle(exa, dim, order, ncell, steps, walls):
    import exa_scenarios as sc
    if ncell == (27, 27):
        luh0, _ = sc.euler_entropy_wave(ncell, order, seed=0)
        size = [1.0, 1.0]
    else:
        rng = np.random.default_rng(3)
        luh0 = euler_cells(rng, int(np.prod(ncell)), (order + 1) ** dim, amp=0.03, dim=dim).reshape(-1)
        size = [1.0, 0.9, 0.8][:dim]
    o = Oracle(dim, order)
    ref = luh0.copy()
    t_ref, dts, _ = o.run(ref, ncell, size, steps, walls=walls)
    s = exa.Solver(exa.PDE_EULER, dim, order)
    bc = exa.BC_WALL if walls else exa.BC_PERIODIC
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    p.set_solution(luh0)
    p.step(steps)
    got = p.get_solution()
    t, dt = p.time()
    assert abs(t[0] - t_ref) <= 1e-13 * t_ref
    assert rel(got, ref) < TOL
    assert p.status() == 0


@pytest.mark.parametrize("dim,ncell,walls", [
    (3, (1, 1, 1), False), (3, (1, 2, 3), False), (3, (3, 1, 2), False), (3, (1, 1, 4), True),
    (3, (2, 1, 1), True), (2, (1, 1), False), (2, (7, 1), False), (2, (1, 5), True), (2, (1, 1), True)])
def test_degenerate_grids_vs_oracle(exa, dim, ncell, walls):
    """Grids one cell thick along some axes: a periodic axis of one cell makes the cell its own
    neighbour (the face joins its high and its low face), a wall-bounded one gives the cell two
    domain faces on that axis. Three steps against the oracle at 1e-12 with equal time steps and
    the last step's Picard-sweep histogram."""
    order = 3
    rng = np.random.default_rng(17)
    nc, nd = int(np.prod(ncell)), (order + 1) ** dim
    luh0 = euler_cells(rng, nc, nd, amp=0.05, dim=dim).reshape(-1)
    size = [0.5, 0.6, 0.7][:dim]
    o = Oracle(dim, order)
    ref = luh0.copy()
    t_ref, _, pic = o.run(ref, ncell, size, 3, walls=walls, want_picard=True)
    s = exa.Solver(exa.PDE_EULER, dim, order)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=exa.BC_WALL if walls else exa.BC_PERIODIC)])
    p.set_solution(luh0)
    p.step(3)
    got = p.get_solution()
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    assert rel(got, ref) < TOL
    assert list(np.bincount(pic[-1], minlength=32)[:32]) == p.stats()["picard_hist"]
    assert p.status() == 0
    p.close()


def test_patch_swe_walls_vs_oracle(exa):
    """2D shallow water with bathymetry (NCP) and reflective walls."""
    rng = np.random.default_rng(9)
    order, ncell = 4, (7, 6)
    n = order + 1
    nc = ncell[0] * ncell[1]
    Q = np.zeros((nc, n * n, 4))
    Q[..., 0] = 1.0 + 0.2 * rng.uniform(0, 1, (nc, n * n))
    Q[..., 1] = 0.05 * rng.normal(size=(nc, n * n))
    Q[..., 2] = 0.05 * rng.normal(size=(nc, n * n))
    Q[..., 3] = 0.1 * rng.uniform(0, 1, (nc, n * n))
    luh0 = Q.reshape(-1)
    o = Oracle(2, order, pde=PDE_SWE)
    ref = luh0.copy()
    t_ref, _, _ = o.run(ref, ncell, [1.0, 1.0], 4, walls=True)
    s = exa.Solver(exa.PDE_SWE, 2, order)
    p = exa.Patch(s, [dict(ncell=ncell, size=[1.0, 1.0], bc=exa.BC_WALL)])
    p.set_solution(luh0)
    p.step(4)
    assert rel(p.get_solution(), ref) < TOL
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref


def test_patch_many_grids_independent(exa):
    """Several grids of different sizes in one patch advance exactly like separate patches."""
    import exa_scenarios as sc
    s = exa.Solver(exa.PDE_EULER, 2, 3)
    specs = [dict(ncell=(9, 7), size=[1.0, 0.8]), dict(ncell=(5, 5), size=[0.5, 0.5], bc=exa.BC_WALL),
             dict(ncell=(12, 4), size=[2.0, 1.0])]
    rng = np.random.default_rng(2)
    inits = [euler_cells(rng, int(np.prod(sp["ncell"])), 16, amp=0.04, dim=2).reshape(-1) for sp in specs]
    multi = exa.Patch(s, specs)
    multi.set_solution(np.concatenate(inits))
    multi.step(3)
    got = multi.get_solution()
    t_multi, _ = multi.time()
    off = 0
    for g, (sp, init) in enumerate(zip(specs, inits)):
        single = exa.Patch(s, [sp])
        single.set_solution(init)
        single.step(3)
        ref = single.get_solution()
        assert np.array_equal(got[off:off + ref.size], ref)
        assert t_multi[g] == single.time()[0][0]
        off += ref.size


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("dim,order,ncell,steps", [(3, 5, (4, 3, 3), 3), (2, 3, (27, 27), 10)])
def test_mixed_precision_patch_vs_fp64_oracle(exa, dim, order, ncell, steps, variant):
    """Mixed mode: the sweeps after sweep 0 as FP32 corrections to sweep 0's FP64 closed form
    (FP32 flux corrections F(luh + dq) - F(luh), contractions and time solve), with the iterate
    update, the residual test, the time averages, the faces, the volume integral, the update and the
    CFL in FP64. The state stays within 1e-9 (relative) of the FP64 oracle and the Picard counts
    are unchanged; both launch forms (2 and 3 CTAs per SM) agree."""
    import exa_scenarios as sc
    if dim == 2:
        luh0, _ = sc.euler_entropy_wave(ncell, order, seed=0)
    else:
        rng = np.random.default_rng(3)
        luh0 = euler_cells(rng, int(np.prod(ncell)), (order + 1) ** dim, amp=0.03, dim=dim).reshape(-1)
    size = [1.0] * dim
    ref = luh0.copy()
    t_ref, _, pic = Oracle(dim, order).run(ref, ncell, size, steps, want_picard=True)
    s = exa.Solver(exa.PDE_EULER, dim, order, precision=exa.PREC_MIXED)
    s.predictor_variant = variant
    p = exa.Patch(s, [dict(ncell=ncell, size=size)])
    p.set_solution(luh0)
    p.step(steps)
    got = p.get_solution()
    assert s.predictor_variant == variant
    assert rel(got, ref) < 1e-9
    assert abs(p.time()[0][0] - t_ref) <= 1e-9 * t_ref
    assert p.stats()["picard_mean"] == pytest.approx(pic[-1].mean())
    assert p.status() == 0


@pytest.mark.parametrize("name,order,var", [("acoustic", 4, 0), ("elastic", 3, 3)])
def test_mixed_precision_linear_waves_source_vs_fp64_oracle(exa, name, order, var):
    """The mixed form on the linear systems with the point source (the source enters sweep 0's
    closed form) and outflow faces, both launch forms."""
    import exa_scenarios as sc
    from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC
    pde = {"acoustic": PDE_ACOUSTIC, "elastic": PDE_ELASTIC}[name]
    ncell, size = (5, 4, 6), [1.0, 0.8, 1.2]
    src = sc.ricker_source(3, size, f0=4.0, variable=var, width=0.1)
    src = src[:4] + (0.05,) + src[5:]
    rng = np.random.default_rng(6)
    luh0 = sc.layered_medium(name, ncell, size, order, seed=2)
    D = exa.NVAR[pde] + exa.NPAR[pde]
    lv = luh0.reshape(-1, D)
    lv[:, :exa.NVAR[pde]] += 0.01 * rng.normal(size=(lv.shape[0], exa.NVAR[pde]))  # every cell iterates
    o = Oracle(3, order, pde, source=src)
    ref = luh0.copy()
    t_ref, _, pic = o.run(ref, ncell, size, 3, walls=3, want_picard=True)
    for variant in (0, 1):
        s = exa.Solver(pde, 3, order, npar=exa.NPAR[pde], precision=exa.PREC_MIXED)
        s.predictor_variant = variant
        p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=3)])
        p.set_point_source(src[:3], src[3], src[4], src[5], src[6], int(src[7]))
        p.set_solution(luh0)
        p.step(3)
        got = p.get_solution()
        assert rel(got, ref) < 1e-9, (variant, rel(got, ref))
        assert abs(p.time()[0][0] - t_ref) <= 1e-9 * t_ref
        assert p.stats()["picard_mean"] == pytest.approx(pic[-1].mean())
        assert pic[-1].mean() > 1.5
        assert p.status() == 0
        p.close()


@pytest.mark.parametrize("case", ["euler3d_n5", "euler2d_n3", "swe_grids", "acoustic_outflow"])
def test_update_launch_forms_agree(exa, case):
    """The update kernel's two launch forms (per-thread loads; persistent CTAs moving whole cell
    blocks by bulk copy) give bit-identical steps, equal to the oracle."""
    import exa_scenarios as sc
    from pyoracle import PDE_ACOUSTIC
    rng = np.random.default_rng(5)
    if case == "euler3d_n5":
        mk = lambda: exa.Solver(exa.PDE_EULER, 3, 5)
        specs = [dict(ncell=(4, 3, 5), size=[1.0, 0.8, 1.1])]
        luh0 = euler_cells(rng, 60, 216, amp=0.04).reshape(-1)
        ref = luh0.copy()
        Oracle(3, 5).run(ref, (4, 3, 5), [1.0, 0.8, 1.1], 3)
    elif case == "euler2d_n3":
        mk = lambda: exa.Solver(exa.PDE_EULER, 2, 3)
        specs = [dict(ncell=(11, 9), size=[1.0, 0.9], bc=exa.BC_WALL)]
        luh0 = euler_cells(rng, 99, 16, amp=0.04, dim=2).reshape(-1)
        ref = luh0.copy()
        Oracle(2, 3).run(ref, (11, 9), [1.0, 0.9], 3, walls=True)
    elif case == "swe_grids":
        mk = lambda: exa.Solver(exa.PDE_SWE, 2, 4)
        specs, states = sc.swe_batched(ngrids=3, order=4, seed=9, nmin=5, nmax=9)
        luh0 = np.concatenate(states)
        ref = None
    else:
        mk = lambda: exa.Solver(PDE_ACOUSTIC, 3, 4, npar=2)
        specs = [dict(ncell=(4, 3, 3), size=[1.0, 0.75, 0.75], bc=exa.BC_OUTFLOW)]
        luh0 = sc.layered_medium("acoustic", (4, 3, 3), [1.0, 0.75, 0.75], 4, seed=1)
        lv = luh0.reshape(-1, 6)
        lv[:, :4] += 0.01 * rng.normal(size=(lv.shape[0], 4))
        ref = luh0.copy()
        Oracle(3, 4, PDE_ACOUSTIC).run(ref, (4, 3, 3), [1.0, 0.75, 0.75], 3, walls=3)
    outs = []
    for variant in (0, 1):
        s = mk()
        s.set_update_variant(variant)
        p = exa.Patch(s, specs)
        p.set_solution(luh0)
        p.step(3)
        outs.append(p.get_solution())
        assert p.status() == 0
        p.close()
    assert np.array_equal(outs[0], outs[1])
    if ref is not None:
        assert rel(outs[1], ref) < TOL


@pytest.mark.parametrize("dim,order,ncell", [(3, 5, (5, 4, 3)), (2, 3, (9, 7)), (3, 3, (6, 5, 4))])
def test_fp64_predictor_launch_forms_agree(exa, dim, order, ncell):
    """The FP64 predictor's two launch forms (one cell group per CTA; persistent CTAs with a
    bulk-copy prefetch of the next group) give bit-identical steps, equal to the oracle; the
    measured default is one of them."""
    rng = np.random.default_rng(21)
    luh0 = euler_cells(rng, int(np.prod(ncell)), (order + 1) ** dim, amp=0.04, dim=dim).reshape(-1)
    size = [1.0] * dim
    ref = luh0.copy()
    Oracle(dim, order).run(ref, ncell, size, 2)
    outs = []
    for variant in (0, 1, -1):
        s = exa.Solver(exa.PDE_EULER, dim, order)
        s.predictor_variant = variant
        p = exa.Patch(s, [dict(ncell=ncell, size=size)])
        p.set_solution(luh0)
        p.step(2)
        outs.append(p.get_solution())
        assert p.status() == 0
        assert s.predictor_variant in (0, 1)
        p.close()
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    assert rel(outs[0], ref) < TOL


def test_mixed_precision_rejected_for_ncp(exa):
    with pytest.raises(exa.ExaError):
        exa.Solver(exa.PDE_SWE, 2, 4, precision=exa.PREC_MIXED)


def test_swe_batched_grids_vs_oracle(exa):
    """Batched shallow water: several wall-bounded grids of uneven sizes in one patch, each with
    its own CFL time step, against the oracle run grid by grid."""
    import exa_scenarios as sc
    specs, states = sc.swe_batched(ngrids=5, order=4, seed=3, nmin=6, nmax=14)
    s = exa.Solver(exa.PDE_SWE, 2, 4)
    p = exa.Patch(s, specs)
    p.set_solution(np.concatenate(states))
    p.step(4)
    got = p.get_solution()
    t, _ = p.time()
    o = Oracle(2, 4, pde=PDE_SWE)
    off = 0
    for g, (sp, st) in enumerate(zip(specs, states)):
        ref = st.copy()
        t_ref, _, _ = o.run(ref, sp["ncell"], sp["size"], 4, walls=True)
        assert rel(got[off:off + ref.size], ref) < TOL, g
        assert abs(t[g] - t_ref) <= 1e-13 * t_ref
        off += ref.size
    assert p.status() == 0


def test_swe_batched_grids_vs_reference_kernels(exa):
    """Batched shallow water against the reference's OWN generic kernels (oracle/_ref, the SWE
    app's solver: NCP g h grad b, reflective walls), grid by grid, with equal Picard sweeps."""
    import exa_scenarios as sc
    from pyoracle import RefKernels
    try:
        ref_k = RefKernels(2, 4, "swe")
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)
    specs, states = sc.swe_batched(ngrids=4, order=4, seed=8, nmin=5, nmax=12)
    s = exa.Solver(exa.PDE_SWE, 2, 4)
    p = exa.Patch(s, specs)
    p.set_solution(np.concatenate(states))
    p.step(4)
    got = p.get_solution()
    t, _ = p.time()
    off = 0
    for g, (sp, st) in enumerate(zip(specs, states)):
        ref = st.copy()
        t_ref, _, _ = ref_k.run(ref, sp["ncell"], sp["size"], 4, walls=True, want_picard=True)
        assert rel(got[off:off + ref.size], ref) < TOL, (g, rel(got[off:off + ref.size], ref))
        assert abs(t[g] - t_ref) <= 1e-13 * t_ref
        assert np.abs(ref - st).max() > 1e-3
        off += ref.size
    assert p.status() == 0
    # Picard sweeps of the last step: the GPU's histogram equals the reference's counts, which
    # are the loop index MaxIterations+2 for converged cells (2D return quirk) -> use the
    # restatement's sweep counts, pinned to the reference above, for the histogram
    o = Oracle(2, 4, pde=PDE_SWE)
    hist = np.zeros(32, dtype=int)
    for sp, st in zip(specs, states):
        _, _, pic_o = o.run(st.copy(), sp["ncell"], sp["size"], 4, walls=True, want_picard=True)
        hist += np.bincount(pic_o[-1], minlength=32)[:32]
    assert list(hist) == p.stats()["picard_hist"]
    assert hist[2:].sum() == hist.sum() and hist[3:].sum() > 0  # non-trivial iterations


@pytest.mark.parametrize("nz,split", [(6, 3), (5, 2)])
def test_two_slabs_with_halo_match_whole_grid(exa, torch, nz, split):
    """The slab-decomposition path on one GPU: two halo patches (lower and upper slab of a periodic
    grid) advanced phase by phase, with the host copying the exchange buffers between them, give
    the same state as one whole-grid patch (the exchange a multi-GPU run does with NCCL)."""
    rng = np.random.default_rng(8)
    order, nx, ny = 3, 3, 4
    nd = (order + 1) ** 3
    size = [1.0, 0.9, 1.1]
    hz = size[2] / nz
    luh0 = euler_cells(rng, nx * ny * nz, nd, amp=0.04).reshape(-1)
    s = exa.Solver(exa.PDE_EULER, 3, order)
    whole = exa.Patch(s, [dict(ncell=(nx, ny, nz), size=size)])
    whole.set_solution(luh0)
    whole.step(3)
    ref = whole.get_solution()
    layer = nx * ny * nd * 5
    slabs = []
    for first, count in ((0, split), (split, nz - split)):
        p = exa.Patch(s, [dict(ncell=(nx, ny, count), size=[size[0], size[1], count * hz],
                               offset=[0, 0, first * hz], bc=[exa.BC_PERIODIC, exa.BC_PERIODIC, exa.BC_HALO])])
        p.set_solution(luh0[first * layer:(first + count) * layer])
        nh = p.halo_doubles()
        bufs = {k: torch.zeros(nh, dtype=torch.float64, device="cuda") for k in ("slo", "shi", "rlo", "rhi")}
        slabs.append((p, bufs))
    dtb = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in slabs]
    with pytest.raises(exa.ExaError):
        slabs[0][0].step(1)  # halo patches refuse the single-device step
    for (p, _), b in zip(slabs, dtb):
        p.dt_copy(b, 0)
    torch.cuda.synchronize()
    m = torch.minimum(dtb[0], dtb[1])
    for (p, _), b in zip(slabs, dtb):
        b.copy_(m)
        p.dt_copy(b, 1)
    for _ in range(3):
        for p, bf in slabs:
            p.step_phase(exa.PHASE_PREDICTOR)
            p.halo_pack(bf["slo"], bf["shi"])
        torch.cuda.synchronize()
        (pa, a), (pb, b) = slabs
        a["rlo"].copy_(b["shi"]); a["rhi"].copy_(b["slo"])  # periodic: each slab is the other's both neighbours
        b["rlo"].copy_(a["shi"]); b["rhi"].copy_(a["slo"])
        torch.cuda.synchronize()
        for p, bf in slabs:
            p.halo_unpack(bf["rlo"], bf["rhi"])
            p.step_phase(exa.PHASE_FACES)
            p.step_phase(exa.PHASE_UPDATE)
        for (p, _), bb in zip(slabs, dtb):
            p.dt_next_copy(bb, 0)
        torch.cuda.synchronize()
        m = torch.minimum(dtb[0], dtb[1])
        for (p, _), bb in zip(slabs, dtb):
            bb.copy_(m)
            p.dt_next_copy(bb, 1)
            p.step_phase(exa.PHASE_ADVANCE)
    got = np.concatenate([p.get_solution() for p, _ in slabs])
    assert rel(got, ref) < TOL
    assert slabs[0][0].time()[0][0] == whole.time()[0][0]


@pytest.mark.parametrize("nz,split", [(6, 3), (7, 4)])
def test_two_slabs_interior_faces_during_exchange_vs_oracle(exa, torch, nz, split):
    """The multi-GPU step order, emulated with two slabs on one GPU: the faces between each slab's
    own cells run before the exchange buffers are delivered (FACES_INTERIOR), the ghost cells'
    faces after the unpack (FACES_HALO). The joined slabs match the oracle's whole periodic grid at
    1e-12 after 3 CFL steps, with the oracle's time."""
    rng = np.random.default_rng(12)
    order, nx, ny = 3, 4, 3
    nd = (order + 1) ** 3
    size = [1.0, 0.8, 1.3]
    hz = size[2] / nz
    luh0 = euler_cells(rng, nx * ny * nz, nd, amp=0.05).reshape(-1)
    ref = luh0.copy()
    t_ref, _, _ = Oracle(3, order).run(ref, (nx, ny, nz), size, 3)
    s = exa.Solver(exa.PDE_EULER, 3, order)
    layer = nx * ny * nd * 5
    slabs = []
    for first, count in ((0, split), (split, nz - split)):
        p = exa.Patch(s, [dict(ncell=(nx, ny, count), size=[size[0], size[1], count * hz],
                               offset=[0, 0, first * hz], bc=[exa.BC_PERIODIC, exa.BC_PERIODIC, exa.BC_HALO])])
        p.set_solution(luh0[first * layer:(first + count) * layer])
        nh = p.halo_doubles()
        slabs.append((p, {k: torch.zeros(nh, dtype=torch.float64, device="cuda") for k in ("slo", "shi", "rlo", "rhi")}))
    dtb = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in slabs]
    for (p, _), b in zip(slabs, dtb):
        p.dt_copy(b, 0)
    torch.cuda.synchronize()
    m = torch.minimum(dtb[0], dtb[1])
    for (p, _), b in zip(slabs, dtb):
        b.copy_(m)
        p.dt_copy(b, 1)
    for _ in range(3):
        for p, bf in slabs:
            p.step_phase(exa.PHASE_PREDICTOR)
            p.halo_pack(bf["slo"], bf["shi"])
            p.step_phase(exa.PHASE_FACES_INTERIOR)  # before the neighbours' traces exist
        torch.cuda.synchronize()
        (pa, a), (pb, b) = slabs
        a["rlo"].copy_(b["shi"]); a["rhi"].copy_(b["slo"])
        b["rlo"].copy_(a["shi"]); b["rhi"].copy_(a["slo"])
        torch.cuda.synchronize()
        for p, bf in slabs:
            p.halo_unpack(bf["rlo"], bf["rhi"])
            p.step_phase(exa.PHASE_FACES_HALO)
            p.step_phase(exa.PHASE_UPDATE)
        for (p, _), bb in zip(slabs, dtb):
            p.dt_next_copy(bb, 0)
        torch.cuda.synchronize()
        m = torch.minimum(dtb[0], dtb[1])
        for (p, _), bb in zip(slabs, dtb):
            bb.copy_(m)
            p.dt_next_copy(bb, 1)
            p.step_phase(exa.PHASE_ADVANCE)
    got = np.concatenate([p.get_solution() for p, _ in slabs])
    assert rel(got, ref) < TOL
    assert abs(slabs[1][0].time()[0][0] - t_ref) <= 1e-13 * t_ref
    for p, _ in slabs:
        assert p.status() == 0
        p.close()


# ------------------------------------------------------------------------------------------
# Linear waves with per-node material parameters, a point source and outflow / wall boundaries
# ------------------------------------------------------------------------------------------

@pytest.mark.parametrize("name,order,var,bc,steps", [
    ("acoustic", 4, 0, 3, 4),   # outflow
    ("acoustic", 4, 0, 0, 3),   # periodic
    ("elastic", 3, 3, 3, 4),    # outflow
    ("elastic", 3, 3, 1, 3),    # rigid walls
    ("elastic", 4, 3, 3, 2),
])
def test_patch_linear_waves_source_vs_oracle(exa, name, order, var, bc, steps):
    import exa_scenarios as sc
    from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC
    pde = {"acoustic": PDE_ACOUSTIC, "elastic": PDE_ELASTIC}[name]
    ncell, size = (5, 4, 6), [1.0, 0.8, 1.2]
    src = sc.ricker_source(3, size, f0=4.0, variable=var, width=0.1)
    src = src[:4] + (0.05,) + src[5:]
    luh0 = sc.layered_medium(name, ncell, size, order, seed=2)
    o = Oracle(3, order, pde, source=src)
    ref = luh0.copy()
    t_ref, dts, _ = o.run(ref, ncell, size, steps, walls=bc)
    s = exa.Solver(pde, 3, order, npar=exa.NPAR[pde])
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    p.set_point_source(src[:3], src[3], src[4], src[5], src[6], int(src[7]))
    p.set_solution(luh0)
    p.step(steps)
    got = p.get_solution()
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    assert rel(got, ref) < TOL
    assert np.abs(ref - luh0).max() > 1e-3
    assert p.status() == 0
    p.close()


def test_point_source_off_matches_sourceless_oracle(exa):
    """Removing the source (exa_patch_set_point_source(NULL)) gives the source-free update."""
    import exa_scenarios as sc
    from pyoracle import PDE_ACOUSTIC
    ncell, size, order = (4, 4, 4), [1.0, 1.0, 1.0], 4
    src = sc.ricker_source(3, size, variable=0, width=0.1)
    luh0 = sc.layered_medium("acoustic", ncell, size, order, seed=5)
    o = Oracle(3, order, PDE_ACOUSTIC)
    ref = luh0.copy()
    o.run(ref, ncell, size, 2, walls=3)
    s = exa.Solver(exa.PDE_ACOUSTIC, 3, order, npar=2)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=exa.BC_OUTFLOW)])
    p.set_point_source(src[:3], src[3], src[4], src[5], src[6], 0)
    p.set_point_source(None)
    p.set_solution(luh0)
    p.step(2)
    assert rel(p.get_solution(), ref) < TOL
    p.close()


@pytest.mark.parametrize("pde_name,order,bc", [("euler", 3, 0), ("acoustic", 4, 3), ("elastic", 3, 1)])
def test_patch_fixed_picard_count_vs_oracle(exa, pde_name, order, bc):
    """max_picard = Order+1: the reference's fixed-count mode (no residual test); lFhi is the flux
    of the last sweep's starting iterate."""
    import exa_scenarios as sc
    from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC, PDE_EULER
    ncell, size, steps = (4, 3, 5), [1.0, 0.75, 1.25], 3
    if pde_name == "euler":
        rng = np.random.default_rng(2)
        luh0 = euler_cells(rng, int(np.prod(ncell)), (order + 1) ** 3, amp=0.05).reshape(-1)
        pde, src = PDE_EULER, None
    else:
        pde = PDE_ACOUSTIC if pde_name == "acoustic" else PDE_ELASTIC
        luh0 = sc.layered_medium(pde_name, ncell, size, order, seed=6)
        src = sc.ricker_source(3, size, f0=4.0, variable=0 if pde_name == "acoustic" else 3, width=0.1)
        src = src[:4] + (0.05,) + src[5:]
    o = Oracle(3, order, pde, source=src, max_picard=order + 1)
    ref = luh0.copy()
    t_ref, _, pic = o.run(ref, ncell, size, steps, walls=bc, want_picard=True)
    assert (pic == order + 1).all()
    s = exa.Solver(pde, 3, order, npar=exa.NPAR[pde], max_picard=order + 1)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    if src is not None:
        p.set_point_source(src[:3], src[3], src[4], src[5], src[6], int(src[7]))
    p.set_solution(luh0)
    p.step(steps)
    assert rel(p.get_solution(), ref) < TOL
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    p.close()


def test_patch_fixed_dt_many_steps_vs_oracle(exa):
    """Several steps with a fixed time step, through exa_patch_step and through the phases."""
    rng = np.random.default_rng(8)
    order, ncell, size, steps = 3, (3, 4, 3), [0.9, 1.0, 0.8], 5
    luh0 = euler_cells(rng, int(np.prod(ncell)), (order + 1) ** 3, amp=0.04).reshape(-1)
    o = Oracle(3, order)
    ref = luh0.copy()
    dt = 0.5 * min(o.dt(luh0[c * 64 * 5:(c + 1) * 64 * 5], np.array(size) / np.array(ncell)) for c in range(36))
    t_ref, dts, _ = o.run(ref, ncell, size, steps, fixed_dt=dt)
    assert np.all(dts == dt)
    s = exa.Solver(exa.PDE_EULER, 3, order)
    p = exa.Patch(s, [dict(ncell=ncell, size=size)])
    p.set_solution(luh0)
    p.step(steps, dt)
    assert rel(p.get_solution(), ref) < TOL
    t, dtp = p.time()
    assert abs(t[0] - steps * dt) <= 1e-14 and dtp[0] == dt
    p.set_solution(luh0)
    for _ in range(steps):
        for ph in (exa.PHASE_PREDICTOR, exa.PHASE_FACES, exa.PHASE_UPDATE, exa.PHASE_ADVANCE):
            p.step_phase(ph, dt)
    assert rel(p.get_solution(), ref) < TOL
    p.close()


@pytest.mark.parametrize("ncell,bc,steps,fixed", [((2, 3, 2), 3, 2, False), ((3, 2, 2), 0, 2, False),
                                                  ((2, 2, 2), 1, 2, True), ((6, 5, 6), 3, 2, False),
                                                  ((8, 5, 8), 1, 2, True)])
def test_patch_elastic_order7_streamed_vs_oracle(exa, ncell, bc, steps, fixed):
    """Order 7 (8^3 nodes x 12 data per cell): the streamed predictor (iterates in global scratch).
    The persistent grid has one CTA per SM (148 on a B200): the 180- and 320-cell grids make CTAs
    walk two or three cells, reusing their scratch slot and per-cell shared state."""
    import exa_scenarios as sc
    from pyoracle import PDE_ELASTIC
    order, size = 7, [1.0, 1.2, 0.9]
    luh0 = sc.layered_medium("elastic", ncell, size, order, seed=4)
    src = sc.ricker_source(3, size, f0=4.0, variable=2, width=0.15)
    src = src[:4] + (0.05,) + src[5:]
    mp = order + 1 if fixed else 0
    o = Oracle(3, order, PDE_ELASTIC, source=src, max_picard=mp)
    ref = luh0.copy()
    t_ref, _, pic = o.run(ref, ncell, size, steps, walls=bc, want_picard=True)
    s = exa.Solver(exa.PDE_ELASTIC, 3, order, npar=3, max_picard=mp)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    p.set_point_source(src[:3], src[3], src[4], src[5], src[6], int(src[7]))
    p.set_solution(luh0)
    p.step(steps)
    assert rel(p.get_solution(), ref) < TOL
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    assert p.status() == 0
    p.close()


@pytest.mark.parametrize("case", ["euler3d_n3", "swe_multigrid", "elastic_n7_fixed"])
def test_step_host_matches_device_steps(exa, torch, case):
    """exa_patch_step_host (chunked copies overlapped with the kernels, cell ranges that do not
    align with cells per CTA) gives the same states as device-resident steps."""
    import exa_scenarios as sc
    steps, fixed = 3, 0.0
    if case == "euler3d_n3":
        rng = np.random.default_rng(12)
        ncell, order = (5, 4, 3), 3
        luh0 = euler_cells(rng, 60, 64, amp=0.05).reshape(-1)
        s = exa.Solver(exa.PDE_EULER, 3, order)
        grids = [dict(ncell=ncell, size=[1.0, 0.8, 0.6])]
    elif case == "swe_multigrid":
        specs, states = sc.swe_batched(ngrids=5, nmin=3, nmax=7, seed=4)
        luh0 = np.concatenate(states)
        s = exa.Solver(exa.PDE_SWE, 2, 4)
        grids = specs
    else:
        ncell, order = (2, 3, 2), 7
        luh0 = sc.layered_medium("elastic", ncell, [1.0, 1.0, 1.0], order, seed=2)
        s = exa.Solver(exa.PDE_ELASTIC, 3, order, npar=3)
        grids = [dict(ncell=ncell, size=[1.0, 1.0, 1.0], bc=exa.BC_OUTFLOW)]
        fixed = 1e-3
    dev = exa.Patch(s, grids)
    dev.set_solution(luh0)
    dev.step(steps, fixed)
    ref = dev.get_solution()
    host = exa.Patch(s, grids)
    buf = torch.from_numpy(luh0.copy()).pin_memory()
    host.set_solution(buf.numpy())
    for _ in range(steps):
        host.step_host(buf, buf, fixed)
    assert rel(buf.numpy(), ref) < 1e-14
    t1, t2 = dev.time()[0], host.time()[0]
    assert np.allclose(t1, t2, rtol=1e-15, atol=0)
    # all steps in one call: uploads of step k overlap the downloads of step k-1
    multi = exa.Patch(s, grids)
    src = torch.from_numpy(luh0.copy()).pin_memory()
    out = torch.zeros_like(src).pin_memory()
    multi.set_solution(src.numpy())
    multi.step_host(src, out, fixed, nsteps=steps)
    assert rel(out.numpy(), ref) < 1e-14
    assert np.array_equal(src.numpy(), luh0)   # the input buffer is only read
    assert np.allclose(multi.time()[0], t1, rtol=1e-15, atol=0)
    dev.close()
    host.close()
    multi.close()


def test_step_host_fixed_then_cfl_and_halo_refusal(exa, torch):
    """Host-buffer steps with a fixed dt followed by CFL steps follow the device-resident sequence
    (the CFL step of the uploaded state is recomputed after fixed steps); halo patches are refused."""
    rng = np.random.default_rng(21)
    order, ncell, size = 3, (4, 3, 3), [1.0, 0.75, 0.75]
    luh0 = euler_cells(rng, 36, 64, amp=0.05).reshape(-1)
    s = exa.Solver(exa.PDE_EULER, 3, order)
    dev = exa.Patch(s, [dict(ncell=ncell, size=size)])
    dev.set_solution(luh0)
    dev.step(2, 2e-3)
    dev.step(2)
    ref = dev.get_solution()
    host = exa.Patch(s, [dict(ncell=ncell, size=size)])
    buf = torch.from_numpy(luh0.copy()).pin_memory()
    host.set_solution(buf.numpy())
    host.step_host(buf, buf, 2e-3, nsteps=2)
    host.step_host(buf, buf, 0.0, nsteps=2)
    assert rel(buf.numpy(), ref) < 1e-14
    assert np.allclose(host.time()[0], dev.time()[0], rtol=1e-15, atol=0)
    halo = exa.Patch(s, [dict(ncell=ncell, size=size, bc=[exa.BC_PERIODIC, exa.BC_PERIODIC, exa.BC_HALO])])
    with pytest.raises(exa.ExaError):
        halo.step_host(buf, buf)
    for p in (dev, host, halo):
        p.close()


def test_empty_batches_and_argument_checks(exa, torch):
    """Zero cells or faces are valid batches that launch nothing and leave the outputs untouched;
    null arrays with a non-empty batch, negative counts and out-of-range directions are refused on
    the host with EXA_ERR_INVALID, before any launch (the reference's kernels take one cell at a
    time, so these are the batched interface's own edge cases)."""
    lib = exa.load_library()
    s = exa.Solver(exa.PDE_EULER, 3, 3)
    dev = torch.device("cuda")
    sentinel = torch.full((64,), 7.0, dtype=torch.float64, device=dev)
    ptr = sentinel.data_ptr()
    import ctypes
    dx = (ctypes.c_double * 3)(0.1, 0.1, 0.1)
    null = None
    # empty batches: OK, nothing written
    assert lib.exa_fused_predictor_volume_integral(s.h, 0, null, null, null, null, null, dx, 0.0, 1e-3, null) == 0
    assert lib.exa_riemann_solver_nonlinear(s.h, 0, null, null, null, null, null, null) == 0
    assert lib.exa_boundary_conditions_wall(s.h, 0, null, null, null, null, null) == 0
    assert lib.exa_surface_integral_and_update(s.h, 0, null, null, null, dx, 1e-3, null) == 0
    assert lib.exa_solution_update(s.h, 0, null, null, null, 1e-3, null) == 0
    torch.cuda.synchronize()
    assert bool((sentinel == 7.0).all())
    # refused on the host
    assert lib.exa_fused_predictor_volume_integral(s.h, 1, null, ptr, ptr, ptr, null, dx, 0.0, 1e-3, null) == 1
    assert lib.exa_fused_predictor_volume_integral(s.h, -1, ptr, ptr, ptr, ptr, null, dx, 0.0, 1e-3, null) == 1
    assert lib.exa_riemann_solver_nonlinear(s.h, -1, null, null, null, null, null, null) == 1
    assert lib.exa_riemann_solver_nonlinear(s.h, 2, null, null, null, ptr, ptr, null) == 1
    assert lib.exa_stable_time_step_size(s.h, -1, null, dx, null, null, null) == 1
    FL = FR = QL = QR = np.zeros(16 * 5)
    with pytest.raises(exa.ExaError):
        s.riemann_cell(FL, FR, QL, QR, 0.1, 3)  # direction out of range in 3D
    assert s.status() == 0
    assert bool((sentinel == 7.0).all())
    s.close()
