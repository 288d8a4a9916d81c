"""Discrete adjoint of the ADER-DG step (acoustic and elastic systems) on the GPU.

There is no reference adjoint. The checks are
* tangent/adjoint dot products: the step is linear in the evolved state for fixed parameters
  and without a source, so <L du, w> = <du, L^T w> must hold to rounding, with L du a forward
  step of du and L^T w one exa_patch_adjoint_step;
* central finite differences (h = 1e-6) of the parameter part of one step;
* central finite differences of the whole checkpointed misfit gradient, through the GPU forward
  model and through the reference's own CPU kernels (fixed Picard count instantiation);
* invariance of the gradient under the checkpoint budget.
"""
import numpy as np
import pytest

from conftest import REPO  # noqa: F401  (path setup)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.fixture(scope="module")
def exa():
    import exa_aderdg
    return exa_aderdg


def _params(exa, pde, ncells, rng):
    if pde == exa.PDE_ACOUSTIC:
        return np.stack([rng.uniform(1.0, 2.5, ncells), rng.uniform(1.5, 3.0, ncells)], -1), 3.0
    cp = rng.uniform(4.0, 6.5, ncells)
    cs = cp / np.sqrt(3.0) * rng.uniform(0.9, 1.1, ncells)
    return np.stack([rng.uniform(2.0, 3.0, ncells), cp, cs], -1), 6.5


def _luh(params, fields, nd):
    ncells, P = params.shape
    V = fields.shape[-1]
    luh = np.zeros((ncells, nd, V + P))
    luh[:, :, :V] = fields
    luh[:, :, V:] = params[:, None, :]
    return luh


CASES = [("acoustic", 4), ("elastic", 3)]
# periodic, reflective walls, outflow, and walls / outflow / periodic per axis
BCS = [0, 1, 3, (1, 3, 0)]
BC_IDS = ["periodic", "walls", "outflow", "mixed"]


@pytest.mark.parametrize("name,order", CASES)
@pytest.mark.parametrize("bc", BCS, ids=BC_IDS)
def test_dot_product_state(exa, torch, name, order, bc):
    from exa_adjoint import cfl_dt
    pde = exa.PDE_ACOUSTIC if name == "acoustic" else exa.PDE_ELASTIC
    V, P = exa.NVAR[pde], exa.NPAR[pde]
    ncell, size = (4, 3, 5), [1.0, 0.75, 1.25]
    nc, nd = int(np.prod(ncell)), (order + 1) ** 3
    rng = np.random.default_rng(7)
    params, cmax = _params(exa, pde, nc, rng)
    dt = cfl_dt(ncell, size, order, cmax)
    s = exa.Solver(pde, 3, order, npar=P, max_picard=order + 1)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    du = rng.normal(size=(nc, nd, V))
    w = rng.normal(size=(nc, nd, V))
    p.set_solution(_luh(params, du, nd).reshape(-1))
    p.step(1, dt)
    Ldu = p.get_solution().reshape(nc, nd, V + P)[:, :, :V]
    lam = torch.tensor(_luh(np.zeros_like(params), w, nd).reshape(-1), device="cuda")
    p.set_solution(_luh(params, du, nd).reshape(-1))
    p.adjoint_step(lam, dt)
    p.sync()
    LTw = lam.cpu().numpy().reshape(nc, nd, V + P)[:, :, :V]
    lhs, rhs = float((Ldu * w).sum()), float((du * LTw).sum())
    # a wrong transpose misses by O(1) of this scale; rounding stays near 1e-15 of it
    scale = float(np.abs(Ldu * w).sum())
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)
    # the adjoint leaves the forward state untouched
    assert np.array_equal(p.get_solution().reshape(nc, nd, V + P)[:, :, :V], du)
    p.close()


@pytest.mark.parametrize("name,order", CASES)
@pytest.mark.parametrize("bc", BCS, ids=BC_IDS)
def test_parameter_adjoint_of_one_step_vs_fd(exa, torch, name, order, bc):
    from exa_adjoint import cfl_dt
    pde = exa.PDE_ACOUSTIC if name == "acoustic" else exa.PDE_ELASTIC
    V, P = exa.NVAR[pde], exa.NPAR[pde]
    ncell, size = (3, 4, 3), [0.75, 1.0, 0.75]
    nc, nd = int(np.prod(ncell)), (order + 1) ** 3
    rng = np.random.default_rng(11)
    params, cmax = _params(exa, pde, nc, rng)
    dt = 0.9 * cfl_dt(ncell, size, order, cmax)
    u = rng.normal(size=(nc, nd, V))
    w = rng.normal(size=(nc, nd, V))
    s = exa.Solver(pde, 3, order, npar=P, max_picard=order + 1)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])

    def f(par):
        p.set_solution(_luh(par, u, nd).reshape(-1))
        p.step(1, dt)
        return float((p.get_solution().reshape(nc, nd, V + P)[:, :, :V] * w).sum())

    lam = torch.tensor(_luh(np.zeros_like(params), w, nd).reshape(-1), device="cuda")
    p.set_solution(_luh(params, u, nd).reshape(-1))
    p.adjoint_step(lam, dt)
    p.sync()
    g = lam.cpu().numpy().reshape(nc, nd, V + P)[:, :, V:].sum(1)    # per-cell parameter gradient
    for k in range(3):
        v = rng.normal(size=params.shape) * params
        h = 1e-6
        fd = (f(params + h * v) - f(params - h * v)) / (2 * h)
        ad = float((g * v).sum())
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-8), (k, fd, ad)
    p.close()


def _small_inversion(exa, ncell, order, nsteps, snaps, nrec=8, seed=3, bc=0):
    from exa_adjoint import WaveInversion, acoustic_model, cfl_dt
    size = [1.0, 1.0, 1.0]
    m = acoustic_model(ncell, size, order, seed=seed, width=0.2)
    dt = cfl_dt(ncell, size, order, 3.0 * 1.05)
    inv = WaveInversion(exa.PDE_ACOUSTIC, ncell, size, order, dt, nsteps, m["receivers"][:nrec], snaps=snaps,
                        bc=bc)
    return inv, m, dt


@pytest.mark.parametrize("bc", [3, (1, 3, 1)], ids=["outflow", "walls_and_outflow"])
def test_misfit_gradient_with_domain_faces_vs_gpu_fd(exa, torch, bc):
    """The checkpointed gradient on a bounded domain (absorbing outflow faces; walls) against
    central finite differences of the GPU forward model."""
    from exa_adjoint import Misfit, fd_directional
    ncell, order, nsteps = (4, 5, 4), 4, 16
    inv, m, dt = _small_inversion(exa, ncell, order, nsteps, snaps=4, bc=bc)
    dev = torch.device("cuda")
    params_true = torch.tensor(np.stack([m["rho"], m["c_true"]], -1), device=dev)
    p0 = torch.tensor(m["p0"], device=dev)
    data = inv.forward_traces(inv.assemble(params_true, p0))
    params = torch.tensor(np.stack([m["rho"], m["c"]], -1), device=dev, requires_grad=True)
    field = p0.clone().requires_grad_(True)
    Misfit.apply(params, field, inv, data).backward()
    gp, gf = params.grad.clone(), field.grad.clone()
    rng = np.random.default_rng(9)
    for k in range(3):
        vp = torch.tensor(rng.normal(size=tuple(params.shape)), device=dev) * params.detach()
        vf = torch.tensor(rng.normal(size=tuple(field.shape)), device=dev)
        fd = fd_directional(inv, params.detach(), field.detach(), vp, vf, data, h=1e-6)
        ad = float((gp * vp).sum() + (gf * vf).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd), (k, fd, ad)
    inv.close()


def test_misfit_gradient_vs_gpu_fd_and_checkpoint_budget(exa, torch):
    from exa_adjoint import Misfit, fd_directional
    ncell, order, nsteps = (5, 4, 6), 4, 24
    inv, m, dt = _small_inversion(exa, ncell, order, nsteps, snaps=4)
    dev = torch.device("cuda")
    params_true = torch.tensor(np.stack([m["rho"], m["c_true"]], -1), device=dev)
    p0 = torch.tensor(m["p0"], device=dev)
    data = inv.forward_traces(inv.assemble(params_true, p0))
    params = torch.tensor(np.stack([m["rho"], m["c"]], -1), device=dev, requires_grad=True)
    field = p0.clone().requires_grad_(True)
    J = Misfit.apply(params, field, inv, data)
    J.backward()
    gp, gf = params.grad.clone(), field.grad.clone()
    assert float(J.detach()) > 0 and torch.isfinite(gp).all() and torch.isfinite(gf).all()
    rng = np.random.default_rng(5)
    for k in range(4):
        vp = torch.tensor(rng.normal(size=tuple(params.shape)), device=dev) * params.detach()
        vf = torch.tensor(rng.normal(size=tuple(field.shape)), device=dev)
        fd = fd_directional(inv, params.detach(), field.detach(), vp, vf, data, h=1e-6)
        ad = float((gp * vp).sum() + (gf * vf).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd), (k, fd, ad)
    # the same gradient when every state is stored
    inv_all, _, _ = _small_inversion(exa, ncell, order, nsteps, snaps=nsteps)
    params2 = params.detach().clone().requires_grad_(True)
    field2 = p0.clone().requires_grad_(True)
    Misfit.apply(params2, field2, inv_all, data).backward()
    assert float((params2.grad - gp).abs().max()) <= 1e-12 * float(gp.abs().max())
    assert float((field2.grad - gf).abs().max()) <= 1e-12 * float(gf.abs().max())
    inv.close()
    inv_all.close()


def test_misfit_gradient_vs_reference_cpu_fd(exa, torch):
    """J and its directional derivatives from the reference's own CPU kernels (fixed Picard
    count), against the GPU forward and the GPU adjoint gradient."""
    from pyoracle import RefKernels
    from exa_adjoint import Misfit
    try:
        ref = RefKernels(3, 4, "acousticfixed", 2)
    except (FileNotFoundError, AttributeError, OSError) as e:
        pytest.skip("reference kernels not built: %s" % e)
    ncell, order, nsteps = (4, 4, 4), 4, 10
    inv, m, dt = _small_inversion(exa, ncell, order, nsteps, snaps=3)
    dev = torch.device("cuda")
    nd = (order + 1) ** 3
    params_np = np.stack([m["rho"], m["c"]], -1)
    data_np = np.zeros((nsteps + 1, inv.rec_cells.numel()))
    rc = inv.rec_cells.cpu().numpy()
    rw = inv.rec_w.cpu().numpy()

    def J_cpu(par, p0, data=None):
        luh = _luh(par, np.stack([p0, 0 * p0, 0 * p0, 0 * p0], -1), nd).reshape(-1)
        tr = np.zeros((nsteps + 1, rc.size))
        for k in range(nsteps):
            ref.run(luh, ncell, [1.0, 1.0, 1.0], 1, t0=k * dt, fixed_dt=dt)
            tr[k + 1] = (rw * luh.reshape(-1, nd, 6)[rc, :, 0]).sum(-1)
        if data is None:
            return tr
        r = tr - data
        r[0] = 0.0
        return 0.5 * float((r * r).sum())

    data_np = J_cpu(np.stack([m["rho"], m["c_true"]], -1), m["p0"])
    data = torch.tensor(data_np, device=dev)
    params = torch.tensor(params_np, device=dev, requires_grad=True)
    field = torch.tensor(m["p0"], device=dev, requires_grad=True)
    J = Misfit.apply(params, field, inv, data)
    J.backward()
    Jc = J_cpu(params_np, m["p0"], data_np)
    assert abs(float(J.detach()) - Jc) <= 1e-10 * Jc
    rng = np.random.default_rng(9)
    for k in range(2):
        vp = rng.normal(size=params_np.shape) * params_np
        vf = rng.normal(size=m["p0"].shape)
        h = 1e-6
        fd = (J_cpu(params_np + h * vp, m["p0"] + h * vf, data_np) -
              J_cpu(params_np - h * vp, m["p0"] - h * vf, data_np)) / (2 * h)
        ad = float((params.grad.cpu().numpy() * vp).sum() + (field.grad.cpu().numpy() * vf).sum())
        assert abs(fd - ad) <= 1e-6 * abs(fd), (k, fd, ad)
    inv.close()


def test_adjoint_rejects_unsupported(exa, torch):
    s = exa.Solver(exa.PDE_EULER, 3, 3)
    p = exa.Patch(s, [dict(ncell=(2, 2, 2), size=[1.0, 1.0, 1.0])])
    lam = torch.zeros(p.ncells * s.sizes["luh"], dtype=torch.float64, device="cuda")
    with pytest.raises(exa.ExaError):
        p.adjoint_step(lam, 1e-3)
    s2 = exa.Solver(exa.PDE_ACOUSTIC, 3, 4, npar=2)   # residual-tested Picard: no adjoint
    p2 = exa.Patch(s2, [dict(ncell=(2, 2, 2), size=[1.0, 1.0, 1.0])])
    lam2 = torch.zeros(p2.ncells * s2.sizes["luh"], dtype=torch.float64, device="cuda")
    with pytest.raises(exa.ExaError):
        p2.adjoint_step(lam2, 1e-3)
    p.close()
    p2.close()


@pytest.mark.parametrize("name,order", CASES)
@pytest.mark.parametrize("bc_other", [0, 1], ids=["periodic", "walls"])
def test_adjoint_of_two_slabs_matches_whole_grid(exa, torch, name, order, bc_other):
    """The multi-GPU adjoint step emulated on one GPU: two halo patches (the lower and upper slab of
    a grid periodic along z) with their exchange buffers swapped by hand between EXA_ADJ_FORWARD
    and EXA_ADJ_REVERSE (face traces, then the boundary layers' lambda) give the whole-grid adjoint
    step's lambda, parameter entries included, to 1e-12."""
    from exa_adjoint import cfl_dt
    pde = exa.PDE_ACOUSTIC if name == "acoustic" else exa.PDE_ELASTIC
    V, P = exa.NVAR[pde], exa.NPAR[pde]
    ncell, size, split = (3, 2, 5), [0.75, 0.5, 1.25], 2
    nc, nd = int(np.prod(ncell)), (order + 1) ** 3
    rng = np.random.default_rng(21)
    params, cmax = _params(exa, pde, nc, rng)
    dt = cfl_dt(ncell, size, order, cmax)
    s = exa.Solver(pde, 3, order, npar=P, max_picard=order + 1)
    luh = _luh(params, rng.normal(size=(nc, nd, V)), nd).reshape(-1)
    w = rng.normal(size=nc * nd * (V + P))  # nonzero parameter entries: they accumulate
    whole = exa.Patch(s, [dict(ncell=ncell, size=size, bc=(bc_other, bc_other, 0))])
    whole.set_solution(luh)
    lam_w = torch.tensor(w, device="cuda")
    whole.adjoint_step(lam_w, dt)
    whole.sync()
    ref = lam_w.cpu().numpy()
    layer = ncell[0] * ncell[1] * nd * (V + P)
    hz = size[2] / ncell[2]
    slabs = []
    for first, count in ((0, split), (split, ncell[2] - split)):
        p = exa.Patch(s, [dict(ncell=(ncell[0], ncell[1], count), size=[size[0], size[1], count * hz],
                               offset=[0, 0, first * hz], bc=[bc_other, bc_other, exa.BC_HALO])])
        p.set_solution(luh[first * layer:(first + count) * layer])
        lam = torch.tensor(w[first * layer:(first + count) * layer], device="cuda")
        nt, nl = p.halo_doubles(), p.adjoint_halo_doubles()
        assert nl == ncell[0] * ncell[1] * nd * (V + P)
        bufs = {k: torch.zeros(nt if k[0] == "t" else nl, dtype=torch.float64, device="cuda")
                for k in ("tslo", "tshi", "trlo", "trhi", "lslo", "lshi", "lrlo", "lrhi")}
        slabs.append((p, lam, bufs))
    torch.cuda.synchronize()
    with pytest.raises(exa.ExaError):
        slabs[0][0].adjoint_step(slabs[0][1], dt)  # halo patches refuse the one-call step
    with pytest.raises(exa.ExaError):
        slabs[0][0].adjoint_phase(exa.ADJ_REVERSE, slabs[0][1], dt)  # REVERSE needs FORWARD first
    for p, lam, b in slabs:
        p.adjoint_phase(exa.ADJ_FORWARD, lam, dt)
        p.halo_pack(b["tslo"], b["tshi"])
        p.adjoint_halo_pack(b["lslo"], b["lshi"])
    torch.cuda.synchronize()
    (_, _, a), (_, _, b) = slabs
    for k in ("t", "l"):  # periodic: each slab is the other's lower and upper neighbour
        a[k + "rlo"].copy_(b[k + "shi"])
        a[k + "rhi"].copy_(b[k + "slo"])
        b[k + "rlo"].copy_(a[k + "shi"])
        b[k + "rhi"].copy_(a[k + "slo"])
    torch.cuda.synchronize()
    for p, lam, bf in slabs:
        p.halo_unpack(bf["trlo"], bf["trhi"])
        p.adjoint_halo_unpack(bf["lrlo"], bf["lrhi"])
        p.adjoint_phase(exa.ADJ_REVERSE, lam, dt)
        p.sync()
    got = np.concatenate([lam.cpu().numpy() for _, lam, _ in slabs])
    assert float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))) < 1e-12
    assert np.abs(ref - w).max() > 1e-3  # the step changed lambda
    # the phases on a patch without halo equal the one-call step
    lam2 = torch.tensor(w, device="cuda")
    torch.cuda.synchronize()
    whole.adjoint_phase(exa.ADJ_FORWARD, lam2, dt)
    whole.adjoint_phase(exa.ADJ_REVERSE, lam2, dt)
    whole.sync()
    assert np.array_equal(lam2.cpu().numpy(), ref)
    for p, _, _ in slabs:
        p.close()
    whole.close()
