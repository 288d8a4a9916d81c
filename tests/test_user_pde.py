"""Application PDE functors compiled against include/exa_aderdg_user.cuh (the drop-in for the
reference's user solver class and its hooks flux / eigenvalues / boundaryValues /
adjustPointSolution, AbstractGenericADERDGSolverHeader.template:34-68, 220-338).

tests/user_pde/user_euler.cu is such an application: Euler written from the reference's Euler app,
with its own boundary_values (a reflective wall) and adjust_point_solution (a density wave), built
into tests/user_pde/libuser_euler.so by the build step. Loading it registers pde EXA_PDE_USER_BASE
for order 3 in 2D and 3D and for the extreme orders (1 and 9 in 2D; 1, 8 and 9 in 3D, where the
largest cells run the streamed predictor with idle tail threads); the GPU tests run it through the
unchanged C ABI against the oracle.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import REPO

USER_LIB = os.path.join(REPO, "tests", "user_pde", "libuser_euler.so")
TOL = 1e-12


def _load():
    import exa_aderdg as exa
    if not os.path.exists(USER_LIB):
        pytest.skip("the application library was not built")
    exa.load_user_pde(USER_LIB)
    return exa


def test_user_pde_registers_its_instantiations():
    exa = _load()
    base = exa.PDE_USER_BASE
    assert exa.pde_available(base, 3, 3, 0) and exa.pde_available(base, 2, 3, 0)
    for dim, order in [(2, 1), (2, 9), (3, 1), (3, 8), (3, 9)]:
        assert exa.pde_available(base, dim, order, 0)
    assert not exa.pde_available(base, 3, 5, 0) and not exa.pde_available(base + 1, 3, 3, 0)
    assert exa.pde_available(exa.PDE_EULER, 3, 5, 0)
    lib = exa.load_library()
    # ids below the user range and null launchers are refused
    assert lib.exa_register_pde(3, 3, 3, 0, None) == 1


def density_wave(x, dim):
    """The application's adjust_point_solution at t = 0, restated in numpy."""
    z = x[..., 2] if dim == 3 else 0.0
    rho = 1.0 + 0.1 * np.sin(2.0 * np.pi * (x[..., 0] + 2.0 * x[..., 1] + 3.0 * z))
    u = np.array([0.3, 0.2, 0.1 if dim == 3 else 0.0])
    Q = np.zeros(x.shape[:-1] + (5,))
    Q[..., 0] = rho
    Q[..., 1:4] = rho[..., None] * u
    Q[..., 4] = 1.0 / 0.4 + 0.5 * rho * (u ** 2).sum()
    return Q.reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,ncell,bc,order", [
    (3, (4, 3, 5), 4, 3), (3, (3, 4, 3), 0, 3), (2, (9, 7), 4, 3), (2, (8, 6), 0, 3),
    # the extreme orders: 2D order 1 (32 cells per CTA, a ragged last CTA), 2D order 9, 3D order 1,
    # 3D orders 8 and 9 (729 and 1000 nodes: the streamed predictor, tail threads without a node)
    (2, (13, 7), 4, 1), (2, (4, 3), 0, 9), (3, (5, 4, 3), 4, 1), (3, (2, 3, 2), 4, 8), (3, (2, 2, 3), 0, 9)])
def test_user_pde_adjust_and_steps_vs_oracle(dim, ncell, bc, order):
    """adjust_point_solution sets the initial state on the device (checked against the numpy
    restatement at the nodal positions); then 3 steps with the application's boundary_values on
    every domain face (EXA_BC_USER) or periodic, against the oracle's Euler system with reflective
    walls or periodic faces, at 1e-12 relative, with equal time steps."""
    import exa_scenarios as sc
    from pyoracle import Oracle
    exa = _load()
    size = [1.0, 0.8, 1.2][:dim]
    s = exa.Solver(exa.PDE_USER_BASE, dim, order)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    p.adjust_solution()
    luh0 = p.get_solution()
    want = density_wave(sc.nodal_positions(ncell, size, order), dim)
    assert np.max(np.abs(luh0 - want)) <= 1e-14 * np.max(np.abs(want))
    ref = luh0.copy()
    t_ref, _, pic = Oracle(dim, order).run(ref, ncell, size, 3, walls=bc == 4, want_picard=True)
    p.step(3)
    got = p.get_solution()
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    assert float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))) < TOL
    assert np.abs(got - luh0).max() > 1e-4
    # equal Picard sweeps in the last step; at order 1 some cells use all 2(N+1) sweeps in the
    # oracle too, and the patch reports that as EXA_ST_PICARD_CAP, not as an error
    assert list(np.bincount(pic[-1], minlength=32)[:32]) == p.stats()["picard_hist"]
    capped = bool((pic == 2 * (order + 1)).any())
    assert p.status() == (exa.ST_PICARD_CAP if capped else 0)
    p.close()
    s.close()


@pytest.mark.gpu
def test_builtin_functor_without_hooks_refuses_them():
    exa = _load()
    s = exa.Solver(exa.PDE_EULER, 3, 3)
    with pytest.raises(exa.ExaError):
        exa.Patch(s, [dict(ncell=(2, 2, 2), size=[1.0] * 3, bc=exa.BC_USER)])
    p = exa.Patch(s, [dict(ncell=(2, 2, 2), size=[1.0] * 3)])
    with pytest.raises(exa.ExaError):
        p.adjust_solution()


ADV_LIB = os.path.join(REPO, "tests", "user_pde", "libuser_advdiff.so")


def _advdiff_state(rng, ncell, order, size):
    """Three smooth periodic fields plus a little noise on the nodes."""
    import exa_scenarios as sc
    dim = len(ncell)
    x = sc.nodal_positions(ncell, size, order)
    f = np.zeros(x.shape[:-1] + (3,))
    for m in range(3):
        k = rng.integers(1, 3, dim)
        f[..., m] = 1.0 + 0.5 * np.sin(2 * np.pi * (x * (k / np.array(size))).sum(-1) + rng.uniform(0, 6.3))
    return (f + 0.01 * rng.normal(size=f.shape)).reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,ncell", [(3, (4, 3, 5)), (2, (9, 7))])
def test_viscous_flux_pde_vs_reference_kernels(dim, ncell):
    """A PDE with a viscous flux (useViscousFlux) through the application-functor route
    (tests/user_pde/user_advdiff.cu) against the reference's own generic kernels instantiated with
    useViscousFlux = true for the same system: three periodic steps to 1e-12 with equal time steps;
    the per-cell predictor (its return value included), the Rusanov face with the viscous term of
    its speed, and the CFL step with the viscous term of its denominator on their own."""
    from pyoracle import RefKernels
    exa = _load()
    if not os.path.exists(ADV_LIB):
        pytest.skip("the application library was not built")
    exa.load_user_pde(ADV_LIB)
    order = 3
    pde = exa.PDE_USER_BASE + 1
    assert exa.pde_available(pde, dim, order, 0)
    s = exa.Solver(pde, dim, order)
    with pytest.raises(exa.ExaError):
        exa.Solver(pde, dim, order, precision=exa.PREC_MIXED)  # the mixed form has no viscous flux
    ref = RefKernels(dim, order, "advdiff")
    rng = np.random.default_rng(3 + dim)
    size = [1.0, 0.75, 1.25][:dim]
    nc, nd = int(np.prod(ncell)), (order + 1) ** dim
    luh0 = _advdiff_state(rng, ncell, order, size)
    p = exa.Patch(s, [dict(ncell=ncell, size=size)])
    p.set_solution(luh0)
    p.step(3)
    got = p.get_solution()
    want = luh0.copy()
    t_ref, _, _ = ref.run(want, ncell, size, 3)
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    assert float(np.max(np.abs(got - want)) / np.max(np.abs(want))) < TOL
    assert np.abs(got - luh0).max() > 1e-3
    assert p.status() == 0
    dx = np.array(size) / np.array(ncell)
    for c in (0, nc // 2, nc - 1):
        cell = luh0.reshape(nc, -1)[c]
        dt = ref.dt(cell, dx)
        assert abs(s.stable_time_step_size_cell(cell, dx) - dt) <= 1e-15 * dt
        a, b = s.space_time_predictor(cell, dx, dt), ref.predictor(cell, dx, dt)
        assert a["ret"] == b["ret"]
        for k in ("lQhbnd", "lFhbnd", "lQhi"):
            assert float(np.max(np.abs(a[k] - b[k])) / np.max(np.abs(b[k]))) < TOL, k
        assert float(np.max(np.abs(a["lFhi"][:dim * nd * 3] - b["lFhi"][:dim * nd * 3])) /
                     np.max(np.abs(b["lFhi"][:dim * nd * 3]))) < TOL
    nf = (order + 1) ** (dim - 1)
    for d in range(dim):
        QL, QR = rng.normal(size=nf * 3), rng.normal(size=nf * 3)
        FL, FR = rng.normal(size=nf * 3), rng.normal(size=nf * 3)
        ga, gb = s.riemann_cell(FL, FR, QL, QR, dx, d)
        ra, rb = ref.riemann(FL, FR, QL, QR, dx, d)
        assert float(np.max(np.abs(ga - ra)) / np.max(np.abs(ra))) < 1e-14
        assert float(np.max(np.abs(gb - rb)) / np.max(np.abs(rb))) < 1e-14
    # the batched face entry point needs the cell size for a viscous flux
    lib = exa.load_library()
    assert lib.exa_riemann_solver_nonlinear(s.h, 0, None, None, None, None, None, None) != 0
    p.close()
    s.close()


REACT_LIB = os.path.join(REPO, "tests", "user_pde", "libuser_advreact.so")


@pytest.mark.gpu
@pytest.mark.parametrize("dim,ncell,bc", [(3, (4, 3, 5), 0), (3, (3, 4, 3), 1), (2, (9, 7), 0), (2, (8, 6), 1)])
def test_algebraic_source_pde_vs_reference_kernels(dim, ncell, bc):
    """A PDE with its own algebraic source (useSource: position-, time- and state-dependent)
    through the application-functor route (tests/user_pde/user_advreact.cu) against the reference's
    own generic kernels instantiated with useSource for the same system: three steps on periodic or
    wall-bounded grids to 1e-12 with equal time steps; the per-cell predictor at a non-zero time
    (its return value, the face values, lQhi and lFhi with the time-averaged source block); and the
    batched predictor with the cells' centres against the reference's volume integral."""
    import torch
    from pyoracle import RefKernels
    exa = _load()
    if not os.path.exists(REACT_LIB):
        pytest.skip("the application library was not built")
    exa.load_user_pde(REACT_LIB)
    order = 3
    pde = exa.PDE_USER_BASE + 2
    s = exa.Solver(pde, dim, order)
    ref = RefKernels(dim, order, "advreact")
    rng = np.random.default_rng(11 + dim + bc)
    size = [1.0, 0.75, 1.25][:dim]
    nc, nd = int(np.prod(ncell)), (order + 1) ** dim
    luh0 = _advdiff_state(rng, ncell, order, size)
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=bc)])
    p.set_solution(luh0)
    p.step(3)
    got = p.get_solution()
    want = luh0.copy()
    t_ref, _, _ = ref.run(want, ncell, size, 3, walls=bc == 1)
    assert abs(p.time()[0][0] - t_ref) <= 1e-13 * t_ref
    assert float(np.max(np.abs(got - want)) / np.max(np.abs(want))) < TOL
    assert np.abs(got - luh0).max() > 1e-4
    assert p.status() == 0
    dx = np.array(size) / np.array(ncell)
    cells = luh0.reshape(nc, -1)
    centres = np.zeros((nc, 3))
    idx = np.arange(nc)
    for d in range(dim):
        stride = int(np.prod(ncell[:d]))
        centres[:, d] = ((idx // stride) % ncell[d] + 0.5) * dx[d]
    t0, dt = 0.3, 0.5 * ref.dt(cells[0], dx)
    for c in (0, nc // 2, nc - 1):
        a = s.space_time_predictor(cells[c], dx, dt, centre=centres[c], t=t0)
        b = ref.predictor(cells[c], dx, dt, centre=centres[c], t=t0)
        assert a["ret"] == b["ret"]
        for k in ("lQhbnd", "lFhbnd", "lQhi", "lFhi"):
            assert float(np.max(np.abs(a[k] - b[k])) / np.max(np.abs(b[k]))) < TOL, (c, k)
    dev = torch.device("cuda")
    t_luh = torch.from_numpy(luh0).to(dev)
    lduh = torch.zeros(nc * nd * 3, dtype=torch.float64, device=dev)
    qhb = torch.zeros(nc * s.sizes["lQhbnd"], dtype=torch.float64, device=dev)
    fhb = torch.zeros_like(qhb)
    with pytest.raises(exa.ExaError):  # the cells' positions are needed
        s.fused_predictor_volume_integral(t_luh, lduh, qhb, fhb, dx, dt, t=t0)
    s.fused_predictor_volume_integral(t_luh, lduh, qhb, fhb, dx, dt, t=t0,
                                      centres=torch.from_numpy(centres).to(dev))
    torch.cuda.synchronize()
    lduh = lduh.cpu().numpy().reshape(nc, -1)
    for c in (1, nc // 3, nc - 2):
        b = ref.predictor(cells[c], dx, dt, centre=centres[c], t=t0)
        want_du = ref.volume(b["lFhi"], dx)
        assert float(np.max(np.abs(lduh[c] - want_du)) / np.max(np.abs(want_du))) < TOL, c
    p.close()
    s.close()
