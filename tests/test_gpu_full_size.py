"""The configurations at their full sizes, through properties that do not depend on the size.
The oracle is too slow for whole grids of this size, so it checks sampled cells only.

* 3D Euler N=5 on 81^3 periodic cells (4.6 GB of state, the benchmark workload). The domain
  integrals of the five conserved variables stay constant over three steps to rounding: the
  scheme is in flux form with conservative Rusanov faces on a periodic grid. The batched
  predictor's outputs for sampled cells equal the oracle's at 1e-12, with equal Picard sweeps.
  The CFL step is the minimum of the per-cell steps, which equal the oracle's at 1e-15.
* 512 wall-bounded SWE grids, N=4 (3.4 M cells). The water volume and the bathymetry's integral
  over every grid are conserved over five steps: no mass crosses a reflective wall, the NCP acts
  on the momenta only, and the Rusanov dissipation that smooths b's jumps between cells is
  conservative too (the wall's ghost copies b).
* The layered elastic medium, N=7, 48^3 cells, active wavefield. The streamed predictor's
  outputs for sampled cells equal the oracle's at 1e-12, and the material parameters do not
  change over a step.
"""
import numpy as np
import pytest

from conftest import REPO  # noqa: F401  (path setup)
from pyoracle import Oracle, PDE_ELASTIC

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.fixture(scope="module")
def exa():
    import exa_aderdg
    return exa_aderdg


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def node_weights(order, dim):
    import exa_scenarios as sc
    w = sc.gl_weights(order)
    return np.einsum("i,j,k->ijk", w, w, w).reshape(-1) if dim == 3 else np.outer(w, w).reshape(-1)


def sampled_cells(ncells, k, seed):
    rng = np.random.default_rng(seed)
    return np.unique(np.concatenate([[0, ncells - 1], rng.integers(0, ncells, k)]))


def check_sampled_predictor(exa, torch, solver, o, luh_host, t_luh, ncells, dx, dt, cells):
    """The batched predictor over the whole state, against the oracle on the sampled cells."""
    sz = solver.sizes
    dev = torch.device("cuda")
    lduh = torch.zeros(ncells * sz["lduh"], dtype=torch.float64, device=dev)
    qhb = torch.zeros(ncells * sz["lQhbnd"], dtype=torch.float64, device=dev)
    fhb = torch.zeros(ncells * sz["lFhbnd"], dtype=torch.float64, device=dev)
    pic = torch.zeros(ncells, dtype=torch.int32, device=dev)
    solver.fused_predictor_volume_integral(t_luh, lduh, qhb, fhb, dx, dt, picard=pic)
    torch.cuda.synchronize()
    idx = torch.from_numpy(cells).to(dev)
    got_d = lduh.view(ncells, -1)[idx].cpu().numpy()
    got_q = qhb.view(ncells, -1)[idx].cpu().numpy()
    got_f = fhb.view(ncells, -1)[idx].cpu().numpy()
    got_p = pic[idx].cpu().numpy()
    for j, c in enumerate(cells):
        r = o.predictor(luh_host[c], dx, dt)
        assert got_p[j] == r["sweeps"], c
        assert rel(got_q[j], r["lQhbnd"]) < TOL and rel(got_f[j], r["lFhbnd"]) < TOL, c
        assert rel(got_d[j], o.volume(r["lFhi"], dx)) < TOL, c
    del lduh, qhb, fhb, pic


def test_euler_81cubed_full_size(exa, torch):
    import exa_scenarios as sc
    order, n = 5, 81
    ncell, size = (n, n, n), [1.0, 1.0, 1.0]
    cells, nd = n ** 3, 6 ** 3
    luh0 = sc.EntropyWave(3, 0).state(sc.nodal_positions(ncell, size, order)).reshape(cells, nd * 5)
    dx = np.array(size) / n
    s = exa.Solver(exa.PDE_EULER, 3, order)
    p = exa.Patch(s, [dict(ncell=ncell, size=size)])
    p.set_solution(luh0.reshape(-1))
    dev = torch.device("cuda")
    t_luh = torch.empty(cells * nd * 5, dtype=torch.float64, device=dev)
    w = torch.tensor(node_weights(order, 3), device=dev) * float(np.prod(dx))

    def integrals():
        p.get_solution(t_luh)
        p.sync()
        return torch.einsum("cpv,p->v", t_luh.view(cells, nd, 5), w).cpu().numpy()

    m0 = integrals()
    # the CFL step: the minimum of the per-cell steps, which the oracle reproduces on sampled cells
    cell_dt = torch.zeros(cells, dtype=torch.float64, device=dev)
    dt_min = s.stable_time_step_size(t_luh, dx, cell_dt=cell_dt)
    _, dt0 = p.time()
    assert dt_min == float(cell_dt.min().item()) == dt0[0]
    o = Oracle(3, order)
    pick = sampled_cells(cells, 40, 5)
    cdt = cell_dt[torch.from_numpy(pick).to(dev)].cpu().numpy()
    for j, c in enumerate(pick):
        want = o.dt(luh0[c], dx)
        assert abs(cdt[j] - want) <= 1e-15 * want, c
    del cell_dt
    # the batched predictor on the whole state, the oracle on sampled cells
    check_sampled_predictor(exa, torch, s, o, luh0, t_luh, cells, dx, dt_min, pick)
    # conservation over three steps
    p.step(3)
    m3 = integrals()
    assert p.status() == 0
    for v in range(5):
        scale = abs(m0[v]) if abs(m0[v]) > 1e-3 else float(np.abs(luh0[:, v::5]).max())
        assert abs(m3[v] - m0[v]) <= 1e-12 * scale, (v, m0[v], m3[v])
    assert np.abs(t_luh.view(cells, nd * 5).cpu().numpy()[pick] - luh0[pick]).max() > 1e-6  # the state moved
    p.close()


def test_swe_512_grids_full_size(exa, torch):
    import exa_scenarios as sc
    order = 4
    specs, states = sc.swe_batched(ngrids=512)
    s = exa.Solver(exa.PDE_SWE, 2, order)
    p = exa.Patch(s, specs)
    p.set_solution(np.concatenate(states))
    nd = (order + 1) ** 2
    w = node_weights(order, 2)
    ncs = [sp["ncell"][0] * sp["ncell"][1] for sp in specs]
    assert sum(ncs) > 3_000_000

    def volumes(luh, var):
        out, off = [], 0
        for nc in ncs:
            q = luh[off:off + nc * nd * 4].reshape(nc, nd, 4)
            out.append(float((q[..., var] * w).sum()) / nc)  # dx^2 = 1 / nc on the unit square
            off += nc * nd * 4
        return np.array(out)

    luh0 = np.concatenate(states)
    p.step(5)
    got = p.get_solution()
    assert p.status() == 0
    for var in (0, 3):  # water height, bathymetry
        v0, v5 = volumes(luh0, var), volumes(got, var)
        assert np.max(np.abs(v5 - v0) / v0) <= 1e-12, var
    assert np.abs(got[0::4] - luh0[0::4]).max() > 1e-3  # the water moved
    p.close()


def test_elastic_48cubed_full_size_sampled_streamed_predictor(exa, torch):
    import exa_scenarios as sc
    order, n = 7, 48
    ncell, size = (n, n, n), [10.0, 10.0, 10.0]
    cells, nd = n ** 3, 8 ** 3
    luh0, _ = sc.elastic_layers(ncell, size, order, seed=0)
    x = sc.nodal_positions(ncell, size, order)
    q = luh0.reshape(cells, nd, 12)
    for k in range(3):  # the active wavefield of the benchmark's elastic workload
        q[..., k] = 0.1 * np.sin(2 * np.pi * (k + 1) * x[..., (k + 1) % 3] / size[0])
    del x
    luh0 = q.reshape(cells, nd * 12)
    s = exa.Solver(exa.PDE_ELASTIC, 3, order, npar=3)
    dev = torch.device("cuda")
    t_luh = torch.from_numpy(luh0.reshape(-1)).to(dev)
    dx = np.array(size) / n
    dt = s.stable_time_step_size(t_luh, dx)
    o = Oracle(3, order, pde=PDE_ELASTIC)
    check_sampled_predictor(exa, torch, s, o, luh0, t_luh, cells, dx, dt, sampled_cells(cells, 12, 6))
    # one whole step with outflow faces: the material parameters stay as they were
    p = exa.Patch(s, [dict(ncell=ncell, size=size, bc=exa.BC_OUTFLOW)])
    p.set_solution(t_luh)
    p.step(1)
    p.get_solution(t_luh)
    p.sync()
    par = t_luh.view(cells, nd, 12)[..., 9:].cpu().numpy()
    assert np.array_equal(par, q[..., 9:])
    assert p.status() == 0
    p.close()
