"""GPU parity of the mesh-level (3d/amrRoutines.cpph) and limiter (limiter/generic/c/Limiter.cpph)
kernels through the C ABI against the reference's own kernels compiled in oracle/_ref, and against
the reference's limiter known-answer vectors. FP64; 1e-12 relative unless stated.
"""
import os

import numpy as np
import pytest

from conftest import REPO
from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC, PDE_EULER, PDE_SWE, RefAmrLimiter

pytestmark = pytest.mark.gpu
GOLD = os.path.join(REPO, "tests", "golden")
TOL = 1e-12

# (pde, order, nvar, npar) of the library's 3D instantiations
CONFIGS = [(PDE_EULER, 3, 5, 1), (PDE_EULER, 5, 5, 0), (PDE_ACOUSTIC, 4, 4, 2), (PDE_ELASTIC, 4, 9, 3)]
IDS = ["euler_n3_p1", "euler_n5", "acoustic_n4", "elastic_n4"]


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(1e-300, np.max(np.abs(b))))


@pytest.fixture(scope="module")
def exa():
    import exa_aderdg
    return exa_aderdg


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


def subcells(rng, level_delta, dim, count):
    k = 3 ** level_delta
    if level_delta == 1 and dim == 3:
        return [(i1, i2, i3) for i3 in range(3) for i2 in range(3) for i1 in range(3)]
    return [tuple(int(x) for x in rng.integers(0, k, dim)) for _ in range(count)]


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
@pytest.mark.parametrize("level_delta", [1, 2, 3])
def test_volume_unknowns_vs_reference(exa, cfg, level_delta):
    pde, order, nvar, npar = cfg
    rng = np.random.default_rng(10 * order + level_delta)
    s = exa.Solver(pde, 3, order, npar=npar)
    ref = RefAmrLimiter(order, nvar, npar)
    nl = s.sizes["luh"]
    for idx in subcells(rng, level_delta, 3, 4):
        coarse = rng.normal(size=nl)
        got = s.volume_prolongation_cell(coarse, 2, 2 + level_delta, idx)
        want = ref.volume(0, np.zeros(nl), coarse, 2, 2 + level_delta, idx)
        assert rel(got, want) < TOL
        fine, acc = rng.normal(size=nl), rng.normal(size=nl)
        got = s.volume_restriction_cell(acc, fine, 1, 1 + level_delta, idx)
        want = ref.volume(1, acc, fine, 1, 1 + level_delta, idx)
        assert rel(got, want) < TOL
    assert s.status() == 0
    s.close()


@pytest.mark.parametrize("cfg", CONFIGS, ids=IDS)
@pytest.mark.parametrize("level_delta", [1, 2])
def test_face_unknowns_vs_reference(exa, cfg, level_delta):
    pde, order, nvar, npar = cfg
    rng = np.random.default_rng(7 + order + level_delta)
    s = exa.Solver(pde, 3, order, npar=npar)
    ref = RefAmrLimiter(order, nvar, npar)
    nq, nf = s.sizes["lQhbnd"] // 6, s.sizes["lFhbnd"] // 6
    for idx in subcells(rng, level_delta, 2, 5):
        qc, fc = rng.normal(size=nq), rng.normal(size=nf)
        gq, gf = s.face_prolongation_cell(qc, fc, 0, level_delta, idx)
        wq, wf = ref.face(0, np.zeros(nq), np.zeros(nf), qc, fc, 0, level_delta, idx)
        assert rel(gq, wq) < TOL and rel(gf, wf) < TOL
        qf, ff = rng.normal(size=nq), rng.normal(size=nf)
        gq, gf = s.face_restriction_cell(qc, fc, qf, ff, 0, level_delta, idx)
        wq, wf = ref.face(1, qc, fc, qf, ff, 0, level_delta, idx)
        assert rel(gq, wq) < TOL and rel(gf, wf) < TOL
        gf = s.face_flux_restriction_cell(ff, idx, level_delta)
        _, wf = ref.face(2, np.zeros(nq), np.zeros(nf), qf, ff, 0, level_delta, idx)
        assert rel(gf, wf) < TOL
    assert s.status() == 0
    s.close()


def test_known_answers_constants_and_polynomials(exa):
    """The reference's own test (GenericEulerKernelTest3D.cpp:776-851) on the GPU -- a constant is
    prolongated exactly and restored by restricting its children -- and a polynomial of degree N
    prolongated two levels down equals its values at the fine nodes."""
    import exa_scenarios as sc
    s = exa.Solver(PDE_EULER, 3, 3, npar=1)
    nl, D = s.sizes["luh"], 6
    ones = np.ones(nl)
    coarse = np.zeros(nl)
    for i3 in range(3):
        for i2 in range(3):
            for i1 in range(3):
                fine = s.volume_prolongation_cell(ones, 0, 1, (i1, i2, i3))
                assert np.abs(fine - 1.0).max() < 1e-13
                coarse = s.volume_restriction_cell(coarse, ones, 0, 1, (i1, i2, i3))
    assert np.abs(coarse - 1.0).max() < 1e-13
    # cubic polynomial on the unit cell, prolongated to subcell (4, 7, 2) of 9^3
    x = sc.nodal_positions([1, 1, 1], [1.0] * 3, 3)[0]
    poly = lambda p: 1 + p[:, 0] ** 3 - 2 * p[:, 1] ** 2 * p[:, 2] + p[:, 0] * p[:, 1] * p[:, 2]
    luh = np.repeat(poly(x)[:, None], D, axis=1).reshape(-1)
    idx = (4, 7, 2)
    fine = s.volume_prolongation_cell(luh, 0, 2, idx)
    xf = (np.array(idx)[None, :] + x) / 9.0
    assert np.abs(fine.reshape(-1, D) - poly(xf)[:, None]).max() < 1e-12
    s.close()


def test_batched_prolongation_and_grouped_restriction(exa, torch):
    """Two coarse cells with their 27 children each: one batched prolongation, then one grouped
    restriction per coarse cell (the children in job order), against the reference call by call."""
    rng = np.random.default_rng(3)
    s = exa.Solver(PDE_EULER, 3, 5, npar=0)
    ref = RefAmrLimiter(5, 5, 0)
    nl = s.sizes["luh"]
    coarse = rng.normal(size=(2, nl))
    kids = [(i1, i2, i3) for i3 in range(3) for i2 in range(3) for i1 in range(3)]
    jobs = np.array([[27 * c + k, c, 1, *kids[k]] for c in range(2) for k in range(27)], dtype=np.int32)
    dev = torch.device("cuda")
    cf = torch.tensor(coarse.reshape(-1), device=dev)
    ff = torch.zeros(54 * nl, dtype=torch.float64, device=dev)
    jt = torch.tensor(jobs, device=dev)
    s.amr_volume(exa.AMR_PROLONGATE, ff, cf, jt)
    torch.cuda.synchronize()
    got = ff.cpu().numpy().reshape(54, nl)
    for j, (f, c, L, i1, i2, i3) in enumerate(jobs):
        assert rel(got[f], ref.volume(0, np.zeros(nl), coarse[c], 0, 1, (i1, i2, i3))) < TOL
    # restriction of perturbed children into the coarse cells, groups of 27
    fine = got + 0.01 * rng.normal(size=got.shape)
    ff = torch.tensor(fine.reshape(-1), device=dev)
    acc0 = rng.normal(size=(2, nl))
    cf = torch.tensor(acc0.reshape(-1), device=dev)
    ptr = torch.tensor([0, 27, 54], dtype=torch.int32, device=dev)
    s.amr_volume(exa.AMR_RESTRICT, ff, cf, jt, group_ptr=ptr)
    torch.cuda.synchronize()
    got = cf.cpu().numpy().reshape(2, nl)
    for c in range(2):
        want = acc0[c].copy()
        for j in range(27 * c, 27 * c + 27):
            f, _, L, i1, i2, i3 = jobs[j]
            want = ref.volume(1, want, fine[f], 0, 1, (i1, i2, i3))
        assert rel(got[c], want) < TOL
    assert s.status() == 0
    s.close()


def test_batched_face_prolongation(exa, torch):
    rng = np.random.default_rng(5)
    s = exa.Solver(PDE_ELASTIC, 3, 4, npar=3)
    ref = RefAmrLimiter(4, 9, 3)
    nq, nf = s.sizes["lQhbnd"] // 6, s.sizes["lFhbnd"] // 6
    # coarse cell 0's face 1 (x right) feeds face 0 of nine fine cells
    qc, fc = rng.normal(size=6 * nq), rng.normal(size=6 * nf)
    jobs = np.array([[6 * k + 0, 1, 1, k % 3, k // 3, 0] for k in range(9)], dtype=np.int32)
    dev = torch.device("cuda")
    Qf = torch.zeros(9 * 6 * nq, dtype=torch.float64, device=dev)
    Ff = torch.zeros(9 * 6 * nf, dtype=torch.float64, device=dev)
    s.amr_face(exa.AMR_PROLONGATE, Qf, Ff, torch.tensor(qc, device=dev), torch.tensor(fc, device=dev),
               torch.tensor(jobs, device=dev))
    torch.cuda.synchronize()
    Qg, Fg = Qf.cpu().numpy().reshape(-1, nq), Ff.cpu().numpy().reshape(-1, nf)
    for f, c, L, i1, i2, _ in jobs:
        wq, wf = ref.face(0, np.zeros(nq), np.zeros(nf), qc[c * nq:(c + 1) * nq], fc[c * nf:(c + 1) * nf], 0, 1, (i1, i2))
        assert rel(Qg[f], wq) < TOL and rel(Fg[f], wf) < TOL
    s.close()


def test_bad_jobs_are_skipped_and_flagged(exa, torch):
    """Out-of-range jobs (level difference 0, a subcell index beyond 3^L, a block beyond the array)
    write nothing and set EXA_ST_BAD_JOB; the valid job of the same launch is applied."""
    s = exa.Solver(PDE_EULER, 3, 3, npar=0)
    nl = s.sizes["luh"]
    dev = torch.device("cuda")
    cf = torch.ones(nl, dtype=torch.float64, device=dev)
    ff = torch.full((4 * nl,), 7.0, dtype=torch.float64, device=dev)
    jobs = torch.tensor([[0, 0, 0, 0, 0, 0], [1, 0, 1, 3, 0, 0], [9, 0, 1, 0, 0, 0], [3, 0, 1, 1, 1, 1]],
                        dtype=torch.int32, device=dev)
    s.amr_volume(exa.AMR_PROLONGATE, ff, cf, jobs)
    torch.cuda.synchronize()
    got = ff.cpu().numpy().reshape(4, nl)
    assert np.all(got[:3] == 7.0)
    assert np.abs(got[3] - 1.0).max() < 1e-13
    assert s.status() & exa.ST_BAD_JOB
    assert s.status() == 0  # read and cleared
    s.close()


@pytest.mark.parametrize("cfg", [(PDE_EULER, 3, 5, 0), (PDE_EULER, 3, 5, 1), (PDE_EULER, 5, 5, 0),
                                 (PDE_ELASTIC, 4, 9, 3)], ids=["euler_n3", "euler_n3_p1", "euler_n5", "elastic_n4"])
@pytest.mark.parametrize("ghost", [0, 1, 2])
def test_limiter_kernels_vs_reference(exa, cfg, ghost):
    pde, order, nvar, npar = cfg
    rng = np.random.default_rng(order * 10 + ghost + npar)
    s = exa.Solver(pde, 3, order, npar=npar)
    ref = RefAmrLimiter(order, nvar, npar)
    nl, nm = s.sizes["luh"], s.limiter_patch_size(ghost)
    luh = rng.normal(size=nl)
    # ghost layers are not written: start both from the same filler
    filler = rng.normal(size=nm)
    got = s.project_on_fv_cell(luh, ghost, lim=filler)
    _, want, _, _ = ref.limiter(0, luh, ghost, out=filler)
    assert rel(got, want) < TOL
    lim = rng.normal(size=nm)
    got = s.project_on_dg_cell(lim, ghost)
    _, want, _, _ = ref.limiter(1, lim, ghost, out=np.zeros(nl))
    assert rel(got, want) < TOL
    gmn, gmx = s.local_min_max_cell(luh, nvar)
    _, _, wmn, wmx = ref.limiter(2, luh, ghost, mn=np.zeros(nvar), mx=np.zeros(nvar))
    assert rel(gmn, wmn) < TOL and rel(gmx, wmx) < TOL
    gmn, gmx = s.fv_min_max_cell(lim, ghost, nvar)
    _, _, wmn, wmx = ref.limiter(3, lim, ghost, mn=np.zeros(nvar), mx=np.zeros(nvar))
    assert np.array_equal(gmn, wmn) and np.array_equal(gmx, wmx)
    # discrete maximum principle: neighbour bounds that contain the cell's extrema (even trials) or
    # that one observable leaves by 10% of its range (odd trials)
    lmin, lmax = s.local_min_max_cell(luh, nvar)
    span = lmax - lmin
    verdicts = set()
    for trial in range(8):
        bmin = (lmin - rng.uniform(0.01, 0.2, (6, nvar)) * span)
        bmax = (lmax + rng.uniform(0.01, 0.2, (6, nvar)) * span)
        if trial % 2:
            v = int(rng.integers(nvar))
            if trial % 4 == 1:
                bmin[:, v] = lmin[v] + 0.1 * span[v]
            else:
                bmax[:, v] = lmax[v] - 0.1 * span[v]
        ok, gmn6, gmx6 = s.dmp_cell(luh, nvar, 1e-4, 1e-3, bmin.reshape(-1), bmax.reshape(-1))
        r, _, wmn6, wmx6 = ref.limiter(4, luh, 0, mn=bmin.reshape(-1), mx=bmax.reshape(-1), relax=1e-4, scale=1e-3)
        assert ok == bool(r) == (trial % 2 == 0)
        assert rel(gmn6, wmn6) < TOL and rel(gmx6, wmx6) < TOL
        verdicts.add(ok)
    assert verdicts == {True, False}
    s.close()


def test_limiter_known_answers(exa):
    """The reference's limiter known-answer vectors (limiter_testdata.cpp: N = 3, nVar = 5, P = 7)."""
    g = np.load(os.path.join(GOLD, "limiter_3d.npz"))
    s = exa.Solver(PDE_EULER, 3, 3, npar=0)
    got = s.project_on_fv_cell(g["testFromLuhConversion.luh_in"], 0)
    assert rel(got, g["testFromLuhConversion.lim_out"]) < 1e-13
    got = s.project_on_dg_cell(g["testToLuhConversion.lim_in"], 0)
    assert rel(got, g["testToLuhConversion.luh_out"]) < 1e-13
    s.close()


def test_limiter_batched_matches_per_cell(exa, torch):
    rng = np.random.default_rng(11)
    s = exa.Solver(PDE_EULER, 3, 5, npar=0)
    nl, ghost = s.sizes["luh"], 2
    nm = s.limiter_patch_size(ghost)
    nc = 37
    luh = rng.normal(size=(nc, nl))
    dev = torch.device("cuda")
    L = torch.tensor(luh.reshape(-1), device=dev)
    lim = torch.zeros(nc * nm, dtype=torch.float64, device=dev)
    s.limiter_project_on_fv(L, lim, ghost)
    back = torch.zeros_like(L)
    s.limiter_project_on_dg(lim, back, ghost)
    bmin = torch.tensor(np.repeat(luh.reshape(nc, -1, 5).min(1)[:, None, :], 6, axis=1).reshape(-1) - 0.5, device=dev)
    bmax = torch.tensor(np.repeat(luh.reshape(nc, -1, 5).max(1)[:, None, :], 6, axis=1).reshape(-1) + 0.5, device=dev)
    bmin0, bmax0 = bmin.cpu().numpy().copy(), bmax.cpu().numpy().copy()
    ok = torch.zeros(nc, dtype=torch.uint8, device=dev)
    s.limiter_dmp(L, 5, 1e-4, 1e-3, bmin, bmax, ok)
    torch.cuda.synchronize()
    limh, backh, okh = lim.cpu().numpy().reshape(nc, nm), back.cpu().numpy().reshape(nc, nl), ok.cpu().numpy()
    bmn, bmx = bmin.cpu().numpy().reshape(nc, -1), bmax.cpu().numpy().reshape(nc, -1)
    for c in range(nc):
        assert rel(limh[c], s.project_on_fv_cell(luh[c], ghost)) < TOL
        assert rel(backh[c], s.project_on_dg_cell(limh[c], ghost)) < TOL
        v, m0, m1 = s.dmp_cell(luh[c], 5, 1e-4, 1e-3, bmin0.reshape(nc, -1)[c], bmax0.reshape(nc, -1)[c])
        assert bool(okh[c]) == v
        assert rel(bmn[c], m0) < TOL and rel(bmx[c], m1) < TOL
    # the DG -> FV -> DG round trip is the identity on polynomials of degree N (mass-conserving
    # least squares of exact subcell means)
    assert rel(backh, luh) < 1e-11
    s.close()


# ------------------------------------------------------------------------------------------
# 2D (the reference's 2d/amrRoutines.cpph and the 2D branches of Limiter.cpph)
# ------------------------------------------------------------------------------------------
CONFIGS_2D = [(PDE_EULER, 3, 5, 0), (PDE_EULER, 3, 5, 1), (PDE_SWE, 4, 4, 0)]
IDS_2D = ["euler2d_n3", "euler2d_n3_p1", "swe2d_n4"]


@pytest.mark.parametrize("cfg", CONFIGS_2D, ids=IDS_2D)
@pytest.mark.parametrize("level_delta", [1, 2])
def test_2d_volume_and_face_unknowns_vs_reference(exa, cfg, level_delta):
    pde, order, nvar, npar = cfg
    rng = np.random.default_rng(31 + order + level_delta + npar)
    s = exa.Solver(pde, 2, order, npar=npar)
    ref = RefAmrLimiter(order, nvar, npar, dim=2)
    nl = s.sizes["luh"]
    nq, nf = s.sizes["lQhbnd"] // 4, s.sizes["lFhbnd"] // 4
    for idx in [tuple(int(x) for x in rng.integers(0, 3 ** level_delta, 2)) for _ in range(6)]:
        coarse = rng.normal(size=nl)
        assert rel(s.volume_prolongation_cell(coarse, 0, level_delta, idx),
                   ref.volume(0, np.zeros(nl), coarse, 0, level_delta, idx)) < TOL
        fine, acc = rng.normal(size=nl), rng.normal(size=nl)
        assert rel(s.volume_restriction_cell(acc, fine, 0, level_delta, idx),
                   ref.volume(1, acc, fine, 0, level_delta, idx)) < TOL
        sub = idx[:1]
        qc, fc, qf, ff = rng.normal(size=nq), rng.normal(size=nf), rng.normal(size=nq), rng.normal(size=nf)
        gq, gf = s.face_prolongation_cell(qc, fc, 0, level_delta, sub)
        wq, wf = ref.face(0, np.zeros(nq), np.zeros(nf), qc, fc, 0, level_delta, sub)
        assert rel(gq, wq) < TOL and rel(gf, wf) < TOL
        gq, gf = s.face_restriction_cell(qc, fc, qf, ff, 0, level_delta, sub)
        wq, wf = ref.face(1, qc, fc, qf, ff, 0, level_delta, sub)
        assert rel(gq, wq) < TOL and rel(gf, wf) < TOL
    assert s.status() == 0
    s.close()


@pytest.mark.parametrize("cfg", CONFIGS_2D, ids=IDS_2D)
@pytest.mark.parametrize("ghost", [1, 2])
def test_2d_limiter_kernels_vs_reference(exa, cfg, ghost):
    pde, order, nvar, npar = cfg
    rng = np.random.default_rng(41 + ghost + order + npar)
    s = exa.Solver(pde, 2, order, npar=npar)
    ref = RefAmrLimiter(order, nvar, npar, dim=2)
    nl, nm = s.sizes["luh"], s.limiter_patch_size(ghost)
    luh = rng.normal(size=nl)
    filler = rng.normal(size=nm)
    _, want, _, _ = ref.limiter(0, luh, ghost, out=filler)
    assert rel(s.project_on_fv_cell(luh, ghost, lim=filler), want) < TOL
    lim = rng.normal(size=nm)
    _, want, _, _ = ref.limiter(1, lim, ghost, out=np.zeros(nl))
    assert rel(s.project_on_dg_cell(lim, ghost), want) < TOL
    gmn, gmx = s.local_min_max_cell(luh, nvar)
    _, _, wmn, wmx = ref.limiter(2, luh, ghost, mn=np.zeros(nvar), mx=np.zeros(nvar))
    assert rel(gmn, wmn) < TOL and rel(gmx, wmx) < TOL
    span = gmx - gmn
    for trial in range(4):
        bmin = gmn - rng.uniform(0.01, 0.2, (4, nvar)) * span
        bmax = gmx + rng.uniform(0.01, 0.2, (4, nvar)) * span
        if trial % 2:
            bmax[:, trial % nvar] = gmx[trial % nvar] - 0.1 * span[trial % nvar]
        ok, m0, m1 = s.dmp_cell(luh, nvar, 1e-4, 1e-3, bmin.reshape(-1), bmax.reshape(-1))
        r, _, w0, w1 = ref.limiter(4, luh, 0, mn=bmin.reshape(-1), mx=bmax.reshape(-1), relax=1e-4, scale=1e-3)
        assert ok == bool(r) == (trial % 2 == 0)
        assert rel(m0, w0) < TOL and rel(m1, w1) < TOL
    s.close()


def test_edge_cases_and_argument_checks(exa, torch):
    """Empty batches are no-ops; out-of-range arguments are refused on the host (EXA_ERR_INVALID)
    before any launch; the per-call shims check level differences and subcell indices."""
    s = exa.Solver(PDE_EULER, 3, 3, npar=0)
    nl = s.sizes["luh"]
    dev = torch.device("cuda")
    luh = torch.zeros(nl, dtype=torch.float64, device=dev)
    empty_jobs = torch.zeros((0, 6), dtype=torch.int32, device=dev)
    s.amr_volume(exa.AMR_PROLONGATE, luh, luh, empty_jobs)
    s.amr_volume(exa.AMR_RESTRICT, luh, luh, empty_jobs)
    lim0 = torch.zeros(0, dtype=torch.float64, device=dev)
    luh0 = torch.zeros(0, dtype=torch.float64, device=dev)
    s.limiter_project_on_fv(luh0, lim0, 1)
    s.limiter_project_on_dg(lim0, luh0, 1)
    torch.cuda.synchronize()
    assert s.status() == 0
    one = np.ones(nl)
    with pytest.raises(exa.ExaError):
        s.volume_prolongation_cell(one, 2, 2, (0, 0, 0))           # level difference 0
    with pytest.raises(exa.ExaError):
        s.volume_prolongation_cell(one, 0, 1, (3, 0, 0))           # index beyond 3^1
    with pytest.raises(exa.ExaError):
        s.volume_restriction_cell(one, one, 0, 13, (0, 0, 0))      # beyond 12 levels
    with pytest.raises(exa.ExaError):
        s.project_on_fv_cell(one, 5)                               # ghost layers 0..4
    with pytest.raises(exa.ExaError):
        s.local_min_max_cell(one, 6)                               # more observables than variables
    with pytest.raises(exa.ExaError):
        s.dmp_cell(one, -1, 1e-4, 1e-3, np.zeros(0), np.zeros(0))
    # the flux-only restriction is a face operation
    jobs = torch.tensor([[0, 0, 1, 0, 0, 0]], dtype=torch.int32, device=dev)
    with pytest.raises(exa.ExaError):
        s.amr_volume(exa.AMR_RESTRICT_FLUX, luh, luh, jobs)
    # a group pointer beyond the job list is flagged and the group skipped
    ptr = torch.tensor([0, 2], dtype=torch.int32, device=dev)
    before = luh.clone()
    s.amr_volume(exa.AMR_RESTRICT, luh, luh, jobs, group_ptr=ptr)
    torch.cuda.synchronize()
    assert s.status() & exa.ST_BAD_JOB
    assert torch.equal(luh, before)
    # the DMP of a cell with no observables holds
    ok, _, _ = s.dmp_cell(one, 0, 1e-4, 1e-3, np.zeros(0), np.zeros(0))
    assert ok
    s.close()
