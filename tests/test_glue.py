"""Generated solver glue: exahype-engine_b200/glue/generate_glue.py emits Abstract<Solver>.{h,cpp}
for an application specification, the counterpart of the reference toolkit's generated
Abstract<App>Solver_ADERDG (AbstractGenericADERDGSolverImplementation.template:104-361) on the B200
C ABI. tests/glue/euler_app.cpp derives the application's solver class from it (host-side
reflective boundaryValues); the build step compiles both into tests/glue/libglue_euler.so.

The GPU tests drive the glue the way the reference's engine does -- per cell and per face, on host
arrays -- and check every method and one whole engine-ordered time step against the oracle.
"""
import ctypes
import json
import os
import sys

import numpy as np
import pytest

from conftest import REPO

GLUE_LIB = os.path.join(REPO, "tests", "glue", "libglue_euler.so")
TOL = 1e-12


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(1e-300, np.max(np.abs(b))))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_generator_emits_the_solver_constants(tmp_path):
    sys.path.insert(0, os.path.join(REPO, "exahype-engine_b200", "glue"))
    import generate_glue
    with open(os.path.join(REPO, "tests", "glue", "euler_glue_spec.json")) as f:
        spec = json.load(f)
    spec.update(order=5, solver="MySolver", project="App")
    h, cpp = generate_glue.generate(spec, str(tmp_path))
    text = open(h).read()
    assert "class AbstractMySolver" in text and "static constexpr int Order = 5;" in text
    assert "static constexpr double PNPM = 0.045;" in text  # the toolkit's table for order 5
    assert "exa_solver_create" in open(cpp).read()
    with pytest.raises(ValueError):
        generate_glue.generate(dict(spec, dimension=4), str(tmp_path))


def _glue():
    import exa_aderdg as exa
    exa.load_library()
    if not os.path.exists(GLUE_LIB):
        pytest.skip("the glue example was not built")
    lib = ctypes.CDLL(GLUE_LIB)
    vp, d, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
    lib.glue_create.restype = vp
    lib.glue_destroy.argtypes = [vp]
    lib.glue_predictor.argtypes = [vp, vp, vp, vp, vp, vp, vp, d, d, i]
    lib.glue_predictor.restype = i
    lib.glue_riemann.argtypes = [vp, vp, vp, vp, vp, d, d, vp, i]
    lib.glue_boundary.argtypes = [vp, vp, vp, vp, vp, d, d, i, i]
    lib.glue_face.argtypes = [vp, vp, vp, i, i, vp, i, vp, d, i]
    lib.glue_adjust.argtypes = [vp, vp, vp, vp, d, d]
    lib.glue_volume_prolong.argtypes = [vp, vp, vp, i, i, vp]
    lib.glue_volume_restrict.argtypes = [vp, vp, vp, i, i, vp]
    lib.glue_face_prolong.argtypes = [vp, vp, vp, vp, vp, i, i, vp]
    lib.glue_update.argtypes = [vp, vp, vp, vp, d]
    lib.glue_dt.argtypes = [vp, vp, vp]
    lib.glue_dt.restype = d
    lib.glue_grid.argtypes = [vp, vp, vp, vp, vp, i, vp]
    lib.glue_grid.restype = i
    return lib


def test_glue_library_exports_the_engine_entry_points():
    lib = _glue()
    for name in ("glue_create", "glue_predictor", "glue_riemann", "glue_boundary", "glue_face", "glue_update",
                 "glue_dt", "glue_grid", "glue_adjust", "glue_volume_prolong", "glue_volume_restrict",
                 "glue_face_prolong"):
        assert hasattr(lib, name)


def euler_cells(rng, ncells, nd, amp=0.05):
    rho = 1.0 + amp * rng.uniform(-1, 1, (ncells, nd))
    u = 0.3 * rng.uniform(-1, 1, (ncells, nd, 3))
    p = 1.0 + amp * rng.uniform(-1, 1, (ncells, nd))
    Q = np.zeros((ncells, nd, 5))
    Q[..., 0] = rho
    Q[..., 1:4] = rho[..., None] * u
    Q[..., 4] = p / 0.4 + 0.5 * rho * (u ** 2).sum(-1)
    return Q


@pytest.mark.gpu
def test_glue_methods_vs_oracle():
    from pyoracle import Oracle
    lib = _glue()
    h = lib.glue_create()
    o = Oracle(3, 3)
    rng = np.random.default_rng(41)
    n, nd, nf = 4, 64, 16
    dx = np.array([0.05, 0.05, 0.05])
    luh = euler_cells(rng, 1, nd).reshape(-1)
    dt = lib.glue_dt(h, _p(luh), _p(dx))
    assert abs(dt - o.dt(luh, dx)) <= 1e-15 * dt
    # fused predictor + volume integral
    lduh, qhb, fhb = np.zeros(nd * 5), np.zeros(6 * nf * 5), np.zeros(6 * nf * 5)
    centre = np.array([0.3, 0.4, 0.5])
    lu = luh.copy()
    it = lib.glue_predictor(h, _p(lduh), _p(qhb), _p(fhb), _p(lu), _p(centre), _p(dx), 0.0, dt, 1)
    r = o.predictor(luh, dx, dt, centre=centre)
    assert it == r["ret"]
    assert rel(qhb, r["lQhbnd"]) < TOL and rel(fhb, r["lFhbnd"]) < TOL
    assert rel(lduh, o.volume(r["lFhi"], dx)) < TOL
    # the addVolumeIntegralResultToUpdate = false form updates luh itself
    lu2 = luh.copy()
    lib.glue_predictor(h, _p(np.zeros(nd * 5)), _p(qhb), _p(fhb), _p(lu2), _p(centre), _p(dx), 0.0, dt, 0)
    assert rel(lu2, o.update(luh, o.volume(r["lFhi"], dx), dt)) < TOL
    # Riemann on a random face, face integral, update
    QL, QR = euler_cells(rng, 1, nf).reshape(-1), euler_cells(rng, 1, nf).reshape(-1)
    FL, FR = rng.normal(size=nf * 5), rng.normal(size=nf * 5)
    a, b = FL.copy(), FR.copy()
    lib.glue_riemann(h, _p(a), _p(b), _p(QL), _p(QR), 0.0, dt, _p(dx), 2)
    ra, rb = o.riemann(FL, FR, QL, QR, dx, 2)
    assert rel(a, ra) < TOL and rel(b, rb) < TOL
    du = rng.normal(size=nd * 5)
    no_sub = np.zeros(2, dtype=np.int32)
    for d in range(3):
        for ori in (0, 1):
            x = du.copy()
            lib.glue_face(h, _p(x), _p(FL), d, ori, _p(no_sub), 0, _p(dx), dt, 1)
            assert rel(x, o.face(du, FL, d, ori, dx)) < 1e-14
    # addToUpdate = false: the face integral goes straight into the solution
    x = luh.copy()
    lib.glue_face(h, _p(x), _p(FL), 1, 0, _p(no_sub), 0, _p(dx), dt, 0)
    assert rel(x, o.update(luh, o.face(np.zeros(nd * 5), FL, 1, 0, dx), dt)) < 1e-14
    out = luh.copy()
    lib.glue_update(h, _p(out), _p(luh), _p(du), dt)
    assert rel(out, o.update(luh, du, dt)) < 1e-14
    # boundaryConditions: the application's reflective wall, then Rusanov with the outer state outside
    for d in range(3):
        for ori in (0, 1):
            fin = FL.copy()
            lib.glue_boundary(h, _p(fin), _p(QL), _p(centre), _p(dx), 0.0, dt, d, ori)
            qg = QL.reshape(nf, 5).copy()
            qg[:, 1 + d] *= -1
            fg = np.stack([o.flux(q)[d] for q in qg]).reshape(-1)
            if ori == 0:
                _, want = o.riemann(fg, FL, qg.reshape(-1), QL, dx, d)
            else:
                want, _ = o.riemann(FL, fg, QL, qg.reshape(-1), dx, d)
            assert rel(fin, want) < TOL
    lib.glue_destroy(h)


@pytest.mark.gpu
def test_glue_engine_loop_and_uniform_grid_vs_oracle():
    """One time step of a 3x2x2 periodic grid in the reference engine's order through the glue
    (stableTimeStepSize per cell -> fused predictor per cell -> riemannSolver per face ->
    faceIntegral per face -> addUpdateToSolution per cell), and three steps of the batched
    updateUniformGrid, against the oracle."""
    from pyoracle import Oracle
    lib = _glue()
    h = lib.glue_create()
    rng = np.random.default_rng(42)
    ncell = (3, 2, 2)
    nc, nd, nf = 12, 64, 16
    size = np.array([0.6, 0.4, 0.4])
    dx = size / np.array(ncell)
    luh0 = euler_cells(rng, nc, nd, amp=0.03).reshape(nc, nd * 5)
    ref = luh0.reshape(-1).copy()
    Oracle(3, 3).run(ref, ncell, list(size), 1)
    dt = min(lib.glue_dt(h, _p(np.ascontiguousarray(luh0[c])), _p(dx)) for c in range(nc))
    lduh = np.zeros((nc, nd * 5))
    qhb = np.zeros((nc, 6, nf * 5))
    fhb = np.zeros((nc, 6, nf * 5))
    luh = luh0.copy()
    idx = lambda x, y, z: (z * ncell[1] + y) * ncell[0] + x
    for c in range(nc):
        x, y, z = c % 3, (c // 3) % 2, c // 6
        centre = (np.array([x, y, z]) + 0.5) * dx
        row, l, q, f = luh[c].copy(), np.zeros(nd * 5), np.zeros(6 * nf * 5), np.zeros(6 * nf * 5)
        lib.glue_predictor(h, _p(l), _p(q), _p(f), _p(row), _p(centre), _p(dx), 0.0, dt, 1)
        lduh[c], qhb[c], fhb[c] = l, q.reshape(6, -1), f.reshape(6, -1)
    for c in range(nc):
        x, y, z = c % 3, (c // 3) % 2, c // 6
        for d in range(3):
            j = [x, y, z]
            j[d] = (j[d] + 1) % ncell[d]
            c2 = idx(*j)
            FL, FR = fhb[c, 2 * d + 1].copy(), fhb[c2, 2 * d].copy()
            lib.glue_riemann(h, _p(FL), _p(FR), _p(np.ascontiguousarray(qhb[c, 2 * d + 1])),
                             _p(np.ascontiguousarray(qhb[c2, 2 * d])), 0.0, dt, _p(dx), d)
            fhb[c, 2 * d + 1], fhb[c2, 2 * d] = FL, FR
    for c in range(nc):
        l = lduh[c].copy()
        for d in range(3):
            for ori in (0, 1):
                lib.glue_face(h, _p(l), _p(np.ascontiguousarray(fhb[c, 2 * d + ori])), d, ori,
                                  _p(np.zeros(2, dtype=np.int32)), 0, _p(dx), dt, 1)
        out = luh[c].copy()
        lib.glue_update(h, _p(out), _p(np.ascontiguousarray(luh[c])), _p(l), dt)
        luh[c] = out
    assert rel(luh.reshape(-1), ref) < TOL
    # the batched path: three steps of the whole grid
    grid = luh0.reshape(-1).copy()
    t = ctypes.c_double(0.0)
    nce = np.array(ncell, dtype=np.int32)
    off = np.zeros(3)
    assert lib.glue_grid(h, _p(grid), _p(nce), _p(off), _p(size), 3, ctypes.byref(t)) == 0
    ref3 = luh0.reshape(-1).copy()
    t3, _, _ = Oracle(3, 3).run(ref3, ncell, list(size), 3)
    assert rel(grid, ref3) < TOL and abs(t.value - t3) <= 1e-13 * t3
    lib.glue_destroy(h)


@pytest.mark.gpu
def test_glue_mesh_levels_adjust_and_coarse_face_integral_vs_reference():
    """The glue's mesh-level methods (volumeUnknownsProlongation / Restriction,
    faceUnknownsProlongation) and faceIntegral on the face of a coarser neighbour (levelDelta > 0:
    faceUnknownsRestriction of the flux, then the face integral with the coarse cell size) against
    the reference's own kernels (oracle/_ref), and adjustSolution with the application's
    adjustPointSolution against its numpy restatement."""
    from pyoracle import Oracle, RefAmrLimiter
    if not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libexaref_amrlim3d.so")):
        pytest.skip("oracle/_ref not built")
    lib = _glue()
    h = lib.glue_create()
    o, ref = Oracle(3, 3), RefAmrLimiter(3, 5, 0)
    rng = np.random.default_rng(43)
    nd, nf = 64, 16
    # adjustSolution: rho = 1 + 0.1 sin(2 pi (x + 2y + 3z)) at the nodes, z slowest
    centre, size = np.array([0.3, 0.4, 0.5]), np.array([0.1, 0.2, 0.05])
    luh = np.zeros(nd * 5)
    lib.glue_adjust(h, _p(luh), _p(centre), _p(size), 0.0, 0.0)
    nodes = o.tables()["nodes"]
    z, y, x = np.meshgrid(nodes, nodes, nodes, indexing="ij")
    X = np.stack([centre[0] + size[0] * (x - 0.5), centre[1] + size[1] * (y - 0.5),
                  centre[2] + size[2] * (z - 0.5)], -1).reshape(-1, 3)
    rho = 1.0 + 0.1 * np.sin(2.0 * np.pi * (X[:, 0] + 2.0 * X[:, 1] + 3.0 * X[:, 2]))
    assert np.max(np.abs(luh.reshape(nd, 5)[:, 0] - rho)) <= 1e-15
    assert np.max(np.abs(luh.reshape(nd, 5)[:, 4] - (2.5 + 0.5 * rho * 0.14))) <= 1e-14
    # volume prolongation / restriction over two levels
    coarse = euler_cells(rng, 1, nd).reshape(-1)
    sub = np.array([2, 0, 1], dtype=np.int32)
    fine = np.zeros(nd * 5)
    lib.glue_volume_prolong(h, _p(fine), _p(coarse), 1, 3, _p(sub))
    assert rel(fine, ref.volume(0, np.zeros(nd * 5), coarse, 1, 3, sub)) < TOL
    acc = coarse.copy()
    lib.glue_volume_restrict(h, _p(acc), _p(fine), 1, 3, _p(sub))
    assert rel(acc, ref.volume(1, coarse, fine, 1, 3, sub)) < TOL
    # face prolongation
    qc, fc = euler_cells(rng, 1, nf).reshape(-1), rng.normal(size=nf * 5)
    sf = np.array([1, 2], dtype=np.int32)
    qf, ff = np.zeros(nf * 5), np.zeros(nf * 5)
    lib.glue_face_prolong(h, _p(qf), _p(ff), _p(qc), _p(fc), 0, 1, _p(sf))
    wq, wf = ref.face(0, np.zeros(nf * 5), np.zeros(nf * 5), qc, fc, 0, 1, sf)
    assert rel(qf, wq) < TOL and rel(ff, wf) < TOL
    # faceIntegral from a fine face into the coarse neighbour's update
    dx = np.array([0.05, 0.05, 0.05])
    du = rng.normal(size=nd * 5)
    fine_flux = rng.normal(size=nf * 5)
    for delta, sfi in ((1, [2, 1]), (2, [5, 7])):
        sfi = np.array(sfi, dtype=np.int32)
        out = du.copy()
        lib.glue_face(h, _p(out), _p(fine_flux), 2, 1, _p(sfi), delta, _p(dx), 1e-3, 1)
        _, cflux = ref.face(2, np.zeros(nf * 5), np.zeros(nf * 5), np.zeros(nf * 5), fine_flux, 0, delta, sfi)
        assert rel(out, o.face(du, cflux, 2, 1, dx * 3 ** delta)) < 1e-13
    lib.glue_destroy(h)
