"""The allocation-free CFL entry point, exa_stable_time_step_size_noalloc.

It serves callers that cannot call cudaMalloc (device memory owned by another runtime, or a step
loop that must not pay an allocation's synchronisation). It keeps its scratch in a file-scope
device array of the library instead. This test drives it through the C ABI on the GPU and checks
it against the allocating entry point, exa_stable_time_step_size, on two calls in a row. The
second call runs on a state with a larger time step, so a stale minimum left in the shared array
would show. The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-15  # same kernel arithmetic: the per-cell values are expected to be bit-identical


def _cells(rng, ncells, nd, scale):
    rho = 1.0 + 0.05 * rng.uniform(-1, 1, (ncells, nd))
    u = scale * rng.uniform(-1, 1, (ncells, nd, 3))
    p = 1.0 + 0.05 * rng.uniform(-1, 1, (ncells, nd))
    Q = np.zeros((ncells, nd, 5))
    Q[..., 0] = rho
    Q[..., 1:4] = rho[..., None] * u
    Q[..., 4] = p / 0.4 + 0.5 * rho * (u ** 2).sum(-1)
    return Q.reshape(-1)


def test_noalloc_cfl_matches_allocating_entry_point():
    import torch
    import exa_aderdg as exa

    lib = exa.load_library()
    f = lib.exa_stable_time_step_size_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(exa._Config), ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                  ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    order, nd = 5, 216
    cfg = exa._Config(3, order, 0, exa.PDE_EULER, 0.9, 0.0, 0, exa.PREC_FP64)
    solver = exa.Solver(exa.PDE_EULER, 3, order)
    dx3 = (ctypes.c_double * 3)(1.0 / 81, 1.0 / 81, 1.0 / 81)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(4)
    previous = None
    for call, (ncells, speed) in enumerate(((3001, 0.6), (1777, 0.1))):
        luh = torch.from_numpy(_cells(rng, ncells, nd, speed)).cuda()
        want_cells = torch.zeros(ncells, dtype=torch.float64, device="cuda")
        want_min = solver.stable_time_step_size(luh, [1.0 / 81] * 3, cell_dt=want_cells)
        got_cells = torch.full((ncells,), -1.0, dtype=torch.float64, device="cuda")
        got_min = ctypes.c_double(-1.0)
        rc = f(ctypes.byref(cfg), ncells, ctypes.c_void_p(luh.data_ptr()), dx3, ctypes.c_void_p(got_cells.data_ptr()),
               ctypes.byref(got_min), stream)
        assert rc == 0, lib.exa_last_error()
        torch.cuda.synchronize()
        w, g = want_cells.cpu().numpy(), got_cells.cpu().numpy()
        assert np.all(w > 0)
        assert np.max(np.abs(g - w) / w) <= TOL
        assert abs(got_min.value - want_min) <= TOL * want_min
        assert got_min.value == w.min()
        if previous is not None:
            assert got_min.value > previous  # the slower state has the larger step: no stale minimum
        previous = got_min.value


def test_noalloc_cfl_rejects_oversized_batches():
    import torch
    import exa_aderdg as exa

    lib = exa.load_library()
    f = lib.exa_stable_time_step_size_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(exa._Config), ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                  ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    cfg = exa._Config(3, 5, 0, exa.PDE_EULER, 0.9, 0.0, 0, exa.PREC_FP64)
    dx3 = (ctypes.c_double * 3)(0.1, 0.1, 0.1)
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = ctypes.c_double(0.0)
    rc = f(ctypes.byref(cfg), 1048576 + 1, ctypes.c_void_p(dummy.data_ptr()), dx3, None, ctypes.byref(out), None)
    assert rc == 1  # EXA_ERR_INVALID, before any device work
    assert b"EXA_NOALLOC_MAX_CELLS" in lib.exa_last_error()


def _noalloc(lib, exa):
    f = lib.exa_stable_time_step_size_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.POINTER(exa._Config), ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                  ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    return f


def test_noalloc_cfl_2d_swe_without_minimum_and_empty_batch():
    """A 2D shallow-water configuration; a call that asks only for the per-cell values (no
    minimum: no synchronisation, no status read); and an empty batch, whose minimum is +inf."""
    import torch
    import exa_aderdg as exa

    lib = exa.load_library()
    f = _noalloc(lib, exa)
    order, nd, ncells = 4, 25, 513
    cfg = exa._Config(2, order, 0, exa.PDE_SWE, 0.9, 0.0, 0, exa.PREC_FP64)
    solver = exa.Solver(exa.PDE_SWE, 2, order)
    rng = np.random.default_rng(12)
    Q = np.zeros((ncells, nd, 4))
    Q[..., 0] = 1.0 + 0.5 * rng.uniform(0, 1, (ncells, nd))
    Q[..., 1:3] = 0.3 * rng.normal(size=(ncells, nd, 2))
    Q[..., 3] = 0.1 * rng.uniform(0, 1, (ncells, nd))
    luh = torch.from_numpy(Q.reshape(-1)).cuda()
    dx = [1.0 / 40, 1.0 / 30]
    dx3 = (ctypes.c_double * 3)(dx[0], dx[1], 1.0)
    want = torch.zeros(ncells, dtype=torch.float64, device="cuda")
    want_min = solver.stable_time_step_size(luh, dx, cell_dt=want)
    got = torch.full((ncells,), -1.0, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        rc = f(ctypes.byref(cfg), ncells, ctypes.c_void_p(luh.data_ptr()), dx3, ctypes.c_void_p(got.data_ptr()),
               None, stream)
        assert rc == 0, lib.exa_last_error()
        torch.cuda.synchronize()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        assert np.max(np.abs(g - w) / w) <= TOL
        assert g.min() == want_min
        got.fill_(-1.0)
    out = ctypes.c_double(0.0)
    rc = f(ctypes.byref(cfg), 0, None, dx3, None, ctypes.byref(out), stream)
    assert rc == 0, lib.exa_last_error()
    assert out.value == float("inf")


def test_noalloc_cfl_reports_a_nonfinite_cell_then_recovers():
    """One NaN entry in cell 57: the call returns EXA_ERR_NUMERICS (4); the status word in the shared
    array is reset by the next call, which succeeds on a clean state."""
    import torch
    import exa_aderdg as exa

    lib = exa.load_library()
    f = _noalloc(lib, exa)
    order, nd, ncells = 3, 64, 200
    cfg = exa._Config(3, order, 0, exa.PDE_EULER, 0.9, 0.0, 0, exa.PREC_FP64)
    rng = np.random.default_rng(13)
    clean = _cells(rng, ncells, nd, 0.3)
    bad = clean.copy()
    bad[57 * nd * 5 + 3] = np.nan
    dx3 = (ctypes.c_double * 3)(0.1, 0.1, 0.1)
    out = ctypes.c_double(0.0)
    cells = torch.zeros(ncells, dtype=torch.float64, device="cuda")
    for state, want_rc in ((bad, 4), (clean, 0)):
        luh = torch.from_numpy(state).cuda()
        rc = f(ctypes.byref(cfg), ncells, ctypes.c_void_p(luh.data_ptr()), dx3, ctypes.c_void_p(cells.data_ptr()),
               ctypes.byref(out), None)
        torch.cuda.synchronize()
        assert rc == want_rc, lib.exa_last_error()
        c = cells.cpu().numpy()
        # the non-finite node counts as +inf, so cell 57 keeps the minimum of its other nodes
        assert np.isfinite(c).all() and out.value == c.min()
