"""Run-to-run determinism of the device step: the same state stepped twice gives the same bits.

The Picard loop stops a cell when the squared residual of its iterate drops below 1e-14. The
residual is a sum over the cell's nodes, and a cell spans several warps; its partials are added in
warp order, so that a cell at the tolerance takes the same number of sweeps in every run. Two
patches stepped from the same state must therefore agree bit for bit, and so must the two launch
forms of the predictor (one cell group per CTA, persistent CTAs) and the two forms of the
Riemann and update kernels, which the launch tuner may pick differently in different processes.
"""
import numpy as np
import pytest

from conftest import REPO  # noqa: F401  (path setup)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def exa():
    import exa_aderdg
    return exa_aderdg


def run_swe(exa, steps, pred_variant=-1, upd_variant=-1):
    import exa_scenarios as sc
    specs, states = sc.swe_batched(ngrids=512)
    s = exa.Solver(exa.PDE_SWE, 2, 4)
    s.predictor_variant = pred_variant
    s.set_update_variant(upd_variant)
    p = exa.Patch(s, specs)
    p.set_solution(np.concatenate(states))
    p.step(steps)
    out = p.get_solution()
    assert p.status() == 0
    p.close()
    return out


def run_euler(exa, steps, pred_variant=-1, upd_variant=-1):
    import exa_scenarios as sc
    order, n = 5, 27
    ncell, size = (n, n, n), [1.0, 1.0, 1.0]
    luh = sc.EntropyWave(3, 0).state(sc.nodal_positions(ncell, size, order)).reshape(-1)
    s = exa.Solver(exa.PDE_EULER, 3, order)
    s.predictor_variant = pred_variant
    s.set_update_variant(upd_variant)
    p = exa.Patch(s, [dict(ncell=ncell, size=size)])
    p.set_solution(luh)
    p.step(steps)
    out = p.get_solution()
    assert p.status() == 0
    p.close()
    return out


def test_swe_512_grids_twice_bitwise(exa):
    # 3.4 M cells at a mean of about 3 sweeps: many cells end within rounding of the tolerance
    a = run_swe(exa, 10, pred_variant=0, upd_variant=1)
    b = run_swe(exa, 10, pred_variant=0, upd_variant=1)
    assert np.array_equal(a, b), np.max(np.abs(a - b))


def test_euler_launch_forms_bitwise(exa):
    ref = run_euler(exa, 6, pred_variant=0, upd_variant=0)
    for pv, uv in ((0, 0), (1, 0), (0, 1), (1, 1)):
        got = run_euler(exa, 6, pred_variant=pv, upd_variant=uv)
        assert np.array_equal(got, ref), (pv, uv, np.max(np.abs(got - ref)))


def test_swe_launch_forms_bitwise(exa):
    ref = run_swe(exa, 4, pred_variant=0, upd_variant=0)
    for pv, uv in ((1, 0), (0, 1), (1, 1)):
        got = run_swe(exa, 4, pred_variant=pv, upd_variant=uv)
        assert np.array_equal(got, ref), (pv, uv, np.max(np.abs(got - ref)))
