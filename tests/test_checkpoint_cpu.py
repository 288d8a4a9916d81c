"""Host logic of the adjoint driver, no GPU: the binomial checkpointing schedule
(exa_checkpoint_schedule, C ABI) and the receiver interpolation."""
from math import comb

import numpy as np
import pytest


def _simulate(exa, sched, steps, snaps):
    slots, cur, adj, fwd = {}, 0, [], 0
    for act, a, b in sched:
        if act == exa.CK_STORE:
            assert cur == b
            slots[a] = b
        elif act == exa.CK_RESTORE:
            assert slots[a] == b
            cur = b
        elif act == exa.CK_ADVANCE:
            assert cur == a and b > a
            fwd += b - a
            cur = b
        else:
            assert act == exa.CK_ADJOINT and cur == a
            adj.append(a)
    assert adj == list(range(steps - 1, -1, -1))
    assert max(slots) < snaps
    return fwd


def _binomial_optimum(steps, snaps):
    """Griewank's minimal recomputation count with `snaps` stored states (initial included)."""
    if snaps == 1:
        return steps * (steps - 1) // 2
    s = snaps
    r = 0
    while comb(s + r, s) < steps:
        r += 1
    if r == 0:
        return 0
    return r * steps - comb(s + r, s + 1)


@pytest.mark.parametrize("steps,snaps", [(1, 1), (2, 1), (7, 1), (5, 2), (10, 3), (37, 4), (100, 2), (300, 20),
                                         (300, 5), (64, 64), (500, 7)])
def test_schedule_is_valid_and_binomial(steps, snaps):
    import exa_aderdg as exa
    sched, fw = exa.checkpoint_schedule(steps, snaps)
    assert sched[0] == (exa.CK_STORE, 0, 0)
    assert _simulate(exa, sched, steps, snaps) == fw
    assert fw == _binomial_optimum(steps, snaps)


def test_schedule_rejects_bad_arguments():
    import exa_aderdg as exa
    for steps, snaps in ((0, 3), (5, 0)):
        with pytest.raises(exa.ExaError):
            exa.checkpoint_schedule(steps, snaps)


@pytest.mark.parametrize("order", [2, 3, 4, 5])
def test_receiver_interpolation_is_exact_for_polynomials(order):
    """rec(u) of the nodal interpolant of a degree-`order` polynomial equals the polynomial."""
    from exa_adjoint import receiver_operator
    from exa_scenarios import nodal_positions
    rng = np.random.default_rng(order)
    ncell, size = (3, 2, 4), [1.0, 0.8, 1.2]
    coef = rng.normal(size=(order + 1, 3))

    def f(x):
        return sum(coef[k, 0] * x[..., 0] ** k + coef[k, 1] * x[..., 1] ** k + coef[k, 2] * x[..., 2] ** k
                   for k in range(order + 1))
    xn = nodal_positions(ncell, size, order)          # [cells][nodes][3]
    u = f(xn)
    pts = rng.uniform(0.0, 1.0, (20, 3)) * np.asarray(size)
    cells, w = receiver_operator(ncell, size, order, pts)
    got = (w * u[cells]).sum(-1)
    assert np.max(np.abs(got - f(pts))) < 1e-11
