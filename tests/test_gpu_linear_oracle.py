"""The GPU path (flux-form functors, nonlinear Picard predictor, Rusanov) against the second oracle:
the reference's linear generic kernels with the PDE terms of its own linear applications
(oracle/_ref, see test_linear_oracle.py). Plane waves: the same time steps, the same error against
the exact wave, and a difference far below that error. Point source: the same total moment.
"""
import os
import sys

import numpy as np
import pytest

from conftest import REPO

sys.path.insert(0, os.path.join(REPO, "exahype-engine_b200"))
import exa_scenarios as sc  # noqa: E402
from pyoracle import RefLinear  # noqa: E402
from test_linear_oracle import ACOUSTIC_MAP, acoustic_plane_wave, elastic_plane_wave, l2  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def exa():
    import exa_aderdg
    return exa_aderdg


def gpu_run(exa, pde, order, ncell, luh0, nsteps, src=None):
    s = exa.Solver(pde, 3, order, npar=exa.NPAR[pde])
    p = exa.Patch(s, [dict(ncell=ncell, size=[1.0, 1.0, 1.0], bc=0)])
    if src is not None:
        p.set_point_source(src[:3], src[3], src[4], src[5], src[6], int(src[7]))
    p.set_solution(luh0)
    p.step(nsteps)
    out, t = p.get_solution(), p.time()[0][0]
    assert p.status() == 0
    p.close()
    return out, t


@pytest.mark.parametrize("order", [3, 4])
def test_gpu_elastic_plane_wave_vs_linear_reference(exa, order):
    nc, nsteps = 4, 24
    x = sc.nodal_positions([nc] * 3, [1.0] * 3, order)
    q0 = elastic_plane_wave(x, 0.0).reshape(-1)
    a = q0.copy()
    t_ref, _ = RefLinear("elastic", order).run(a, [nc] * 3, [1.0] * 3, nsteps)
    got, t = gpu_run(exa, exa.PDE_ELASTIC, order, (nc, nc, nc), q0, nsteps)
    assert abs(t - t_ref) <= 1e-13 * t_ref
    sh = (-1, (order + 1) ** 3, 12)
    ra, rg = a.reshape(sh)[..., :9], got.reshape(sh)[..., :9]
    ex = elastic_plane_wave(x, t).reshape(sh)[..., :9]
    err_ref, err_gpu = l2(ra - ex, order), l2(rg - ex, order)
    assert abs(err_gpu - err_ref) <= 1e-2 * err_ref
    assert l2(ra - rg, order) <= 1e-3 * err_ref


def test_gpu_acoustic_plane_wave_vs_linear_reference(exa):
    order, nc, nsteps = 4, 4, 20
    x = sc.nodal_positions([nc] * 3, [1.0] * 3, order)
    q = acoustic_plane_wave(x, 0.0)
    a = (q[..., :4] @ ACOUSTIC_MAP).reshape(-1).copy()
    t_ref, _ = RefLinear("acoustic", order).run(a, [nc] * 3, [1.0] * 3, nsteps)
    got, t = gpu_run(exa, exa.PDE_ACOUSTIC, order, (nc, nc, nc), q.reshape(-1), nsteps)
    assert abs(t - t_ref) <= 1e-13 * t_ref
    ra = a.reshape(-1, (order + 1) ** 3, 4) @ ACOUSTIC_MAP
    rg = got.reshape(-1, (order + 1) ** 3, 6)[..., :4]
    ex = acoustic_plane_wave(x, t)[..., :4]
    err_ref, err_gpu = l2(ra - ex, order), l2(rg - ex, order)
    assert abs(err_gpu - err_ref) <= 1e-2 * err_ref
    assert l2(ra - rg, order) <= 1e-3 * err_ref


def test_gpu_point_source_total_moment_vs_delta_distribution(exa):
    """Same case as the CPU test: the moment of s13 injected by the GPU's regularised source
    (amplitude -A) and by the reference's delta distribution (amplitude A, subtracted there)."""
    order, nc, A, nsteps = 3, 6, 1.0, 80
    dx = 1.0 / nc
    x = sc.nodal_positions([nc] * 3, [1.0] * 3, order)
    q0 = np.zeros(x.shape[:-1] + (12,))
    q0[..., 9], q0[..., 10], q0[..., 11] = 2.0, 3.0, 1.5
    q0 = q0.reshape(-1)
    src = (0.53, 0.47, 0.51, 4.0, 0.3, A, 0.5 * dx, 7.0)
    a = q0.copy()
    t_ref, _ = RefLinear("elastic", order, source=src).run(a, [nc] * 3, [1.0] * 3, nsteps)
    got, t = gpu_run(exa, exa.PDE_ELASTIC, order, (nc, nc, nc), q0, nsteps, src=src[:5] + (-A,) + src[6:])
    assert abs(t - t_ref) <= 1e-13 * t_ref
    w = sc.gl_weights(order)
    wn = (w[:, None, None] * w[None, :, None] * w[None, None, :]).reshape(-1)
    Ia = (a.reshape(-1, wn.size, 12)[..., 7] * wn).sum() * dx ** 3
    Ig = (got.reshape(-1, wn.size, 12)[..., 7] * wn).sum() * dx ** 3
    assert abs(Ia) > 1e-5
    assert abs(Ig - Ia) <= 1e-3 * abs(Ia)
