"""Second oracle for the acoustic and elastic systems: the reference's LINEAR generic kernels
(Cauchy-Kowalewski predictor 3d/spaceTimePredictorLinear.cpph, linear Riemann solver
3d/riemannSolverLinear.cpph, point sources by 3d/deltaDistribution.cpph) with the PDE terms of the
reference's own linear applications (ApplicationExamples/Linear/ElasticWave3D,
ApplicationExamples/AcousticWave/acousticwaveCPP), compiled into oracle/_ref.

That scheme shares nothing with the nonlinear path but the basis: a different predictor, a
fluctuation-form Riemann solver, a material-matrix formulation of the PDE and a delta-distribution
point source. So it checks the physics of the flux-form functors (exa_pde.cuh, restated in
oracle/oracle.c) rather than the kernels:
  * the PDE terms themselves, pointwise, to rounding;
  * plane waves: both schemes against the exact solution and against each other (their difference
    is far below either's discretisation error) and their convergence order;
  * the point source: the total moment injected into the domain.
CPU only; the GPU path runs the same cases in test_gpu_linear_oracle.py.
"""
import os
import sys

import numpy as np
import pytest

from conftest import REPO

sys.path.insert(0, os.path.join(REPO, "exahype-engine_b200"))
import exa_scenarios as sc  # noqa: E402
from pyoracle import PDE_ACOUSTIC, PDE_ELASTIC, Oracle, RefLinear  # noqa: E402

ref_missing = not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libexaref3d.so"))
pytestmark = pytest.mark.skipif(ref_missing, reason="oracle/_ref not built")

# flux-form acoustic velocity = minus the acoustic application's velocity (unit density and speed)
ACOUSTIC_MAP = np.diag([1.0, -1.0, -1.0, -1.0])


def elastic_plane_wave(x, t, rho=2.0, cp=3.0, cs=1.5, amp=(1e-2, 5e-3)):
    """P wave (polarised along n) plus S wave (along m, m.n = 0) travelling along n = (1,1,1)/sqrt(3),
    periodic on the unit cube: v = n f_p + m f_s, sigma = -(lam I + 2 mu n n) f_p / cp
    - mu (n m + m n) f_s / cs, f(s) = a sin(2 pi sqrt(3) s)."""
    n = np.ones(3) / np.sqrt(3)
    m = np.array([1.0, -1.0, 0.0]) / np.sqrt(2)
    mu = rho * cs * cs
    lam = rho * cp * cp - 2 * mu
    s = x @ n
    fp = amp[0] * np.sin(2 * np.pi * np.sqrt(3) * (s - cp * t))
    fs = amp[1] * np.sin(2 * np.pi * np.sqrt(3) * (s - cs * t))
    S = -(lam * np.eye(3) + 2 * mu * np.outer(n, n)) * (fp / cp)[..., None, None] \
        - mu * (np.outer(n, m) + np.outer(m, n)) * (fs / cs)[..., None, None]
    Q = np.zeros(x.shape[:-1] + (12,))
    Q[..., 0:3] = n * fp[..., None] + m * fs[..., None]
    Q[..., 3], Q[..., 4], Q[..., 5] = S[..., 0, 0], S[..., 1, 1], S[..., 2, 2]
    Q[..., 6], Q[..., 7], Q[..., 8] = S[..., 0, 1], S[..., 0, 2], S[..., 1, 2]
    Q[..., 9], Q[..., 10], Q[..., 11] = rho, cp, cs
    return Q


def acoustic_plane_wave(x, t, amp=1e-2):
    """p = f, v = n f with f(s) = a sin(2 pi sqrt(3) (s - t)), unit density and speed (flux form)."""
    n = np.ones(3) / np.sqrt(3)
    f = amp * np.sin(2 * np.pi * np.sqrt(3) * (x @ n - t))
    Q = np.zeros(x.shape[:-1] + (6,))
    Q[..., 0] = f
    Q[..., 1:4] = n * f[..., None]
    Q[..., 4] = Q[..., 5] = 1.0
    return Q


def l2(u, order):
    w = sc.gl_weights(order)
    wn = (w[:, None, None] * w[None, :, None] * w[None, None, :]).reshape(-1)
    u = np.asarray(u).reshape(-1, wn.size, u.shape[-1])
    return float(np.sqrt((u ** 2 * wn[None, :, None]).sum() / u.shape[0]))


def run_elastic(order, nc, T=0.1):
    """The plane wave through both schemes to time T (fixed dt from the CFL bound)."""
    x = sc.nodal_positions([nc] * 3, [1.0] * 3, order)
    q0 = elastic_plane_wave(x, 0.0)
    dt = 0.9 * sc_pnpm(order) * (1.0 / nc) / 3.0 / 3.0
    ns = int(np.ceil(T / dt))
    a = q0.reshape(-1).copy()
    RefLinear("elastic", order).run(a, [nc] * 3, [1.0] * 3, ns, fixed_dt=T / ns)
    b = q0.reshape(-1).copy()
    Oracle(3, order, PDE_ELASTIC).run(b, [nc] * 3, [1.0] * 3, ns, fixed_dt=T / ns)
    ex = elastic_plane_wave(x, T)
    sh = (-1, (order + 1) ** 3, 12)
    return a.reshape(sh)[..., :9], b.reshape(sh)[..., :9], ex.reshape(sh)[..., :9]


def sc_pnpm(order):
    from pyoracle import PNPM
    return PNPM[order]


def test_linear_apps_pde_terms_match_flux_form_functors():
    """M(Q) (F_d(dQ/dx_d) + B_d(grad Q)) of the reference applications equals the flux-form
    functors' F_d(dQ/dx_d) for random states, material parameters and gradients."""
    rng = np.random.default_rng(0)
    el, orc = RefLinear("elastic", 3), Oracle(3, 3, PDE_ELASTIC)
    for _ in range(100):
        cp = rng.uniform(2.0, 5.0)
        par = [rng.uniform(1.0, 3.0), cp, rng.uniform(0.3, cp / 1.6)]
        Q = np.concatenate([rng.normal(size=9), par])
        G = rng.normal(size=(3, 9))
        ref = el.terms(Q, G)
        ours = np.array([orc.flux(np.concatenate([G[d], par]))[d] for d in range(3)])
        assert np.abs(ref - ours).max() <= 1e-14 * np.abs(ref).max()
        lam_ref, lam_ours = el.eigenvalues(Q), orc_eigen_elastic(Q)
        assert np.abs(lam_ref).max() == np.abs(lam_ours).max()
        assert sorted(lam_ref) == sorted(lam_ours)
    ac, orca = RefLinear("acoustic", 3), Oracle(3, 3, PDE_ACOUSTIC)
    for _ in range(100):
        Q, G = rng.normal(size=4), rng.normal(size=(3, 4))
        ref = ac.terms(Q, G)
        ours = np.array([orca.flux(np.concatenate([ACOUSTIC_MAP @ G[d], [1.0, 1.0]]))[d] for d in range(3)])
        assert np.abs(ours - ref @ ACOUSTIC_MAP).max() <= 1e-15 * np.abs(ref).max()
        assert np.abs(ac.eigenvalues(Q)).max() == 1.0


def orc_eigen_elastic(Q):
    cp, cs = Q[10], Q[11]
    return [-cp, -cs, -cs, 0.0, 0.0, 0.0, cs, cs, cp]


@pytest.mark.parametrize("order", [3, 4])
def test_elastic_plane_wave_linear_reference_vs_oracle(order):
    """Both schemes on the oblique P + S plane wave, 4^3 periodic cells: each within its expected
    discretisation error of the exact solution, and within 1e-3 of that error of each other."""
    a, b, ex = run_elastic(order, 4)
    err_ref, err_ours, diff = l2(a - ex, order), l2(b - ex, order), l2(a - b, order)
    scale = l2(ex, order)
    assert err_ours < {3: 5e-3, 4: 5e-4}[order] * scale
    assert abs(err_ours - err_ref) <= 1e-2 * err_ref
    assert diff <= 1e-3 * err_ref


def test_elastic_plane_wave_convergence_both_schemes():
    """Order 3 on 4^3 and 8^3 cells: both errors fall by at least 12x (2^(N+1) = 16 expected)."""
    a4, b4, e4 = run_elastic(3, 4)
    a8, b8, e8 = run_elastic(3, 8)
    assert l2(a4 - e4, 3) / l2(a8 - e8, 3) > 12.0
    assert l2(b4 - e4, 3) / l2(b8 - e8, 3) > 12.0
    assert l2(a8 - b8, 3) <= 1e-3 * l2(a8 - e8, 3)


def test_acoustic_plane_wave_linear_reference_vs_oracle():
    """The acoustic application (unit medium, its velocity = minus the flux-form one) against the
    flux-form acoustics with rho = c = 1, both with their own CFL time step: the same step sizes, the
    same error against the exact wave, and a difference far below it."""
    order, nc = 3, 4
    x = sc.nodal_positions([nc] * 3, [1.0] * 3, order)
    q = acoustic_plane_wave(x, 0.0)
    a = (q[..., :4] @ ACOUSTIC_MAP).reshape(-1).copy()
    t_ref, dts_ref = RefLinear("acoustic", order).run(a, [nc] * 3, [1.0] * 3, 20)
    b = q.reshape(-1).copy()
    t_ours, dts_ours, _ = Oracle(3, order, PDE_ACOUSTIC).run(b, [nc] * 3, [1.0] * 3, 20, walls=0)
    assert np.allclose(dts_ref, dts_ours, rtol=1e-14, atol=0)
    ra = a.reshape(-1, (order + 1) ** 3, 4) @ ACOUSTIC_MAP
    rb = b.reshape(-1, (order + 1) ** 3, 6)[..., :4]
    ex = acoustic_plane_wave(x, t_ours)[..., :4]
    err_ref, err_ours, diff = l2(ra - ex, order), l2(rb - ex, order), l2(ra - rb, order)
    assert err_ours < 5e-3 * l2(ex, order)
    assert abs(err_ours - err_ref) <= 1e-2 * err_ref
    assert diff <= 1e-3 * err_ref


def test_point_source_total_moment_vs_delta_distribution():
    """An elastic point source (Ricker wavelet on s13) injected by the reference's delta distribution
    and by the regularised Gaussian of the nonlinear path: the same total moment in the domain
    (the integral of s13 over the periodic cube, which only the source changes) at two times.
    The reference's linear kernels add the time-averaged source to lFhi
    (3d/spaceTimePredictorLinear.cpph:480-500), which volumeIntegralLinear subtracts, so a source
    of amplitude A there injects -A; the nonlinear path is given -A."""
    order, nc, A = 3, 6, 1.0
    dx = 1.0 / nc
    x = sc.nodal_positions([nc] * 3, [1.0] * 3, order)
    q0 = np.zeros(x.shape[:-1] + (12,))
    q0[..., 9], q0[..., 10], q0[..., 11] = 2.0, 3.0, 1.5
    w = sc.gl_weights(order)
    wn = (w[:, None, None] * w[None, :, None] * w[None, None, :]).reshape(-1)
    f0, t0 = 4.0, 0.3
    src = (0.53, 0.47, 0.51, f0, t0, A, 0.5 * dx, 7.0)
    ours_src = src[:5] + (-A,) + src[6:]

    def ricker_integral(T):  # d/dt [(t - t0) exp(-a^2)] = (1 - 2 a^2) exp(-a^2), a = pi f0 (t - t0)
        g = lambda t: (t - t0) * np.exp(-(np.pi * f0 * (t - t0)) ** 2)
        return g(T) - g(0.0)

    for nsteps in (30, 80):
        a = q0.reshape(-1).copy()
        t_ref, _ = RefLinear("elastic", order, source=src).run(a, [nc] * 3, [1.0] * 3, nsteps)
        b = q0.reshape(-1).copy()
        t_ours, _, _ = Oracle(3, order, PDE_ELASTIC, source=ours_src).run(b, [nc] * 3, [1.0] * 3, nsteps, walls=0)
        assert abs(t_ref - t_ours) <= 1e-14 * t_ref
        Ia = (a.reshape(-1, wn.size, 12)[..., :9] * wn[None, :, None]).sum((0, 1)) * dx ** 3
        Ib = (b.reshape(-1, wn.size, 12)[..., :9] * wn[None, :, None]).sum((0, 1)) * dx ** 3
        expect = -A * ricker_integral(t_ref)
        assert abs(expect) > 1e-5
        assert abs(Ia[7] - expect) <= 1e-9 * abs(expect)
        assert abs(Ib[7] - expect) <= 1e-3 * abs(expect)
        others = [k for k in range(9) if k != 7]
        assert np.abs(Ia[others]).max() <= 1e-12 * abs(expect)
        assert np.abs(Ib[others]).max() <= 1e-12 * abs(expect)
