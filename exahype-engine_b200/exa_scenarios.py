"""Seeded synthetic initial states for the benchmark and parity workloads.

The reference fills a cell by evaluating the user's ``adjustPointSolution`` at the
Gauss-Legendre nodes, x = centre + dx * (node - 0.5) (ExaHyPE/kernels/aderdg/generic/c/3d/
solutionAdjustment.cpph:38-58): nodal interpolation, not L2 projection. ``nodal_positions``
restates that placement; the state functions below play the role of adjustPointSolution.

Workloads (numpy.random.default_rng(seed), seed 0 unless stated):

* ``euler2d_entropy_wave`` -- 2D Euler, rho = 1 + 0.2 * sum of 4 Fourier modes (integer k,
  0 < |k| <= 3, random phases), u = v = 0.3, p = 1, periodic unit square.
* ``euler3d_entropy_wave`` -- 3D Euler, rho = 1 + 0.1 * (1/8) * sum of 8 Fourier modes
  (0 < |k| <= 4), u = (0.3, 0.2, 0.1), p = 1, periodic unit cube.

Both are entropy waves: pressure and velocity are uniform, so the exact solution of the Euler
equations is rho advected with u (``*_exact``), which gives an analytic L2 error next to the
error against the FP64 oracle.
"""
import numpy as np

GAMMA = 1.4


def gl_nodes(order):
    """Gauss-Legendre nodes on [0,1], ascending."""
    x, _ = np.polynomial.legendre.leggauss(order + 1)
    return 0.5 * (x + 1.0)


def gl_weights(order):
    _, w = np.polynomial.legendre.leggauss(order + 1)
    return 0.5 * w


def nodal_positions(ncell, size, order, offset=None):
    """Node coordinates of every cell, shape [cells][nodes][dim], reference node order.

    Cell c = (iz*ny + iy)*nx + ix; node p = (z*n + y)*n + x (2D: y*n + x).
    """
    dim = len(ncell)
    offset = np.zeros(dim) if offset is None else np.asarray(offset, dtype=float)
    dx = np.asarray(size, dtype=float) / np.asarray(ncell)
    xi = gl_nodes(order)
    n = order + 1
    if dim == 3:
        nx, ny, nz = ncell
        iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        kz, ky, kx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        cx = offset[0] + (ix.reshape(-1, 1) + xi[kx.reshape(1, -1)]) * dx[0]
        cy = offset[1] + (iy.reshape(-1, 1) + xi[ky.reshape(1, -1)]) * dx[1]
        cz = offset[2] + (iz.reshape(-1, 1) + xi[kz.reshape(1, -1)]) * dx[2]
        return np.stack([cx, cy, cz], axis=-1)
    nx, ny = ncell
    iy, ix = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    ky, kx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    cx = offset[0] + (ix.reshape(-1, 1) + xi[kx.reshape(1, -1)]) * dx[0]
    cy = offset[1] + (iy.reshape(-1, 1) + xi[ky.reshape(1, -1)]) * dx[1]
    return np.stack([cx, cy], axis=-1)


def _modes(rng, nmodes, kmax, dim):
    ks = []
    while len(ks) < nmodes:
        k = rng.integers(-kmax, kmax + 1, size=dim)
        if 0 < np.linalg.norm(k) <= kmax:
            ks.append(k)
    phases = rng.uniform(0.0, 2.0 * np.pi, size=nmodes)
    return np.array(ks, dtype=float), phases


class EntropyWave:
    """rho = 1 + amp * sum_m cos(2 pi k_m.(x - u t) + phi_m), uniform u and p."""

    def __init__(self, dim, seed=0):
        rng = np.random.default_rng(seed)
        self.dim = dim
        if dim == 2:
            self.k, self.phi = _modes(rng, 4, 3, 2)
            self.amp = 0.2
            self.u = np.array([0.3, 0.3])
        else:
            self.k, self.phi = _modes(rng, 8, 4, 3)
            self.amp = 0.1 / 8.0
            self.u = np.array([0.3, 0.2, 0.1])
        self.p = 1.0

    def rho(self, x, t=0.0):
        xs = x - self.u * t
        arg = 2.0 * np.pi * np.tensordot(xs, self.k.T, axes=([-1], [0])) + self.phi
        return 1.0 + self.amp * np.cos(arg).sum(-1)

    def state(self, x, t=0.0):
        """Conserved Euler state (rho, rho u, rho v, rho w, E) at points x[..., dim]; nVar = 5."""
        rho = self.rho(x, t)
        Q = np.zeros(x.shape[:-1] + (5,))
        Q[..., 0] = rho
        for d in range(self.dim):
            Q[..., 1 + d] = rho * self.u[d]
        Q[..., 4] = self.p / (GAMMA - 1.0) + 0.5 * rho * float(self.u @ self.u)
        return Q


def euler_entropy_wave(ncell, order, seed=0, t=0.0):
    """Initial (or exact at time t) nodal state, shape [cells * nodes * 5], periodic unit box."""
    dim = len(ncell)
    wave = EntropyWave(dim, seed)
    x = nodal_positions(ncell, [1.0] * dim, order)
    return wave.state(x, t).reshape(-1), wave


def l2_linf_error(luh, exact, order, dim, nvar_out=1, nvar=5):
    """Quadrature-weighted L2 and max errors of the first ``nvar_out`` variables (unit box)."""
    w = gl_weights(order)
    if dim == 3:
        wn = (w[:, None, None] * w[None, :, None] * w[None, None, :]).reshape(-1)
    else:
        wn = (w[:, None] * w[None, :]).reshape(-1)
    a = np.asarray(luh).reshape(-1, wn.size, nvar)[..., :nvar_out]
    b = np.asarray(exact).reshape(-1, wn.size, nvar)[..., :nvar_out]
    ncells = a.shape[0]
    e2 = ((a - b) ** 2 * wn[None, :, None]).sum() / ncells
    return float(np.sqrt(e2)), float(np.max(np.abs(a - b)))


# ------------------------------------------------------------------------------------------
# Batched shallow water: many independent grids of uneven sizes
# ------------------------------------------------------------------------------------------

def swe_grid_specs(ngrids=512, seed=0, nmin=16, nmax=128):
    """Per-grid square sizes drawn uniformly from nmin..nmax cells per side, unit square each."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(nmin, nmax + 1, size=ngrids)
    return [dict(ncell=(int(s), int(s)), size=[1.0, 1.0]) for s in sides]


def swe_bumps_state(ncell, order, rng):
    """h = 1 + 1..5 circular bumps (height U[0.2,1], radius U[0.05,0.2]), zero velocity,
    bathymetry b = 0.1 * a smooth random field; (h, hu, hv, b) per node."""
    x = nodal_positions(ncell, [1.0, 1.0], order)  # [cells][nodes][2]
    nb = int(rng.integers(1, 6))
    h = np.ones(x.shape[:-1])
    for _ in range(nb):
        c = rng.uniform(0.2, 0.8, 2)
        hgt = rng.uniform(0.2, 1.0)
        rad = rng.uniform(0.05, 0.2)
        r2 = ((x - c) ** 2).sum(-1)
        h += hgt * np.exp(-r2 / (rad * rad))
    kx, ky = rng.integers(1, 4, 2)
    ph = rng.uniform(0, 2 * np.pi, 2)
    b = 0.1 * 0.5 * (np.cos(2 * np.pi * kx * x[..., 0] + ph[0]) * np.cos(2 * np.pi * ky * x[..., 1] + ph[1]) + 1.0)
    Q = np.zeros(x.shape[:-1] + (4,))
    Q[..., 0] = h
    Q[..., 3] = b
    return Q.reshape(-1)


def swe_batched(ngrids=512, order=4, seed=0, nmin=16, nmax=128):
    """Grid specs (reflective walls) and the concatenated initial state of every grid."""
    specs = swe_grid_specs(ngrids, seed, nmin, nmax)
    rng = np.random.default_rng(seed + 1)
    states = [swe_bumps_state(sp["ncell"], order, rng) for sp in specs]
    for sp in specs:
        sp["bc"] = 1  # reflective walls on every side
    return specs, states


# ------------------------------------------------------------------------------------------
# Linear waves in a layered medium, driven by a point source
# ------------------------------------------------------------------------------------------

def layered_medium(pde, ncell, size, order, seed=0, offset=None):
    """Initial state of the acoustic (V=4, P=2) or elastic (V=9, P=3) system with material
    parameters constant per cell: two layers split at mid-height of the last axis (upper layer
    slower), with a +-5 % seeded random perturbation per cell. Acoustic: a Gaussian pressure pulse
    (width 0.08 of the box) at 0.3 of the box; elastic: at rest. Returns luh [cells*nodes*D]."""
    rng = np.random.default_rng(seed)
    dim = len(ncell)
    x = nodal_positions(ncell, size, order, offset)          # [cells][nodes][dim]
    ncells, nd = x.shape[0], x.shape[1]
    off = np.zeros(dim) if offset is None else np.asarray(offset, dtype=float)
    size = np.asarray(size, dtype=float)
    cz = x.mean(axis=1)[:, -1]                               # cell-centre height
    upper = cz > off[-1] + 0.5 * size[-1]
    jitter = 1.0 + 0.05 * rng.uniform(-1, 1, ncells)
    if pde == "acoustic":
        rho = np.where(upper, 1.0, 1.5)
        c = np.where(upper, 1.0, 1.6) * jitter
        Q = np.zeros((ncells, nd, 6))
        r2 = (((x - (off + 0.3 * size)) / (0.08 * size)) ** 2).sum(-1)
        Q[..., 0] = np.exp(-r2)
        Q[..., 4] = rho[:, None]
        Q[..., 5] = c[:, None]
        return Q.reshape(-1)
    if pde == "elastic":
        rho = np.where(upper, 1.0, 1.4)
        cp = np.where(upper, 1.7, 2.4) * jitter
        cs = np.where(upper, 1.0, 1.4) * jitter
        Q = np.zeros((ncells, nd, 12))
        Q[..., 9] = rho[:, None]
        Q[..., 10] = cp[:, None]
        Q[..., 11] = cs[:, None]
        return Q.reshape(-1)
    raise ValueError(pde)


def ricker_source(dim, size, offset=None, f0=4.0, amplitude=1.0, width=None, variable=0, at=0.5):
    """(x, y, z, f0, t0, amplitude, width, variable) of a point source at fraction `at` of the box,
    delayed by t0 = 1.2 / f0 so that the wavelet starts from (near) zero."""
    off = np.zeros(dim) if offset is None else np.asarray(offset, dtype=float)
    size = np.asarray(size, dtype=float)
    pos = list(off + at * size) + [0.0] * (3 - dim)
    w = float(width) if width is not None else float(0.04 * size.min())
    return tuple(pos) + (float(f0), 1.2 / float(f0), float(amplitude), w, float(variable))


def elastic_layers(ncell, size, order, seed=0, nlayers=6, offset=None):
    """The layered elastic configuration: nlayers horizontal layers (constant in x, y) with seeded
    interface depths along z, per layer rho ~ U[2.0, 3.0], cp ~ U[4.0, 6.5], cs = cp / sqrt(3) *
    U[0.9, 1.1]; parameters constant per cell (from the cell centre), the medium at rest.
    Returns (luh [cells*nodes*12], layer table [nlayers][4] = z_top, rho, cp, cs)."""
    rng = np.random.default_rng(seed)
    off = np.zeros(3) if offset is None else np.asarray(offset, dtype=float)
    size = np.asarray(size, dtype=float)
    depths = np.sort(rng.uniform(0.0, 1.0, nlayers - 1)) * size[2] + off[2]
    rho = rng.uniform(2.0, 3.0, nlayers)
    cp = rng.uniform(4.0, 6.5, nlayers)
    cs = cp / np.sqrt(3.0) * rng.uniform(0.9, 1.1, nlayers)
    x = nodal_positions(ncell, size, order, offset)
    cz = x.mean(axis=1)[:, 2]
    layer = np.searchsorted(depths, cz)
    Q = np.zeros(x.shape[:-1] + (12,))
    Q[..., 9] = rho[layer][:, None]
    Q[..., 10] = cp[layer][:, None]
    Q[..., 11] = cs[layer][:, None]
    table = np.stack([np.append(depths, size[2] + off[2]), rho, cp, cs], -1)
    return Q.reshape(-1), table


def elastic_source(size, seed=0, f0=10.0, width=None, variable=2, offset=None):
    """Ricker point source at a seeded interior point (middle 60% of the box), on the vertical
    velocity by default, delayed by 1.2 / f0; width defaults to 1% of the box."""
    rng = np.random.default_rng(seed + 101)
    off = np.zeros(3) if offset is None else np.asarray(offset, dtype=float)
    size = np.asarray(size, dtype=float)
    pos = off + size * rng.uniform(0.2, 0.8, 3)
    w = float(width) if width is not None else float(0.01 * size.min())
    return tuple(pos) + (float(f0), 1.2 / float(f0), 1.0, w, float(variable))
