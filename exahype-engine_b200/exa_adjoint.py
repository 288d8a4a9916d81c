"""Full-waveform misfit gradients through the discrete adjoint of the ADER-DG step.

The forward model is the device patch stepping a linear wave system (acoustic: p, u, v, w with
per-cell rho, c; elastic: 9 velocity-stress fields with per-cell rho, cp, cs) with a fixed time
step and a fixed Picard sweep count (the reference's UseMaxPicardIterations mode), on a periodic
grid. Receivers record the pressure (acoustic) or a chosen field at fixed points after every
step; the misfit is

    J = 1/2 sum_{k=1..K} sum_r (rec_r(u_k) - d_{k,r})^2,

rec_r(u) being the DG polynomial of the receiver's cell evaluated at the receiver (tensor
Lagrange basis on the Gauss-Legendre nodes). dJ/d(per-cell parameters) and dJ/d(initial field)
come from exa_patch_adjoint_step, one call per step in reverse order, with the states the
adjoint needs recomputed from binomial checkpoints (exa_checkpoint_schedule: `snaps` stored
states, the initial one included).

`Misfit.apply(params, field0, inversion, data)` is the torch.autograd.Function the tests use.
Everything runs on the device; the host only walks the schedule.
"""
import numpy as np
import torch

import exa_aderdg as exa
from exa_scenarios import gl_nodes


def lagrange_basis(order, xi):
    """Values of the n = order + 1 Lagrange polynomials on the Gauss-Legendre nodes at xi."""
    x = gl_nodes(order)
    n = order + 1
    out = np.ones(n)
    for j in range(n):
        for i in range(n):
            if i != j:
                out[j] *= (xi - x[i]) / (x[j] - x[i])
    return out


def receiver_operator(ncell, size, order, positions, offset=None):
    """(cell index [R], node weights [R, nd]) so that rec_r(u) = sum_p w[r, p] u[cell_r, p, var]."""
    dim = len(ncell)
    off = np.zeros(dim) if offset is None else np.asarray(offset, dtype=float)
    dx = np.asarray(size, dtype=float) / np.asarray(ncell)
    cells, weights = [], []
    for x in np.asarray(positions, dtype=float):
        idx = np.minimum(np.floor((x - off) / dx).astype(int), np.asarray(ncell) - 1)
        idx = np.maximum(idx, 0)
        xi = (x - off) / dx - idx
        L = [lagrange_basis(order, xi[d]) for d in range(dim)]
        if dim == 3:
            w = (L[2][:, None, None] * L[1][None, :, None] * L[0][None, None, :]).reshape(-1)
            c = (idx[2] * ncell[1] + idx[1]) * ncell[0] + idx[0]
        else:
            w = (L[1][:, None] * L[0][None, :]).reshape(-1)
            c = idx[1] * ncell[0] + idx[0]
        cells.append(int(c))
        weights.append(w)
    return np.array(cells, dtype=np.int64), np.array(weights)


class WaveInversion:
    """One forward model: grid, order, time step, receivers, checkpoint budget."""

    def __init__(self, pde, ncell, size, order, dt, nsteps, receivers, rec_var=0, snaps=20, source=None,
                 device="cuda", bc=0):
        """bc: domain faces of the grid (exa_aderdg.BC_*, one or per axis): periodic, reflective
        walls or outflow (absorbing for normal waves)."""
        if pde not in (exa.PDE_ACOUSTIC, exa.PDE_ELASTIC):
            raise ValueError("the adjoint is built for the acoustic and elastic systems")
        self.pde, self.ncell, self.size, self.order = pde, tuple(ncell), list(size), order
        self.dt, self.nsteps, self.rec_var, self.snaps = float(dt), int(nsteps), int(rec_var), int(snaps)
        self.dev = torch.device(device)
        self.V, self.P = exa.NVAR[pde], exa.NPAR[pde]
        self.D = self.V + self.P
        self.n = order + 1
        self.nd = self.n ** len(ncell)
        self.ncells = int(np.prod(ncell))
        # the reference's fixed-count Picard mode: MaxPicardIterations = Order + 1
        self.solver = exa.Solver(pde, len(ncell), order, npar=self.P, max_picard=order + 1)
        self.patch = exa.Patch(self.solver, [dict(ncell=self.ncell, size=self.size, bc=bc)])
        self.source = source
        if source is not None:
            self.patch.set_point_source(source[:3], source[3], source[4], source[5], source[6], int(source[7]))
        cells, w = receiver_operator(self.ncell, self.size, order, receivers)
        self.rec_cells = torch.as_tensor(cells, device=self.dev)
        self.rec_w = torch.as_tensor(w, device=self.dev, dtype=torch.float64)
        self.schedule, self.recompute_steps = exa.checkpoint_schedule(self.nsteps, self.snaps)
        shape = (self.ncells, self.nd, self.D)
        self._slots = [torch.empty(shape, dtype=torch.float64, device=self.dev) for _ in range(self.snaps)]
        self._last = torch.empty(shape, dtype=torch.float64, device=self.dev)
        self._cur = torch.empty(shape, dtype=torch.float64, device=self.dev)
        self.stream = torch.cuda.ExternalStream(self.patch.stream)

    # ---------------- model assembly ----------------
    def assemble(self, params, field0):
        """luh [cells, nd, D] from per-cell parameters [cells, P] and the initial fields
        [cells, nd, V] (or [cells, nd] for the receiver variable only)."""
        luh = torch.zeros((self.ncells, self.nd, self.D), dtype=torch.float64, device=self.dev)
        if field0.dim() == 2:
            luh[:, :, self.rec_var] = field0
        else:
            luh[:, :, :self.V] = field0
        luh[:, :, self.V:] = params[:, None, :]
        return luh

    def record(self, luh):
        """Receiver values of a state [R]."""
        return (self.rec_w * luh[self.rec_cells, :, self.rec_var]).sum(-1)

    def _rec_adjoint(self, lam, resid):
        """lam += d(1/2 |rec(u) - d|^2)/du for one step's residual [R]."""
        contrib = resid[:, None] * self.rec_w
        lam[:, :, self.rec_var].index_put_((self.rec_cells,), contrib, accumulate=True)

    # ---------------- patch state helpers ----------------
    def _set(self, luh, step):
        self.patch.set_solution(luh.reshape(-1))
        self.patch.set_time(step * self.dt)

    def _get(self, out):
        self.patch.get_solution(out.reshape(-1))
        return out

    def _advance(self, k0, k1, traces=None):
        for k in range(k0, k1):
            self.patch.step(1, self.dt)
            if traces is not None:
                self._get(self._cur)
                traces[k + 1] = self.record(self._cur)

    # ---------------- forward ----------------
    def forward_traces(self, luh0):
        """Plain forward run: receiver traces [K+1, R] (row 0 = the initial state)."""
        return self._on_patch_stream(self._forward_traces, luh0)

    def _forward_traces(self, luh0):
        traces = torch.zeros((self.nsteps + 1, self.rec_cells.numel()), dtype=torch.float64, device=self.dev)
        self._set(luh0, 0)
        traces[0] = self.record(luh0)
        self._advance(0, self.nsteps, traces)
        return traces

    def _on_patch_stream(self, fn, *args):
        """Run fn with torch work ordered on the patch stream (the library's kernels run there)."""
        cur = torch.cuda.current_stream(self.dev)
        self.stream.wait_stream(cur)
        with torch.cuda.stream(self.stream):
            out = fn(*args)
        cur.wait_stream(self.stream)
        return out

    def forward(self, luh0, data):
        """J and the residuals [K+1, R]; leaves the checkpoints the reverse sweep starts from.

        Runs the schedule's leading stores and advances (its first pass reaches u_{K-1}), keeps
        u_{K-1} aside and takes the last step for the final receivers."""
        return self._on_patch_stream(self._forward, luh0, data)

    def _forward(self, luh0, data):
        R = self.rec_cells.numel()
        traces = torch.zeros((self.nsteps + 1, R), dtype=torch.float64, device=self.dev)
        self._set(luh0, 0)
        traces[0] = self.record(luh0)
        i = 0
        for i, (act, a, b) in enumerate(self.schedule):
            if act == exa.CK_STORE:
                self._get(self._slots[a])
            elif act == exa.CK_ADVANCE:
                self._advance(a, b, traces)
            elif act == exa.CK_ADJOINT:
                break
            else:
                raise RuntimeError("restore before the first adjoint step")
        self._resume = i
        self._get(self._last)                      # u_{K-1}
        self._advance(self.nsteps - 1, self.nsteps, traces)
        resid = traces - data
        resid[0] = 0.0                             # the misfit starts at step 1
        J = 0.5 * (resid * resid).sum()
        return J, resid, traces

    # ---------------- reverse ----------------
    def backward(self, resid):
        """dJ/du_0 (luh layout); its parameter entries hold dJ/d(parameter) per node."""
        return self._on_patch_stream(self._backward, resid)

    def _backward(self, resid):
        lam = torch.zeros((self.ncells, self.nd, self.D), dtype=torch.float64, device=self.dev)
        self._rec_adjoint(lam, resid[self.nsteps])
        self._set(self._last, self.nsteps - 1)
        for act, a, b in self.schedule[self._resume:]:
            if act == exa.CK_ADJOINT:
                self.patch.adjoint_step(lam, self.dt)
                if a >= 1:
                    self._rec_adjoint(lam, resid[a])
            elif act == exa.CK_RESTORE:
                self._set(self._slots[a], b)
            elif act == exa.CK_ADVANCE:
                self._advance(a, b)
            elif act == exa.CK_STORE:
                self._get(self._slots[a])
        return lam

    def close(self):
        self.patch.close()


def fd_directional(inv, params, field0, vp, vf, data, h=1e-6, with_scale=False):
    """Central finite difference (J(x + h v) - J(x - h v)) / (2 h) of the misfit along (vp, vf),
    evaluated as sum_k (tr+ - tr-) . ((tr+ + tr-)/2 - d) / (2 h): the same two model runs and the
    same difference, without forming J+ and J- first (their leading digits cancel). With
    with_scale, also returns sum_k |(tr+ - tr-) . ((tr+ + tr-)/2 - d)| / (2 h), the scale against
    which the sum's cancellation (and so its rounding) is measured."""
    trp = inv.forward_traces(inv.assemble(params + h * vp, field0 + h * vf))
    trm = inv.forward_traces(inv.assemble(params - h * vp, field0 - h * vf))
    diff = (trp - trm)[1:]
    mean = 0.5 * (trp + trm)[1:] - data[1:]
    terms = diff * mean
    fd = float(terms.sum()) / (2.0 * h)
    if with_scale:
        return fd, float(terms.abs().sum()) / (2.0 * h)
    return fd


class Misfit(torch.autograd.Function):
    """J(params [cells, P], field0 [cells, nd] or [cells, nd, V]) for a WaveInversion and data."""

    @staticmethod
    def forward(ctx, params, field0, inv, data):
        luh0 = inv.assemble(params.detach(), field0.detach())
        J, resid, _ = inv.forward(luh0, data)
        ctx.inv = inv
        ctx.field_dim = field0.dim()
        ctx.save_for_backward(resid)
        return J

    @staticmethod
    def backward(ctx, gJ):
        (resid,) = ctx.saved_tensors
        inv = ctx.inv
        lam = inv.backward(resid) * gJ
        g_params = lam[:, :, inv.V:].sum(1)
        g_field = lam[:, :, inv.rec_var] if ctx.field_dim == 2 else lam[:, :, :inv.V]
        return g_params, g_field, None, None


# ------------------------------------------------------------------------------------------
# seeded models (the acoustic adjoint workload)
# ------------------------------------------------------------------------------------------

def smooth_field(ncell, size, lo, hi, rng, nmodes=6, kmax=2):
    """Periodic smooth random per-cell field with values in [lo, hi] (cell centres)."""
    dim = len(ncell)
    dx = np.asarray(size, dtype=float) / np.asarray(ncell)
    axes = [(np.arange(ncell[d]) + 0.5) * dx[d] / size[d] for d in range(dim)]
    grids = np.meshgrid(*axes[::-1], indexing="ij")[::-1]   # x fastest in the flattened order
    g = np.zeros(grids[0].shape)
    for _ in range(nmodes):
        k = rng.integers(-kmax, kmax + 1, size=dim)
        if not k.any():
            k[0] = 1
        ph = rng.uniform(0, 2 * np.pi)
        g += rng.uniform(0.5, 1.0) * np.cos(2 * np.pi * sum(k[d] * grids[d] for d in range(dim)) + ph)
    g = (g - g.min()) / max(g.max() - g.min(), 1e-300)
    return (lo + (hi - lo) * g).reshape(-1)


def acoustic_model(ncell, size, order, seed=0, width=0.05, anomaly=0.05):
    """Per-cell (rho, c), the perturbed c with a +anomaly Gaussian blob, the initial pressure
    (Gaussian pulse of the given width) and 64 receiver positions."""
    from exa_scenarios import nodal_positions
    rng = np.random.default_rng(seed)
    rho = smooth_field(ncell, size, 1.0, 2.5, rng)
    c = smooth_field(ncell, size, 1.5, 3.0, rng)
    size_a = np.asarray(size, dtype=float)
    x0 = size_a * rng.uniform(0.3, 0.7, 3)
    xa = size_a * rng.uniform(0.3, 0.7, 3)
    dx = size_a / np.asarray(ncell)
    cc = np.stack(np.meshgrid(*[(np.arange(ncell[d]) + 0.5) * dx[d] for d in range(3)][::-1],
                              indexing="ij")[::-1], -1).reshape(-1, 3)
    blob = np.exp(-((cc - xa) ** 2).sum(-1) / (2 * (0.1 * size_a.min()) ** 2))
    c_true = c * (1.0 + anomaly * blob)
    xn = nodal_positions(ncell, size, order)
    p0 = np.exp(-((xn - x0) ** 2).sum(-1) / (width * size_a.min()) ** 2)
    receivers = size_a * rng.uniform(0.05, 0.95, (64, 3))
    return dict(rho=rho, c=c, c_true=c_true, p0=p0, receivers=receivers)


def cfl_dt(ncell, size, order, cmax, cfl=0.9):
    """The solver's CFL step for the fastest wave speed cmax (PNPM of the order)."""
    pnpm = [1.0, 0.33, 0.17, 0.1, 0.069, 0.045, 0.038, 0.03, 0.02, 0.015][order]
    dx = np.asarray(size, dtype=float) / np.asarray(ncell)
    return cfl * pnpm / sum(cmax / dx[d] for d in range(len(ncell)))
