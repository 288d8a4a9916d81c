"""Slab decomposition of one uniform grid over the ranks of a torch.distributed process group.

The reference distributes its spacetree with MPI: cells next to a remote rank send their face
data (ADERDGSolver::sendDataToNeighbour, mergeWithNeighbourData; ADERDGSolver.cpp:1946-2010),
and the admissible time step is reduced over all ranks before the next step
(ADERDGSolver.cpp:369-416). Here the grid is cut along its last axis into contiguous slabs, one
per rank (one rank per GPU). A rank's patch carries EXA_BC_HALO on that axis. Every step:

    predictor + volume integral          (local)
    pack the two boundary layers' face traces -> start the exchange with the lower / upper rank
    Rusanov on the faces between own cells (overlaps the exchange)
    finish the exchange, unpack into the ghost cells -> Rusanov on the ghost cells' faces
    surface integral + update + local CFL  -> all-reduce(min) of the time step
    advance t and dt

Only face traces cross ranks: per neighbour and step, one layer of (D + V) * n^(d-1) doubles per
cell face (81^2 cells x 360 doubles = 18.9 MB for the 81^3 N=5 Euler slab). The time step costs
one 8-byte all-reduce. With one rank the slab is the whole grid and no exchange happens.

The exchange pairs sends and receives the same way on every backend: each rank sends its high
layer up (tag 1) and its low layer down (tag 2), and receives the lower rank's high layer and the
upper rank's low layer, all inside one batched P2P call (NCCL needs the batch for two messages
between the same pair of ranks when there are only two ranks).
"""
import torch
import torch.distributed as dist

import exa_aderdg as exa


def slab_partition(n, world, rank):
    """(first, count) of rank's contiguous share of n layers; the first n % world ranks get one more."""
    base, extra = divmod(n, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def start_halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world, group=None):
    """Starts recv_lo <- lower rank's send_hi and recv_hi <- upper rank's send_lo (periodic ring);
    returns the requests. With NCCL the transfers are ordered after the current stream's work and
    run on NCCL's stream, so kernels enqueued afterwards overlap them."""
    up = (rank + 1) % world
    down = (rank - 1) % world
    ops = [dist.P2POp(dist.isend, send_hi, up, group, 1),
           dist.P2POp(dist.isend, send_lo, down, group, 2),
           dist.P2POp(dist.irecv, recv_lo, down, group, 1),
           dist.P2POp(dist.irecv, recv_hi, up, group, 2)]
    return dist.batch_isend_irecv(ops)


def finish_halo_exchange(reqs):
    """With NCCL, Work.wait() makes the current stream wait for the transfers (no host wait); with
    gloo it waits on the host."""
    for req in reqs:
        req.wait()


def halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world, group=None):
    """recv_lo <- lower rank's send_hi; recv_hi <- upper rank's send_lo (periodic ring)."""
    finish_halo_exchange(start_halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world, group))


def min_all_reduce(buf, group=None):
    dist.all_reduce(buf, op=dist.ReduceOp.MIN, group=group)


class SlabPatch:
    """A rank's slab of a global uniform grid, periodic along the cut axis (a ring of ranks)."""

    def __init__(self, solver, ncell, size, offset=None, bc_other=exa.BC_PERIODIC, rank=0, world=1, group=None):
        self.solver, self.rank, self.world, self.group = solver, rank, world, group
        dim = len(ncell)
        self.dim = dim
        offset = list(offset) if offset is not None else [0.0] * dim
        n_last = ncell[-1]
        self.first, self.count = slab_partition(n_last, world, rank)
        if self.count <= 0:
            raise ValueError("more ranks than layers along the cut axis")
        h = size[-1] / n_last
        lnc = tuple(ncell[:-1]) + (self.count,)
        lsize = list(size[:-1]) + [self.count * h]
        loff = list(offset[:-1]) + [offset[-1] + self.first * h]
        bcs = [bc_other] * (dim - 1) + [exa.BC_HALO if world > 1 else exa.BC_PERIODIC]
        self._local = (lnc, lsize, loff)
        self.patch = exa.Patch(solver, [dict(ncell=lnc, size=lsize, offset=loff, bc=bcs)])
        self.layer_cells = 1
        for k in ncell[:-1]:
            self.layer_cells *= k
        self.cells_per_layer_doubles = self.layer_cells * solver.sizes["luh"]
        self.stream = torch.cuda.ExternalStream(self.patch.stream)
        if world > 1:
            nh = self.patch.halo_doubles()
            dev = torch.device("cuda")
            self.send_lo = torch.zeros(nh, dtype=torch.float64, device=dev)
            self.send_hi = torch.zeros_like(self.send_lo)
            self.recv_lo = torch.zeros_like(self.send_lo)
            self.recv_hi = torch.zeros_like(self.send_lo)
            self.dtbuf = torch.zeros(1, dtype=torch.float64, device=dev)

    def local_range(self):
        """Slice of the global cell-major luh array this rank owns (its layers are contiguous)."""
        lo = self.first * self.cells_per_layer_doubles
        return lo, lo + self.count * self.cells_per_layer_doubles

    def set_solution(self, luh_global):
        lo, hi = self.local_range()
        self.set_local_solution(luh_global[lo:hi])

    def set_local_solution(self, luh_local):
        """This rank's cells only (host numpy array or CUDA tensor, reference layout)."""
        self.patch.set_solution(luh_local)
        if self.world > 1:  # the first time step is the minimum over every rank's cells
            with torch.cuda.stream(self.stream):
                self.patch.dt_copy(self.dtbuf, 0)
                min_all_reduce(self.dtbuf, self.group)
                self.patch.dt_copy(self.dtbuf, 1)

    def step(self, nsteps=1, fixed_dt=0.0):
        p = self.patch
        for _ in range(nsteps):
            if self.world == 1:
                p.step(1, fixed_dt)
                continue
            with torch.cuda.stream(self.stream):
                p.step_phase(exa.PHASE_PREDICTOR, fixed_dt)
                p.halo_pack(self.send_lo, self.send_hi)
                reqs = start_halo_exchange(self.send_lo, self.send_hi, self.recv_lo, self.recv_hi, self.rank,
                                           self.world, self.group)
                # the faces between this rank's own cells while the traces are in flight
                p.step_phase(exa.PHASE_FACES_INTERIOR, fixed_dt)
                finish_halo_exchange(reqs)
                p.halo_unpack(self.recv_lo, self.recv_hi)
                p.step_phase(exa.PHASE_FACES_HALO, fixed_dt)
                p.step_phase(exa.PHASE_UPDATE, fixed_dt)
                if not fixed_dt > 0:
                    p.dt_next_copy(self.dtbuf, 0)
                    min_all_reduce(self.dtbuf, self.group)
                    p.dt_next_copy(self.dtbuf, 1)
                p.step_phase(exa.PHASE_ADVANCE, fixed_dt)

    def adjoint_step(self, lam, dt):
        """The discrete adjoint of one fixed-dt step over all ranks: lam (CUDA float64, this rank's
        cells, luh layout) holds dJ/du_{k+1} on entry and this rank's part of dJ/du_k on exit. The
        transposed faces between slabs need the neighbours' face traces (the forward exchange) and
        their boundary layers' lambda (a second exchange on the same ring)."""
        p = self.patch
        if self.world == 1:
            p.adjoint_step(lam, dt)
            return
        if not hasattr(self, "lam_send_lo"):
            nl = p.adjoint_halo_doubles()
            self.lam_send_lo = torch.zeros(nl, dtype=torch.float64, device=lam.device)
            self.lam_send_hi = torch.zeros_like(self.lam_send_lo)
            self.lam_recv_lo = torch.zeros_like(self.lam_send_lo)
            self.lam_recv_hi = torch.zeros_like(self.lam_send_lo)
        with torch.cuda.stream(self.stream):
            p.adjoint_phase(exa.ADJ_FORWARD, lam, dt)
            p.halo_pack(self.send_lo, self.send_hi)
            p.adjoint_halo_pack(self.lam_send_lo, self.lam_send_hi)
            halo_exchange(self.send_lo, self.send_hi, self.recv_lo, self.recv_hi, self.rank, self.world, self.group)
            halo_exchange(self.lam_send_lo, self.lam_send_hi, self.lam_recv_lo, self.lam_recv_hi, self.rank,
                          self.world, self.group)
            p.halo_unpack(self.recv_lo, self.recv_hi)
            p.adjoint_halo_unpack(self.lam_recv_lo, self.lam_recv_hi)
            p.adjoint_phase(exa.ADJ_REVERSE, lam, dt)

    def get_solution(self, out=None):
        return self.patch.get_solution(out)

    def local_grid(self):
        """(ncell, size, offset) of this rank's slab."""
        return self._local

    def close(self):
        self.patch.close()
