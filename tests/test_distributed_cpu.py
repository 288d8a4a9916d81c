"""Multi-rank logic of the slab decomposition, on CPU with gloo ranks (no GPU involved).

* slab_partition covers the cut axis exactly once;
* halo_exchange (the function the GPU path calls, here on CPU tensors) delivers the lower rank's
  high layer and the upper rank's low layer, for 2 and 3 ranks;
* SlabPatch.adjoint_step (around a fake patch) runs FORWARD, both exchanges on the ring and REVERSE
  in order;
* one emulated time step per rank -- the C library's own face lists with ghost cells
  (exa_build_face_lists, host-only), the halo packing layout of exa_patch_halo_pack/unpack, the
  exchange and the all-reduce(min) of the time step, with the oracle doing each cell's and each
  face's arithmetic -- reproduces the single-domain oracle run of the whole grid.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _paths():
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    for p in (repo, os.path.join(repo, "oracle"), os.path.join(repo, "exahype-engine_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)


def test_slab_partition_covers_axis():
    _paths()
    from exa_distributed import slab_partition
    for n in (1, 7, 81, 100):
        for world in range(1, min(n, 9) + 1):
            parts = [slab_partition(n, world, r) for r in range(world)]
            assert parts[0][0] == 0
            for (f0, c0), (f1, _) in zip(parts, parts[1:]):
                assert f0 + c0 == f1
            assert sum(c for _, c in parts) == n
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1


def _exchange_worker(rank, world, port, q):
    _paths()
    from exa_distributed import halo_exchange
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        send_lo = torch.full((5,), 100.0 * rank + 1)
        send_hi = torch.full((5,), 100.0 * rank + 2)
        recv_lo, recv_hi = torch.zeros(5), torch.zeros(5)
        halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world)
        q.put((rank, recv_lo[0].item(), recv_hi[0].item()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_ring(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pc = mp.start_processes(_exchange_worker, args=(world, _free_port(), q), nprocs=world, start_method="spawn",
                            join=False)
    got = dict((r, (lo, hi)) for r, lo, hi in (q.get(timeout=120) for _ in range(world)))
    while not pc.join(timeout=60):
        pass
    for r in range(world):
        down, up = (r - 1) % world, (r + 1) % world
        assert got[r][0] == 100.0 * down + 2  # lower rank's high layer
        assert got[r][1] == 100.0 * up + 1    # upper rank's low layer


def _euler_cells(rng, ncells, nd, amp=0.04):
    rho = 1.0 + amp * rng.uniform(-1, 1, (ncells, nd))
    u = 0.3 * rng.uniform(-1, 1, (ncells, nd, 3))
    p = 1.0 + amp * rng.uniform(-1, 1, (ncells, nd))
    Q = np.zeros((ncells, nd, 5))
    Q[..., 0] = rho
    Q[..., 1:4] = rho[..., None] * u
    Q[..., 4] = p / 0.4 + 0.5 * rho * (u ** 2).sum(-1)
    return Q.reshape(-1)


NCELL, ORDER, STEPS = (3, 2, 5), 3, 2
SIZE = [1.0, 0.8, 1.2]


def _slab_worker(rank, world, port, q):
    _paths()
    import exa_aderdg as exa
    from exa_distributed import halo_exchange, slab_partition
    from pyoracle import Oracle
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        o = Oracle(3, ORDER)
        n, v, D, nd, nf = o.n, o.v, o.D, o.nd, o.nf
        sq, sf = 6 * nf * D, 6 * nf * v
        luh_global = _euler_cells(np.random.default_rng(1), int(np.prod(NCELL)), nd)
        first, count = slab_partition(NCELL[2], world, rank)
        hz = SIZE[2] / NCELL[2]
        grid = dict(ncell=(NCELL[0], NCELL[1], count), size=[SIZE[0], SIZE[1], count * hz],
                    offset=[0.0, 0.0, first * hz], bc=[exa.BC_PERIODIC, exa.BC_PERIODIC, exa.BC_HALO])
        fl = exa.build_face_lists(3, [grid])
        nc, ng = fl["ncells"], fl["nghost"]
        layer = NCELL[0] * NCELL[1]
        dx = np.array([SIZE[0] / NCELL[0], SIZE[1] / NCELL[1], hz])
        luh = luh_global[first * layer * nd * D:(first + count) * layer * nd * D].copy().reshape(nc, nd * D)
        dtbuf = torch.tensor([min(o.dt(luh[c], dx) for c in range(nc))], dtype=torch.float64)
        dist.all_reduce(dtbuf, op=dist.ReduceOp.MIN)
        for _ in range(STEPS):
            dt = float(dtbuf.item())
            qhb = np.zeros((nc + ng, sq))
            fhb = np.zeros((nc + ng, sf))
            lduh = np.zeros((nc, nd * v))
            for c in range(nc):
                r = o.predictor(luh[c], dx, dt)
                qhb[c], fhb[c] = r["lQhbnd"], r["lFhbnd"]
                lduh[c] = o.volume(r["lFhi"], dx)
            # exa_patch_halo_pack layout: [Q face blocks of the layer][F face blocks of the layer]
            fq, ff = nf * D, nf * v
            face = lambda blk, cells, f, w: blk[cells, f * w:(f + 1) * w].reshape(-1)
            low, high = np.arange(0, layer), np.arange(nc - layer, nc)
            send_lo = torch.from_numpy(np.concatenate([face(qhb, low, 4, fq), face(fhb, low, 4, ff)]))
            send_hi = torch.from_numpy(np.concatenate([face(qhb, high, 5, fq), face(fhb, high, 5, ff)]))
            recv_lo, recv_hi = torch.zeros_like(send_lo), torch.zeros_like(send_hi)
            halo_exchange(send_lo, send_hi, recv_lo, recv_hi, rank, world)
            rl, rh = recv_lo.numpy(), recv_hi.numpy()
            glo, ghi = np.arange(nc, nc + layer), np.arange(nc + layer, nc + 2 * layer)
            qhb[glo, 5 * fq:6 * fq] = rl[:layer * fq].reshape(layer, fq)
            fhb[glo, 5 * ff:6 * ff] = rl[layer * fq:].reshape(layer, ff)
            qhb[ghi, 4 * fq:5 * fq] = rh[:layer * fq].reshape(layer, fq)
            fhb[ghi, 4 * ff:5 * ff] = rh[layer * fq:].reshape(layer, ff)
            for L, R, d in zip(fl["left"], fl["right"], fl["dir"]):
                d = int(d)
                FL, FR = o.riemann(fhb[L, (2 * d + 1) * ff:(2 * d + 2) * ff], fhb[R, 2 * d * ff:(2 * d + 1) * ff],
                                   qhb[L, (2 * d + 1) * fq:(2 * d + 2) * fq], qhb[R, 2 * d * fq:(2 * d + 1) * fq], dx, d)
                fhb[L, (2 * d + 1) * ff:(2 * d + 2) * ff], fhb[R, 2 * d * ff:(2 * d + 1) * ff] = FL, FR
            for c in range(nc):
                du = o.surface(lduh[c], fhb[c], dx)
                luh[c] = o.update(luh[c], du, dt)
            dtbuf = torch.tensor([min(o.dt(luh[c], dx) for c in range(nc))], dtype=torch.float64)
            dist.all_reduce(dtbuf, op=dist.ReduceOp.MIN)
        q.put((rank, first, luh.reshape(-1)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_steps_match_single_domain(world):
    _paths()
    from pyoracle import Oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pc = mp.start_processes(_slab_worker, args=(world, _free_port(), q), nprocs=world, start_method="spawn",
                            join=False)
    parts = sorted((q.get(timeout=300) for _ in range(world)), key=lambda x: x[1])
    while not pc.join(timeout=60):
        pass
    got = np.concatenate([p[2] for p in parts])
    o = Oracle(3, ORDER)
    ref = _euler_cells(np.random.default_rng(1), int(np.prod(NCELL)), o.nd)
    o.run(ref, NCELL, SIZE, STEPS)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12


class _FakeSlabPatch:
    """Stands in for a rank's halo patch: records the adjoint step's calls and fills the send
    buffers with rank-coded values (traces 1000 r + 1 / + 2, lambda 1000 r + 3 / + 4)."""

    def __init__(self, rank):
        self.rank, self.calls, self.got = rank, [], {}

    def adjoint_halo_doubles(self):
        return 4

    def adjoint_phase(self, phase, lam, dt):
        self.calls.append(("phase", phase))

    def halo_pack(self, lo, hi):
        self.calls.append(("pack",))
        lo.fill_(1000.0 * self.rank + 1)
        hi.fill_(1000.0 * self.rank + 2)

    def adjoint_halo_pack(self, lo, hi):
        self.calls.append(("lam_pack",))
        lo.fill_(1000.0 * self.rank + 3)
        hi.fill_(1000.0 * self.rank + 4)

    def halo_unpack(self, lo, hi):
        self.calls.append(("unpack",))
        self.got["traces"] = (lo[0].item(), hi[0].item())

    def adjoint_halo_unpack(self, lo, hi):
        self.calls.append(("lam_unpack",))
        self.got["lam"] = (lo[0].item(), hi[0].item())


def _adjoint_exchange_worker(rank, world, port, q):
    _paths()
    import exa_aderdg as exa
    from exa_distributed import SlabPatch
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        sp = object.__new__(SlabPatch)  # the rank's SlabPatch around a fake patch, CPU tensors
        sp.patch, sp.rank, sp.world, sp.group, sp.stream = _FakeSlabPatch(rank), rank, world, None, None
        sp.send_lo, sp.send_hi, sp.recv_lo, sp.recv_hi = (torch.zeros(3, dtype=torch.float64) for _ in range(4))
        lam = torch.zeros(8, dtype=torch.float64)
        sp.adjoint_step(lam, 1e-3)
        q.put((rank, sp.patch.got, sp.patch.calls, exa.ADJ_FORWARD, exa.ADJ_REVERSE))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_slab_adjoint_step_exchanges_traces_and_lambda(world):
    """SlabPatch.adjoint_step on gloo ranks around a fake patch: FORWARD, both packs, both
    exchanges on the ring (the lower rank's high layer into recv_lo, the upper rank's low layer
    into recv_hi, for the traces and for lambda), both unpacks, then REVERSE."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    pc = mp.start_processes(_adjoint_exchange_worker, args=(world, _free_port(), q), nprocs=world,
                            start_method="spawn", join=False)
    got = {r: (g, c, fw, rv) for r, g, c, fw, rv in (q.get(timeout=120) for _ in range(world))}
    while not pc.join(timeout=60):
        pass
    for r, (g, calls, fw, rv) in got.items():
        down, up = (r - 1) % world, (r + 1) % world
        assert g["traces"] == (1000.0 * down + 2, 1000.0 * up + 1)
        assert g["lam"] == (1000.0 * down + 4, 1000.0 * up + 3)
        names = [c[0] for c in calls]
        assert calls[0] == ("phase", fw) and calls[-1] == ("phase", rv)
        assert set(names[1:-1]) == {"pack", "lam_pack", "unpack", "lam_unpack"}
        assert names.index("pack") < names.index("unpack") and names.index("lam_pack") < names.index("lam_unpack")
