"""Benchmark: ADER-DG DoF-updates/s on 3D compressible Euler, order N=5, 81^3 periodic cells.

One "step" is one ADER-DG time step of the whole grid: CFL dt (fused into the previous step's
update), fused space-time predictor + volume integral, Rusanov on every face, surface integral +
solution update. Seeded synthetic entropy-wave state (the headline workload, 3D Euler N=5 81^3),
inputs resident in HBM; 4.6 GB of luh per step, far above the 126 MB L2, so no L2 flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0). With --gpus N > 1 (torchrun) the grid is 81 x 81 x 81N cells cut
into one 81^3 slab per rank (weak scaling): each step exchanges the slabs' face traces with the
neighbours and all-reduces the CFL dt over NCCL; timing is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "exahype-engine_b200"))

NCELL = (81, 81, 81)
ORDER = 5
NVAR = 5
METRIC = "ADER-DG DoF-updates/s (3D Euler N=5, 81^3 cells)"
# CPU baseline sample: the 27^3 corner block of the same state (same dx, same dt scale), with
# outflow faces so that the block's edges add no jump
SAMPLE_NCELL = (27, 27, 27)


def euler_sample_state():
    """The benchmark's entropy wave at the nodes of its 27^3 corner block (dx = 1/81)."""
    import exa_scenarios as sc
    size = [SAMPLE_NCELL[k] / NCELL[k] for k in range(3)]
    return sc.EntropyWave(3, 0).state(sc.nodal_positions(SAMPLE_NCELL, size, ORDER)).reshape(-1), size


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncell", type=int, default=81, help="cells per axis (81 = the benchmark workload)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--workload", default="euler3d",
                    choices=["euler3d", "swe_batched", "acoustic_adjoint", "elastic3d"],
                    help="euler3d: the headline workload; swe_batched: 512 wall-bounded 2D SWE grids, N=4; "
                         "acoustic_adjoint: misfit gradient of a 32^3 N=4 acoustic run, 300 steps; "
                         "elastic3d: layered elastic medium, N=7, 48^3 cells, absorbing faces, 10 Hz source")
    ap.add_argument("--ncell-elastic", type=int, default=48)
    ap.add_argument("--swe-grids", type=int, default=512, help="swe_batched: number of grids (512 = the workload)")
    ap.add_argument("--elastic-active", action="store_true",
                    help="elastic3d: start from a smooth random velocity field so that every cell iterates")
    ap.add_argument("--fd-directions", type=int, default=16, help="acoustic_adjoint: finite-difference checks")
    ap.add_argument("--predictor-variant", type=int, default=-1, choices=[-1, 0, 1],
                    help="predictor launch form: -1 the one measured as faster on the first state (default), "
                         "0 one cell group per CTA, 1 persistent (mixed: 2 or 3 CTAs per SM)")
    ap.add_argument("--update-variant", type=int, default=-1, choices=[-1, 0, 1],
                    help="launch form of the Rusanov and update kernels: 0 per-thread loads, 1/-1 bulk copies")
    ap.add_argument("--max-picard", type=int, default=0,
                    help="euler3d: a fixed Picard sweep count (the reference's UseMaxPicardIterations mode); "
                         "0 = the residual test (the benchmark); used to measure per-sweep costs")
    ap.add_argument("--no-workloads", action="store_true",
                    help="euler3d at N=1: skip the short runs of the other configurations (the workloads record)")
    return ap.parse_args()


def amr_limiter_record(exa, solver, torch, stream, luh_dev, cells, nd, hbm_peak, fp64_peak, reps=5):
    """The mesh-level and limiter kernels on the benchmark state (CUDA events on `stream`):
    the discrete maximum principle over every cell, the DG -> FV -> DG projections (P = 11
    subcells, 2 ghost layers) over a block of cells, and the prolongation of 27 children per coarse
    cell and their grouped restriction. Algorithmic bytes count every block read or written once."""
    V = solver.nvar
    blk = nd * V * 8.0
    out = {}

    def timed(fn):
        fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def rec(ms, nbytes, what):
        gbs = nbytes / (ms * 1e-3) / 1e9
        return {"ms": ms, "algorithmic_bytes": nbytes, "gbs": gbs,
                "frac_of_measured_hbm": gbs / hbm_peak if hbm_peak else None, "work": what}

    with torch.cuda.stream(stream):
        nobs = V
        bmin = torch.full((cells * 6 * nobs,), -1e30, dtype=torch.float64, device="cuda")
        bmax = torch.full((cells * 6 * nobs,), 1e30, dtype=torch.float64, device="cuda")
        ok = torch.zeros(cells, dtype=torch.uint8, device="cuda")
        ms = timed(lambda: solver.limiter_dmp(luh_dev, nobs, 1e-4, 1e-3, bmin, bmax, ok))
        out["dmp"] = rec(ms, cells * (blk + 2 * 6 * nobs * 8 + 2 * 2 * nobs * 8 + 1),
                         "%d cells, %d observables (nodes, Lobatto nodes, 11^3 subcell means)" % (cells, nobs))
        # the projections onto the Gauss-Lobatto nodes (3 n^4 multiply-adds per observable) and
        # the subcell means (n^3 P + n^2 P^2 + n P^3) bound it, not memory
        n_, P_ = solver.order + 1, 2 * solver.order + 1
        fma_cell = nobs * (3 * n_ ** 4 + n_ ** 3 * P_ + n_ ** 2 * P_ ** 2 + n_ * P_ ** 3)
        tf = 2.0 * fma_cell * cells / (ms * 1e-3) / 1e12
        out["dmp"].update({"fp64_tflops": tf, "algorithmic_flops": 2.0 * fma_cell * cells,
                           "frac_of_measured_fp64": tf / fp64_peak if fp64_peak else None})
        del bmin, bmax, ok
        nl = min(cells, 32768)
        ghost = 2
        lim = torch.zeros(nl * solver.limiter_patch_size(ghost), dtype=torch.float64, device="cuda")
        part = luh_dev[: nl * nd * V]
        back = torch.empty_like(part)
        sub = (2 * solver.order + 1) ** 3 * V * 8.0
        ms = timed(lambda: solver.limiter_project_on_fv(part, lim, ghost))
        out["project_on_fv"] = rec(ms, nl * (blk + sub), "%d cells -> 11^3 subcells + 2 ghost layers" % nl)
        ms = timed(lambda: solver.limiter_project_on_dg(lim, back, ghost))
        out["project_on_dg"] = rec(ms, nl * (blk + sub), "%d cells" % nl)
        del lim, back
        nc = min(cells, 4096)
        kids = [(i1, i2, i3) for i3 in range(3) for i2 in range(3) for i1 in range(3)]
        jobs = torch.tensor([[27 * c + k, c, 1, *kids[k]] for c in range(nc) for k in range(27)], dtype=torch.int32,
                            device="cuda")
        coarse = luh_dev[: nc * nd * V].clone()
        fine = torch.empty(27 * nc * nd * V, dtype=torch.float64, device="cuda")
        ptr = torch.arange(0, 27 * nc + 1, 27, dtype=torch.int32, device="cuda")
        ms = timed(lambda: solver.amr_volume(exa.AMR_PROLONGATE, fine, coarse, jobs))
        out["volume_prolongation"] = rec(ms, nc * 28 * blk, "%d coarse cells x 27 children" % nc)
        ms = timed(lambda: solver.amr_volume(exa.AMR_RESTRICT, fine, coarse, jobs, group_ptr=ptr))
        out["volume_restriction"] = rec(ms, nc * 29 * blk, "%d coarse cells <- 27 children each" % nc)
        del coarse, fine, jobs, ptr
    out["status_bits"] = solver.status()
    return out


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region (every 200 ms).

    Reads the same counters nvidia-smi reports (clocks.sm, clocks.max.sm, clocks_event_reasons)
    through NVML in this process, so that sampling starts no child process while the timed region
    is being enqueued; falls back to nvidia-smi where NVML is unavailable. The first sample is taken
    before __enter__ returns."""

    FIELDS = "clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.t = threading.Thread(target=self.run, daemon=True)
        self.nvml = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.handle = pynvml.nvmlDeviceGetHandleByIndex(index)
        except Exception:
            self.nvml = None

    def sample(self):
        try:
            if self.nvml is not None:
                n = self.nvml
                sm = n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)
                mx = n.nvmlDeviceGetMaxClockInfo(self.handle, n.NVML_CLOCK_SM)
                r = n.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                flags = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                         n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
                self.samples.append([str(sm), str(mx)] + ["Active" if r & f else "Not Active" for f in flags])
            else:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
        except Exception:
            pass

    def run(self):
        while not self.stop.wait(0.2):
            self.sample()

    def __enter__(self):
        self.sample()
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)
        self.sample()

    def summary(self):
        sm = [float(s[0]) for s in self.samples if len(s) >= 6 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if len(s) >= 6 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples if len(s) >= 6 for k in range(4) if s[2 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples),
                "source": "NVML" if self.nvml is not None else "nvidia-smi"}


def flops_per_cell_step(sweeps):
    """Algorithmic FLOPs of one cell-step of the reference algorithm (3D Euler, N=5):
    395,280 per Picard sweep (contractions 2(d+1) n^(d+2) v + n^(d+1) (flux 40 + 5v)),
    116,640 for time averaging, extrapolation and volume integral, 31,000 for faces, update, CFL."""
    return 395280.0 * sweeps + 116640.0 + 31000.0


PRED_BYTES_PER_CELL = 8.0 * (1080 + 1080 + 1080 + 1080)  # luh in; lduh, lQhbnd, lFhbnd out
# DRAM bytes per cell of one predictor launch measured by ncu on a 27^3 block (19,683 cells):
# 172.00 MB read + 466.63 MB written
PRED_DRAM_BYTES_PER_CELL = (171.954432e6 + 462.412288e6) / 19683
# FP64 operations the FP64 predictor (3D Euler N=5) executes per cell, from ncu's SASS counters
# (2 dfma + dadd + dmul, predicated on) of launches on a 27^3 block with a fixed 2 and 4 sweeps:
# 14,437,695,109 and 31,836,609,564 per launch. Sweep 0 (closed form) with the tail costs less
# than the algorithmic count credits it; a further sweep costs more (residual, rhs scaling).
PRED_EXEC_FLOPS_SWEEP0_TAIL = 291532.69
PRED_EXEC_FLOPS_PER_SWEEP = 441978.22


def cpu_baseline(steps=20, kind="reference"):
    """The reference's own generic kernels (oracle/_ref) with OpenMP on every host core, on a
    27^3 periodic block of the benchmark state. Returns DoF-updates/s."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import exa_scenarios as sc
    from pyoracle import Oracle, RefKernels
    luh, size = euler_sample_state()
    try:
        runner = RefKernels(3, ORDER)
    except Exception:
        runner, kind = Oracle(3, ORDER), "port"
    cores = os.cpu_count()
    runner.run(luh, SAMPLE_NCELL, size, 1, walls=3, nthreads=cores)  # warm-up
    t0 = time.perf_counter()
    _, _, pic = runner.run(luh, SAMPLE_NCELL, size, steps, walls=3, nthreads=cores, want_picard=True)
    el = time.perf_counter() - t0
    cells = int(np.prod(SAMPLE_NCELL))
    dof = cells * NVAR * (ORDER + 1) ** 3 * steps
    # the reference kernels report the break index of the Picard loop (3D), i.e. sweeps - 1
    sweeps = float(np.mean(pic)) + (1.0 if kind == "reference" else 0.0)
    out = {"value": dof / el, "unit": "DoF-updates/s", "cores": cores, "kind": kind, "picard_sweeps_mean": sweeps,
           "sample": "%dx%dx%d corner block of the 81^3 N=5 Euler state (dx=1/81, outflow faces), %d steps, %.1f s"
                     % (SAMPLE_NCELL + (steps, el))}
    # the reference's generated optimised kernels (KernelGenerator, plain loops; the libxsmm variant
    # cannot be generated: its submodule is empty), same sample and driver order
    try:
        from pyoracle import KGKernels
        kg = KGKernels(ORDER)
        luh2, _ = euler_sample_state()
        kg.run(luh2, SAMPLE_NCELL, size, 1, walls=3, nthreads=cores)
        t0 = time.perf_counter()
        _, _, pk = kg.run(luh2, SAMPLE_NCELL, size, steps, walls=3, nthreads=cores, want_picard=True)
        el2 = time.perf_counter() - t0
        out["kernelgenerator"] = {"value": dof / el2, "unit": "DoF-updates/s", "cores": cores,
                                  "kind": "reference (KernelGenerator plain-loop output)",
                                  "picard_sweeps_mean": float(np.mean(pk)),
                                  "sample": "the same block and steps, %.1f s" % el2}
    except Exception as e:  # not generated on this machine
        out["kernelgenerator"] = {"value": None, "unavailable": str(e)}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    W, K = args.warmup, args.steps
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import exa_scenarios as sc
    from pyoracle import Oracle, RefKernels
    kind = "reference"
    try:
        runner = RefKernels(3, ORDER)
    except Exception:
        runner, kind = Oracle(3, ORDER), "port"
    luh, size = euler_sample_state()
    cores = os.cpu_count()
    runner.run(luh, SAMPLE_NCELL, size, W, walls=3, nthreads=cores)
    t0 = time.perf_counter()
    _, _, pic = runner.run(luh, SAMPLE_NCELL, size, K, walls=3, nthreads=cores, want_picard=True)
    el = time.perf_counter() - t0
    # Picard sweeps per cell: the reference kernels return the break index (3D), i.e. sweeps - 1
    sweeps = float(np.mean(pic)) + (1.0 if kind == "reference" else 0.0)
    cells = int(np.prod(SAMPLE_NCELL))
    value = cells * NVAR * (ORDER + 1) ** 3 * K / el
    sample = "%dx%dx%d corner block of the 81^3 N=5 Euler state (dx=1/81, outflow faces) per step" % SAMPLE_NCELL
    line = {"metric": METRIC, "value": value, "unit": "DoF-updates/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": 1e3 * el / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "3D Euler N=5 entropy wave, generic kernels, OpenMP over cells",
                       "sample": sample, "cells_per_step": cells},
            "picard_sweeps_mean": sweeps,
            "cpu_baseline": {"value": value, "unit": "DoF-updates/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "DoF-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def swe_cpu_sample(specs, states, steps=1, min_s=1.0):
    """Reference generic kernels (oracle/_ref, SWE N=4, walls) on the first 8 grids, OpenMP."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    from pyoracle import Oracle, RefKernels, PDE_SWE
    kind = "reference"
    try:
        runner = RefKernels(2, 4, pde="swe")
    except Exception:
        runner, kind = Oracle(2, 4, pde=PDE_SWE), "port"
    cores = os.cpu_count()
    sample = list(zip(specs, states))[:8]
    cells = sum(sp["ncell"][0] * sp["ncell"][1] for sp, _ in sample)
    work = [st.copy() for _, st in sample]
    # whole steps of the 8 grids, repeated until at least min_s seconds have passed
    nsteps = 0
    t0 = time.perf_counter()
    while True:
        for (sp, _), st in zip(sample, work):
            runner.run(st, sp["ncell"], sp["size"], steps, walls=True, nthreads=cores)
        nsteps += steps
        el = time.perf_counter() - t0
        if el >= min_s:
            break
    return {"value": cells * 4 * 25 * nsteps / el, "unit": "DoF-updates/s", "cores": cores, "kind": kind,
            "sample": "first 8 of the 512 grids (%d cells), %d steps, %.1f s" % (cells, nsteps, el)}


def swe_flops_per_cell_step(sweeps):
    """Algorithmic FP64 work of the 2D SWE N=4 predictor per cell (d=2, n=5, v=4, nd=25), per
    Picard sweep: 2(d+1) n^(d+2) v = 15,000 for the Kxi contractions and the iK1 time solve,
    2 d n^(d+2) v = 10,000 for the NCP gradients (dudx along every line), and n^(d+1) (flux 16 +
    NCP 4 + rhs 5v) = 5,000; per cell once: 1,000 for the time averages, 2,000 for the volume
    integral, 1,600 for the face extrapolation."""
    return 30000.0 * sweeps + 4600.0


def run_swe_batched(args):
    """512 independent wall-bounded 2D shallow-water grids (16^2..128^2 cells, N=4), each with its
    own CFL time step, advanced together: one CUDA graph launch per step."""
    import torch
    import exa_aderdg as exa
    import exa_scenarios as sc
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs, states = sc.swe_batched(ngrids=args.swe_grids)
    cells = sum(sp["ncell"][0] * sp["ncell"][1] for sp in specs)
    dof_step = cells * 4 * 25
    solver = exa.Solver(exa.PDE_SWE, 2, 4)
    patch = exa.Patch(solver, specs)
    patch.set_solution(np.concatenate(states))
    stream = torch.cuda.ExternalStream(patch.stream)
    W, K = args.warmup, args.steps
    patch.step(W)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        ev0.record(stream)
        patch.step(K)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / K
    sweeps = patch.stats()["picard_mean"]
    # the predictor alone (same state, each grid's own dt)
    reps = 3
    ev0.record(stream)
    for _ in range(reps):
        patch.step_phase(exa.PHASE_PREDICTOR, 0.0)
    ev1.record(stream)
    ev1.synchronize()
    pred_ms = ev0.elapsed_time(ev1) / reps
    flops_launch = swe_flops_per_cell_step(sweeps) * cells
    fp64_peak = fp64_peak_tflops()
    achieved = flops_launch / (pred_ms * 1e-3) / 1e12
    line = {"metric": "ADER-DG DoF-updates/s (batched 2D SWE N=4, %d grids)" % len(specs), "value": dof_step / (ms * 1e-3),
            "unit": "DoF-updates/s", "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "%d 2D shallow-water grids (h,hu,hv,b; NCP), sides U{16..128}, N=4, " % len(specs) +
                                   "reflective walls, per-grid CFL dt, one CUDA graph per step",
                       "cells": cells, "dof_per_step": dof_step},
            "picard_sweeps_mean": sweeps, "status_bits": patch.status(),
            "roofline": {"bound": "fp64", "kernel": "predictor_kernel (SWE, NCP)", "achieved": achieved,
                         "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                         "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run", "traffic": None,
                         "launch_ms": pred_ms, "algorithmic_flops_per_launch": flops_launch},
            "gpu_launches": K * 5, "clocks": clocks.summary()}
    if not args.no_cpu:
        line["cpu_baseline"] = swe_cpu_sample(specs, states)
    patch.close()
    return line


def run_acoustic_adjoint(args):
    """Gradient of a receiver misfit with respect to per-cell (rho, c) and the initial pressure:
    3D acoustics, N=4, 32^3 periodic cells, 300 fixed steps, 64 receivers, binomial checkpointing
    with 20 stored states. One timed "step" is one whole gradient (forward run with the receivers,
    reverse sweep with recomputation). Checked against central finite differences (h = 1e-6)
    of the GPU forward model along seeded random directions."""
    import torch
    import exa_aderdg as exa
    from exa_adjoint import Misfit, WaveInversion, acoustic_model, cfl_dt, fd_directional
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ncell, size, order, nsteps, snaps = (32, 32, 32), [1.0, 1.0, 1.0], 4, 300, 20
    m = acoustic_model(ncell, size, order, seed=0, width=0.05)
    dt = cfl_dt(ncell, size, order, float(m["c_true"].max()))
    inv = WaveInversion(exa.PDE_ACOUSTIC, ncell, size, order, dt, nsteps, m["receivers"], snaps=snaps)
    dev = torch.device("cuda")
    p0 = torch.tensor(m["p0"], device=dev)
    data = inv.forward_traces(inv.assemble(torch.tensor(np.stack([m["rho"], m["c_true"]], -1), device=dev), p0))
    params0 = torch.tensor(np.stack([m["rho"], m["c"]], -1), device=dev)
    stream = inv.stream

    def gradient():
        params = params0.clone().requires_grad_(True)
        field = p0.clone().requires_grad_(True)
        J = Misfit.apply(params, field, inv, data)
        J.backward()
        return J.detach(), params.grad, field.grad

    W, K = max(args.warmup, 1), max(args.steps, 1)
    for _ in range(W):
        gradient()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        ev0.record(stream)
        for _ in range(K):
            J, gp, gf = gradient()
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / K
    # forward step and adjoint step alone
    luh0 = inv.assemble(params0, p0)
    inv._set(luh0, 0)
    torch.cuda.synchronize()
    ev0.record(stream)
    inv.patch.step(20, dt)
    ev1.record(stream)
    ev1.synchronize()
    ms_fwd = ev0.elapsed_time(ev1) / 20
    lam = torch.randn((inv.ncells, inv.nd, inv.D), dtype=torch.float64, device=dev)
    inv._set(luh0, 0)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(20):
        inv.patch.adjoint_step(lam, dt)
    ev1.record(stream)
    ev1.synchronize()
    ms_adj = ev0.elapsed_time(ev1) / 20
    # finite differences along seeded directions
    rng = np.random.default_rng(1)
    errs, kinks = [], []
    dirder, cond_ad, cond_fd, err_scaled = [], [], [], []
    cgrid = params0[:, 1].reshape(ncell[2], ncell[1], ncell[0])

    def kink_faces(vc, h):
        """Faces whose Rusanov wave speed max(c_L, c_R) switches sides between c + h v and c - h v,
        and the mask of the cells on either side of them."""
        cp_ = (params0[:, 1] + h * vc).reshape(cgrid.shape)
        cm_ = (params0[:, 1] - h * vc).reshape(cgrid.shape)
        cnt = 0
        mask = torch.zeros_like(cp_, dtype=torch.bool)
        for ax in range(3):
            dp = cp_ - torch.roll(cp_, -1, dims=ax)
            dm = cm_ - torch.roll(cm_, -1, dims=ax)
            k = (dp >= 0) != (dm >= 0)
            cnt += int(k.sum())
            mask |= k | torch.roll(k, 1, dims=ax)
        return cnt, mask.reshape(-1)

    errs_smooth = []
    for _ in range(args.fd_directions):
        vp = torch.tensor(rng.normal(size=tuple(params0.shape)), device=dev) * params0
        vf = torch.tensor(rng.normal(size=tuple(p0.shape)), device=dev)
        fd, fd_scale = fd_directional(inv, params0, p0, vp, vf, data, h=1e-6, with_scale=True)
        ad = float((gp * vp).sum() + (gf * vf).sum())
        errs.append(abs(fd - ad) / max(abs(fd), 1e-300))
        # cancellation in the two sums: sum of |terms| over |sum|; a relative error this many
        # times the rounding of one term is what the sums themselves allow
        ad_scale = float((gp * vp).abs().sum() + (gf * vf).abs().sum())
        dirder.append(ad)
        err_scaled.append(abs(fd - ad) / max(ad_scale, 1e-300))
        cond_ad.append(ad_scale / max(abs(ad), 1e-300))
        cond_fd.append(fd_scale / max(abs(fd), 1e-300))
        nk, mask = kink_faces(vp[:, 1], 1e-6)
        kinks.append(nk)
        # the same direction with c left unperturbed next to those faces: the misfit is smooth along
        # it, so its FD check isolates the Rusanov max switches from the adjoint itself
        if nk:
            vq = vp.clone()
            vq[mask, 1] = 0.0
            fd2 = fd_directional(inv, params0, p0, vq, vf, data, h=1e-6)
            ad2 = float((gp * vq).sum() + (gf * vf).sum())
            errs_smooth.append(abs(fd2 - ad2) / max(abs(fd2), 1e-300))
        else:
            errs_smooth.append(errs[-1])
    errs_all = list(errs)
    cells = inv.ncells
    dof_step = cells * inv.V * inv.nd
    line = {"metric": "ADER-DG adjoint gradient, simulated DoF-updates/s (3D acoustic N=4, 32^3, 300 steps)",
            "value": nsteps * dof_step / (ms * 1e-3), "unit": "DoF-updates/s", "n_gpus": 1, "steps": K,
            "warmup": W, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "misfit gradient w.r.t. per-cell (rho, c) and initial pressure: 3D acoustics "
                                   "N=4, 32^3 periodic cells, fixed dt, %d Picard sweeps, %d steps, 64 receivers, "
                                   "binomial checkpointing with %d stored states" % (order + 1, nsteps, snaps),
                       "cells": cells, "dof_per_step": dof_step, "recomputed_steps": inv.recompute_steps,
                       "dt": dt},
            "forward_ms_per_step": ms_fwd, "adjoint_ms_per_step": ms_adj,
            "gradient_s": ms * 1e-3, "misfit": float(J),
            "fd_check": {"directions": len(errs), "h": 1e-6, "max_rel_err": max(errs) if errs else None,
                         "median_rel_err": float(np.median(errs)) if errs else None,
                         "rel_err_per_direction": errs_all,
                         "kink_faces_per_direction": kinks,
                         "directional_derivative_per_direction": dirder,
                         "cancellation_adjoint_per_direction": cond_ad,
                         "cancellation_fd_per_direction": cond_fd,
                         "cancellation": "sum of |terms| / |sum| of the adjoint dot product g.v and of "
                                         "the finite difference's trace sum",
                         "abs_err_over_sum_abs_terms_per_direction": err_scaled,
                         "max_abs_err_over_sum_abs_terms": max(err_scaled) if err_scaled else None,
                         "rel_err_per_direction_kink_free": errs_smooth,
                         "max_rel_err_kink_free": max(errs_smooth) if errs_smooth else None,
                         "kink_free": "the same directions with the c perturbation zeroed on the cells next "
                                      "to faces where max(c_L, c_R) switches sides between theta +- h v"},
            # per gradient: the schedule's forward steps plus the final one (4 kernels each:
            # predictor, Riemann, update, advance) and one adjoint step per step (3 kernels:
            # forward predictor, adjoint faces, adjoint predictor); the receivers are torch ops
            "gpu_launches": K * (4 * (inv.recompute_steps + 1) + 3 * nsteps), "clocks": clocks.summary()}
    if not args.no_cpu:
        # the reference has no adjoint: its generic kernels (fixed Picard count) time forward steps
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from pyoracle import RefKernels
        try:
            ref, kind = RefKernels(3, order, "acousticfixed", 2), "reference"
            luh = luh0.cpu().numpy().reshape(-1).copy()
            cores = os.cpu_count()
            ref.run(luh, ncell, size, 1, fixed_dt=dt, nthreads=cores)
            t0 = time.perf_counter()
            ref.run(luh, ncell, size, 2, t0=dt, fixed_dt=dt, nthreads=cores)
            el = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": 2 * dof_step / el, "unit": "DoF-updates/s", "cores": cores, "kind": kind,
                                    "sample": "2 forward steps of the 32^3 N=4 acoustic model (fixed Picard count); "
                                              "the reference has no adjoint, %.1f s" % el}
        except Exception as e:  # reference kernels not built on this machine
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    inv.close()
    return line


def fp64_peak_tflops():
    """FP64 peak measured here with cuBLAS DGEMM 8192^3 (MEASURED_PEAKS.json carries no FP64 figure)."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    for _ in range(3):
        torch.matmul(a, b)
    g1.record()
    g1.synchronize()
    peak = 3 * 2 * 8192.0 ** 3 / (g0.elapsed_time(g1) * 1e-3) / 1e12
    del a, b
    return peak


def elastic_flops_per_cell_step(sweeps):
    """Algorithmic FLOPs of one cell-step, 3D elastic flux form, N=7 (n=8, v=9, D=12):
    per Picard sweep 2(d+1) n^(d+2) v = 2,359,296 (contractions and the time solve) plus
    n^(d+1) (flux 75 + 5v) = 491,520; tail 2 n^(d+1)(d v + D) + 4 d n^d (v + D) + 2 d n^(d+1) v
    = 669,696 (time averaging, extrapolation, volume integral)."""
    return 2850816.0 * sweeps + 669696.0


def cells_of(ncell):
    return int(np.prod(ncell))


def run_elastic3d(args):
    """Layered elastic medium (6 seeded horizontal layers), order 7, 48^3 cells on a 10 km cube,
    absorbing (outflow) faces, 10 Hz Ricker source on the vertical velocity at a seeded interior
    point, CFL time step. The streamed predictor (Picard iterates in global scratch) runs it."""
    import torch
    import exa_aderdg as exa
    import exa_scenarios as sc
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.ncell_elastic
    ncell, size, order = (n, n, n), [10.0, 10.0, 10.0], 7
    luh0, table = sc.elastic_layers(ncell, size, order, seed=0)
    if args.elastic_active:
        x = sc.nodal_positions(ncell, size, order)
        q = luh0.reshape(cells_of(ncell), -1, 12)
        for k in range(3):
            q[..., k] = 0.1 * np.sin(2 * np.pi * (k + 1) * x[..., (k + 1) % 3] / size[0])
    src = sc.elastic_source(size, seed=0, f0=10.0, width=10.0 / n)
    solver = exa.Solver(exa.PDE_ELASTIC, 3, order, npar=3)
    patch = exa.Patch(solver, [dict(ncell=ncell, size=size, bc=exa.BC_OUTFLOW)])
    patch.set_point_source(src[:3], src[3], src[4], src[5], src[6], int(src[7]))
    patch.set_solution(luh0)
    stream = torch.cuda.ExternalStream(patch.stream)
    cells = int(np.prod(ncell))
    dof_step = cells * 9 * (order + 1) ** 3
    W, K = args.warmup, args.steps
    patch.step(W)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        ev0.record(stream)
        patch.step(K)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / K
    st = patch.stats()
    sweeps = st["picard_mean"]
    # the predictor alone (same state, same dt)
    reps = 3
    ev0.record(stream)
    for _ in range(reps):
        patch.step_phase(exa.PHASE_PREDICTOR, 0.0)
    ev1.record(stream)
    ev1.synchronize()
    pred_ms = ev0.elapsed_time(ev1) / reps
    flops_launch = elastic_flops_per_cell_step(sweeps) * cells
    fp64_peak = fp64_peak_tflops()
    achieved = flops_launch / (pred_ms * 1e-3) / 1e12
    line = {"metric": "ADER-DG DoF-updates/s (3D elastic N=7, 48^3 cells)", "value": dof_step / (ms * 1e-3),
            "unit": "DoF-updates/s", "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "3D elastic (velocity-stress, flux form, per-cell rho/cp/cs), N=7, %d^3 cells on "
                                   "[0,10 km]^3, 6 seeded horizontal layers, outflow faces, 10 Hz Ricker source, "
                                   "CFL 0.9; streamed predictor" % n,
                       "cells": cells, "dof_per_step": dof_step, "l2": "inputs 5.4 GB > L2, no flush needed"},
            "picard_sweeps_mean": sweeps, "status_bits": patch.status(),
            "initial_state": "smooth random velocity field" if args.elastic_active else "at rest (source-driven)",
            "roofline": {"bound": "fp64", "kernel": "predictor_streamed_kernel", "achieved": achieved,
                         "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                         "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run", "traffic": None,
                         "launch_ms": pred_ms, "algorithmic_flops_per_launch": flops_launch},
            "gpu_launches": K * 5, "clocks": clocks.summary()}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        from pyoracle import RefKernels
        try:
            ref = RefKernels(3, order, "elastic", 3, source=src)
            sample = (12, 12, 12)
            lsm, _ = sc.elastic_layers(sample, [10.0 * k / n for k in sample], order, seed=0)
            cores = os.cpu_count()
            if args.elastic_active:
                xs = sc.nodal_positions(sample, [10.0 * k / n for k in sample], order)
                qs = lsm.reshape(cells_of(sample), -1, 12)
                for k in range(3):
                    qs[..., k] = 0.1 * np.sin(2 * np.pi * (k + 1) * xs[..., (k + 1) % 3] / size[0])
            t0 = time.perf_counter()
            ref.run(lsm, sample, [10.0 * k / n for k in sample], 2, walls=3, nthreads=cores)
            el = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": int(np.prod(sample)) * 9 * 512 * 2 / el, "unit": "DoF-updates/s",
                                    "cores": cores, "kind": "reference",
                                    "sample": "12^3 block of the same medium at the same dx, 2 steps, %.1f s" % el}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    patch.close()
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    runners = {"swe_batched": run_swe_batched, "acoustic_adjoint": run_acoustic_adjoint,
               "elastic3d": run_elastic3d}
    if args.workload in runners:
        print(json.dumps(runners[args.workload](args)), flush=True)
        return
    import torch
    import torch.distributed as dist
    import exa_aderdg as exa
    import exa_scenarios as sc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    W, K = args.warmup, args.steps
    ncell = (args.ncell,) * 3
    cells = int(np.prod(ncell))
    dof_step = cells * NVAR * (ORDER + 1) ** 3

    precision = exa.PREC_MIXED if args.precision == "mixed" else exa.PREC_FP64
    solver = exa.Solver(exa.PDE_EULER, 3, ORDER, precision=precision, max_picard=args.max_picard)
    solver.set_update_variant(args.update_variant)
    solver.predictor_variant = args.predictor_variant
    # every rank owns one 81^3 slab of an 81 x 81 x (81 N) periodic grid (dx = 1/81 everywhere)
    from exa_distributed import SlabPatch
    slab = SlabPatch(solver, (ncell[0], ncell[1], ncell[2] * world), [1.0, 1.0, float(world)], rank=rank,
                     world=world)
    patch = slab.patch
    lnc, lsize, loff = slab.local_grid()
    wave = sc.EntropyWave(3, 0)
    luh0 = wave.state(sc.nodal_positions(lnc, lsize, ORDER, offset=loff)).reshape(-1)
    slab.set_local_solution(luh0)
    stream = slab.stream

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident steps (graph per step), CUDA events on the patch's stream ----
    slab.step(W)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        ev0.record(stream)
        slab.step(K)
        ev1.record(stream)
        ev1.synchronize()
        barrier()
    ms = ev0.elapsed_time(ev1) / K
    ms_t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    stats = patch.stats()
    status = patch.status()
    t_now, dt_now = patch.time()
    # accuracy after W+K steps: rho against the exact entropy wave on every 37th cell
    sol = patch.get_solution().reshape(cells, -1)
    pick = np.arange(0, cells, 37)
    xs = sc.nodal_positions(lnc, lsize, ORDER, offset=loff).reshape(cells, -1, 3)[pick]
    exact = wave.state(xs, float(t_now[0]))
    l2_exact, linf_exact = sc.l2_linf_error(sol[pick], exact, ORDER, 3)

    # the other precision on the same state and step count, for the mixed-vs-FP64 comparison
    other = None
    if rank == 0:
        oprec = exa.PREC_FP64 if precision == exa.PREC_MIXED else exa.PREC_MIXED
        s2 = exa.Solver(exa.PDE_EULER, 3, ORDER, precision=oprec)
        p2 = exa.Patch(s2, [dict(ncell=ncell, size=[1.0, 1.0, 1.0])])
        p2.set_solution(luh0)
        st2 = torch.cuda.ExternalStream(p2.stream)
        p2.step(W)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(st2)
        p2.step(K)
        a1.record(st2)
        a1.synchronize()
        ms2 = a0.elapsed_time(a1) / K
        sol2 = p2.get_solution().reshape(cells, -1)
        d = sol2 - sol
        l2o, linfo = sc.l2_linf_error(sol2[pick], exact, ORDER, 3)
        other = {"precision": "fp64" if oprec == exa.PREC_FP64 else "mixed",
                 "value": dof_step / (ms2 * 1e-3), "ms_per_step": ms2,
                 "speedup_of_mixed_over_fp64": (ms2 / ms) if oprec == exa.PREC_FP64 else (ms / ms2),
                 "l2_rho_vs_exact": l2o, "linf_rho_vs_exact": linfo,
                 "max_abs_diff_vs_this_run": float(np.max(np.abs(d))),
                 "l2_rel_diff_vs_this_run": float(np.linalg.norm(d) / np.linalg.norm(sol)),
                 "status_bits": p2.status()}
        p2.close()
        s2.close()
        del sol2, d

    # ---- dominant kernel (predictor) timed alone, events on the same stream ----
    import ctypes
    lib = exa.load_library()
    nd, nf = (ORDER + 1) ** 3, (ORDER + 1) ** 2
    luh_dev = torch.empty(cells * nd * NVAR, dtype=torch.float64, device="cuda")
    patch.get_solution(luh_dev)
    lduh = torch.empty(cells * nd * NVAR, dtype=torch.float64, device="cuda")
    qhb = torch.empty(cells * 6 * nf * NVAR, dtype=torch.float64, device="cuda")
    fhb = torch.empty_like(qhb)
    pic = torch.zeros(cells, dtype=torch.int32, device="cuda")
    dxv = [1.0 / ncell[0]] * 3
    dtv = float(dt_now[0])
    with torch.cuda.stream(stream):
        for _ in range(2):
            solver.fused_predictor_volume_integral(luh_dev, lduh, qhb, fhb, dxv, dtv, picard=pic, stream=patch.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record(stream)
        for _ in range(reps):
            solver.fused_predictor_volume_integral(luh_dev, lduh, qhb, fhb, dxv, dtv, picard=pic, stream=patch.stream)
        e1.record(stream)
    e1.synchronize()
    pred_ms = e0.elapsed_time(e1) / reps
    mean_sweeps = float(pic.double().mean().item())
    # the HBM-bound kernels alone on the patch (Rusanov on every face; surface integral + update +
    # CFL), events on the patch stream; the state advances, nothing reads it afterwards
    phase_ms = {}
    for name, ph in (("riemann", exa.PHASE_FACES), ("update", exa.PHASE_UPDATE)):
        e0.record(stream)
        for _ in range(reps):
            patch.step_phase(ph, 0.0)
        e1.record(stream)
        e1.synchronize()
        phase_ms[name] = e0.elapsed_time(e1) / reps
    nface = 3 * cells
    hbm_peak = peaks()[0].get("hbm_gbs")
    hbm = {"riemann": {"ms": phase_ms["riemann"], "algorithmic_bytes": nface * 8640.0,
                       "gbs": nface * 8640.0 / (phase_ms["riemann"] * 1e-3) / 1e9},
           "update": {"ms": phase_ms["update"], "algorithmic_bytes": cells * 34560.0,
                      "gbs": cells * 34560.0 / (phase_ms["update"] * 1e-3) / 1e9}}
    for v in hbm.values():
        v["frac_of_measured_hbm"] = v["gbs"] / hbm_peak if hbm_peak else None
    fp64_peak = fp64_peak_tflops()
    amr_lim = (amr_limiter_record(exa, solver, torch, stream, luh_dev, cells, nd, hbm_peak, fp64_peak)
               if world == 1 else None)
    flops_launch = cells * (395280.0 * mean_sweeps + 116640.0)
    achieved = flops_launch / (pred_ms * 1e-3) / 1e12
    exec_flops = cells * (PRED_EXEC_FLOPS_SWEEP0_TAIL + (mean_sweeps - 1.0) * PRED_EXEC_FLOPS_PER_SWEEP)

    # ---- end to end through the C ABI with host buffers: H2D state, step, D2H state ----
    e2e = None
    if not args.no_e2e:
        host_in = torch.from_numpy(luh0).pin_memory()
        host_out = torch.empty_like(host_in).pin_memory()
        nbytes = host_in.numel() * 8
        if world == 1:
            # a host-resident time loop: every step uploads the host state, steps it and writes the
            # new state back (exa_patch_run_host: chunked copies overlapped with the kernels, the
            # download of step k with the upload of step k+1)
            slab.set_local_solution(host_in.numpy())

            def e2e_steps(k):
                patch.step_host(host_in, host_in, nsteps=k)
        else:
            def e2e_step():
                slab.set_local_solution(host_in.numpy())  # H2D + CFL dt of the uploaded state
                slab.step(1)
                slab.get_solution(host_out.numpy())  # D2H of the result
            def e2e_steps(k):
                for _ in range(k):
                    e2e_step()
        e2e_steps(1)
        barrier()
        t0 = time.perf_counter()
        ke = max(2, K)
        e2e_steps(ke)
        barrier()
        e2e_ms = (time.perf_counter() - t0) * 1e3 / ke
        e2e_t = torch.tensor([e2e_ms], device="cuda")
        if world > 1:
            dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
        e2e_ms = float(e2e_t.item())
        e2e = {"api": "exa_patch_run_host (chunked H2D/D2H overlapped with the kernels and with each other)"
                      if world == 1 else
                      "exa_patch_set_solution + step + exa_patch_get_solution",
               "value": world * dof_step / (e2e_ms * 1e-3), "unit": "DoF-updates/s",
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes, "ms_per_step": e2e_ms}

    pk, pk_kind = peaks()
    line = {
        "metric": METRIC, "value": world * dof_step / (ms * 1e-3), "unit": "DoF-updates/s", "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "3D Euler N=5 (6^3 nodes, nVar=5) entropy wave, %d^3 periodic cells per GPU "
                               "(slab of %dx%dx%d), CFL 0.9, Picard predictor + Rusanov + update, one CUDA graph "
                               "per step on 1 GPU; halo exchange + dt all-reduce over NCCL on N GPUs"
                               % (ncell[0], ncell[0], ncell[1], ncell[2] * world),
                   "cells": cells, "dof_per_step": dof_step, "l2": "inputs 4.6 GB > L2, no flush needed",
                   "precision": args.precision,
                   "picard": "fixed %d sweeps" % args.max_picard if args.max_picard > 0 else "residual test"},
        "cell_updates_per_s": world * cells / (ms * 1e-3),
        "picard_sweeps_mean": stats["picard_mean"], "status_bits": status,
        "accuracy": {"t": float(t_now[0]), "l2_rho_vs_exact": l2_exact, "linf_rho_vs_exact": linf_exact,
                     "sample": "every 37th cell, exact entropy wave at t"},
        "other_precision": other,
        "roofline": {"bound": "fp64", "kernel": "predictor_kernel (fused Picard + volume integral)",
                     "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                     "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run",
                     "traffic": PRED_DRAM_BYTES_PER_CELL * cells,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one predictor launch "
                                       "on a 27^3 block, scaled by cells",
                     "algorithmic_flops_per_launch": flops_launch, "launch_ms": pred_ms,
                     "executed_flops_per_launch": exec_flops if args.precision == "fp64" else None,
                     "executed_tflops": exec_flops / (pred_ms * 1e-3) / 1e12 if args.precision == "fp64" else None,
                     "executed_frac": (exec_flops / (pred_ms * 1e-3) / 1e12 / fp64_peak
                                       if args.precision == "fp64" else None),
                     "executed_source": "per-cell FP64 operations of the kernel from ncu SASS counters (27^3, "
                                        "fixed 2 and 4 sweeps) x the launch's cells and mean sweeps",
                     "hbm_gbs_of_launch": cells * PRED_BYTES_PER_CELL / (pred_ms * 1e-3) / 1e9,
                     "hbm_peak_gbs": pk.get("hbm_gbs"), "hbm_peak_source": pk_kind},
        "gpu_launches": K * 4,
        "predictor_launch_form": solver.predictor_variant,
        "amr_limiter_kernels": amr_lim,
        "hbm_kernels": dict(hbm, launch_form="bulk copies" if args.update_variant != 0 else "per-thread loads",
                            bytes="Rusanov 8,640 B per face (2 x (Q + F) in, 2 x F out); update 34,560 B per "
                                  "cell (luh, lduh, lFhbnd in; luh out)"),
        "clocks": clocks.summary(),
    }
    if e2e:
        line["e2e"] = e2e
    if rank == 0 and not args.no_cpu:
        try:
            line["cpu_baseline"] = cpu_baseline()
        except Exception as ex:  # the baseline must not sink the GPU line
            line["cpu_baseline"] = {"value": None, "error": str(ex)}
    slab.close()
    if rank == 0 and world == 1 and not args.no_workloads:
        line["workloads"] = other_workloads(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def other_workloads(args):
    """Short runs of the other configurations, reported beside the headline line: 512 batched SWE
    grids (5 timed steps), the elastic 48^3 N=7 medium with an active wavefield (3 timed steps) and
    the acoustic 32^3 adjoint gradient (1 timed gradient, 4 finite-difference directions). Each
    record keeps its workload's value, time per step, Picard sweeps, roofline and checks."""
    import copy
    out = {}
    keep = ("metric", "value", "unit", "ms_per_step", "steps", "warmup", "picard_sweeps_mean", "status_bits",
            "roofline", "cpu_baseline", "clocks", "config", "initial_state", "forward_ms_per_step",
            "adjoint_ms_per_step", "gradient_s", "fd_check", "gpu_launches")
    plans = [("swe_batched_512", run_swe_batched, dict(steps=5, warmup=2)),
             ("elastic3d_n7_48cubed_active", run_elastic3d, dict(steps=3, warmup=1, elastic_active=True)),
             ("acoustic_adjoint_n4_32cubed", run_acoustic_adjoint, dict(steps=1, warmup=1, fd_directions=4))]
    for name, fn, over in plans:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        try:
            rec = fn(a)
            out[name] = {k: rec[k] for k in keep if k in rec}
        except Exception as e:  # a sub-record must not sink the headline line
            out[name] = {"error": str(e)}
        out[name]["wall_s"] = time.perf_counter() - t0
    return out


if __name__ == "__main__":
    main()
