#!/usr/bin/env python
"""Benchmark of the batched varRCWA S-matrix solve on B200.

Workload (default, `--workload c3`): the uneven batch of config 3 -- a queue
of 4096 pillar unit cells (400 nm square period, tapered circular pillar of
eps 5.8 and height 600 nm on SiO2 under air, base radius U[60,140] nm,
sidewall angle U[85,90] deg, wavelength U[450,650] nm, harmonic truncation
drawn from {7x7, 9x9, 11x11, 13x13, 15x15}, i.e. n = 98..450 complex128,
rasterised on 256x256 pixels per z-sample), each solved by adaptive varRCWA
(pe = 1e-2) and reduced to per-order reflected/transmitted power for both
polarisations.  A step is one C-ABI call on the next wave of `--batch` cells
of the queue (the whole queue does not fit a minute of timing: at ~15
solves/s it is several minutes of work), so K steps solve K distinct waves.

Metric: S-matrix solves per second (whole job, all ranks).  `value` is the
device time of the calls (CUDA events on the engine stream); `e2e` is the
wall time of the same C-ABI calls from host structure descriptors to host
order powers.  Multi-GPU runs are independent replicas (one process per
GPU, the queue sharded by cost, no collective on the data path).

Sub-lines of the default run (one GPU, outside the timed region): config 2
(11x11 orders), and the forward + adjoint half of the metric on config-4
freeform metagratings (600 nm period, 633 nm, four 150 nm layers of 64x64
permittivity pixels; per-order powers and the gradient of T(+1,0) with
respect to all 16384 pixels per stack) at 9x9 and at 15x15 orders, each
against the same stacks solved one per call.

`--impl reference` times the CPU restatement of the reference algorithm
(the oracle) on this machine's host cores on the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=None,
                   help="cells per step per GPU (c3: 64 cells per wave; c2 / c4: 128; c1: 8, whose ~6600 "
                        "segments per cell are all held until the star reduction)")
    p.add_argument("--queue", type=int, default=4096, help="c3: cells in the job queue (sharded over ranks)")
    p.add_argument("--workload", default="c3", choices=["c1", "c2", "c3", "c4", "c5"],
                   help="c5: config-5 mode converters, forward + adjoint of --batch cells (one GPU)")
    p.add_argument("--pe", type=float, default=None, help="varRCWA tolerance (default 1e-6 for c1, else 1e-2)")
    p.add_argument("--npix", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=90.0,
                   help="bound on the CPU samples (rounds of one cell per host core)")
    p.add_argument("--plain-cells", type=int, default=8,
                   help="cells timed one per call (the plain per-solve form of the metric); 0 skips")
    p.add_argument("--no-sub", action="store_true", help="skip the c2 and forward+adjoint sub-lines")
    p.add_argument("--no-c5", action="store_true", help="skip the config-5 forward+adjoint sub-line")
    p.add_argument("--orders", type=int, default=9, help="c4: harmonics per axis (9 = config 4, 15 = 15x15 orders)")
    p.add_argument("--kernel", default=None, choices=["zgemm", "eig", "assembly"],
                   help="time one kernel entry of the C ABI instead of a workload, for kernel profiles: vrc_zgemm "
                        "or vrc_eig on seeded random n x n matrices (--n, --batch), or vrc_sample_pq on --batch "
                        "z samples of a config-2 pillar cell (11x11 orders, 256x256 raster)")
    p.add_argument("--n", type=int, default=242, help="--kernel: matrix order")
    a = p.parse_args()
    if a.pe is None:
        a.pe = 1e-6 if a.workload == "c1" else 1e-2
    if a.batch is None:
        a.batch = {"c1": 8, "c3": 64, "c5": 4}.get(a.workload, 128)
    return a


def make_cells(workload, batch, rank, npix, step_seed=0, orders=9):
    from varrcwa_b200.replicas import make_cells as mc
    return mc(workload, batch, rank, npix, step_seed, orders)


class Waves:
    """The cells of each step.  c3: consecutive waves of `batch` cells of this
    rank's cost-balanced share of the job queue (wrapping around); other
    workloads: the same seeded batch every step."""

    def __init__(self, a, rank, world):
        self.batch = a.batch
        if a.workload == "c3":
            from varrcwa_b200.replicas import rank_queue
            self.queue = rank_queue("c3", max(a.queue, a.batch * world), rank, world, a.npix)
        else:
            self.queue = make_cells(a.workload, a.batch, rank, a.npix, orders=a.orders)
        self.k = 0

    def next(self):
        q, b = self.queue, self.batch
        out = [q[(self.k * b + i) % len(q)] for i in range(b)]
        self.k += 1
        return out


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def dgemm_peak_tflops(device):
    """Measured FP64 tensor-core throughput of cuBLAS DGEMM (torch float64
    matmul, 8192^3, best of 5) on this GPU: the denominator for the FP64
    DMMA GEMM roofline (no FP64 figure is driver-measured)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize(device)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize(device)
        ms = e0.elapsed_time(e1)
        best = max(best, 2.0 * n ** 3 / (ms * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


# ---------------------------------------------------------------------------
# CPU arms (oracle = CPU restatement of the reference algorithm)
# ---------------------------------------------------------------------------
def _oracle_cell(args):
    desc, pe = args
    from oracle import varrcwa_oracle as O
    from oracle.structures_adapter import end_bases, make_sampler
    s = make_sampler(desc)
    e0, e1 = end_bases(desc, s)
    S = O.redheffer_compute(s, desc["z0"], desc["z1"], pe=pe, end0=e0, end1=e1)
    if desc.get("end1") is None:  # config 1: the S-matrix itself is the output
        return float(abs(S.Tuu).sum())
    R, T = O.order_powers(S, s, desc["end1"], desc["end0"], 1.0, 0.0, side="top")
    return float(R.sum() + T.sum())


def _oracle_stack(desc):
    """Forward + adjoint of one config-4 stack through the oracle."""
    import numpy as np
    from oracle.stack_adjoint import Stack, order_index, stack_backward, stack_forward
    st = Stack(desc["lam"], desc["nx"], desc["ny"], desc["Lx"], desc["Ly"], desc["layers"], desc["thick"],
               desc["eps_in"], desc["eps_out"])
    R, T, tp = stack_forward(st)
    m = desc["nx"] * desc["ny"]
    wT = np.zeros(m)
    wT[order_index(desc["nx"], desc["ny"], 1, 0)] = 1.0
    g = stack_backward(st, tp, np.zeros(m), wT)
    return float(T.sum() + sum(float(x.sum()) for x in g))


def _oracle_task(args):
    desc, pe = args
    return _oracle_stack(desc) if "layers" in desc else _oracle_cell((desc, pe))


def _c5_oracle_task(args):
    """The oracle's forward replay, conversion adjoint and knot gradient of a
    config-5 cell over the given cuts (single-threaded BLAS); seconds taken."""
    desc, cuts = args
    import numpy as np
    from threadpoolctl import threadpool_limits
    from oracle.segments_adjoint import knot_gradient, mode_conversion_adjoint, segments_forward
    from oracle.structures_adapter import make_sampler
    with threadpool_limits(1):
        t0 = time.perf_counter()
        fw = segments_forward(make_sampler(desc), cuts)
        j0 = int(np.argmax(fw["b0"].gam.real))
        j1 = int(np.argsort(-fw["b1"].gam.real)[1])
        _, gS, gW0, gV0, gW1, gV1 = mode_conversion_adjoint(fw, j0, j1)
        knot_gradient(desc, cuts, gS, gW0, gV0, gW1, gV1, h=1e-6 * float(desc["x"][-1] - desc["x"][0]), fw=fw)
        return time.perf_counter() - t0


def cpu_rounds(cells, pe, seconds, warm=None):
    """The oracle on the host cores, one cell per process (spawn pool,
    single-threaded BLAS): rounds of one cell per core, taken in queue order,
    until `seconds` have elapsed (at least one round).  Returns (cells solved,
    seconds, rounds, processes)."""
    import multiprocessing as mp
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["MKL_NUM_THREADS"] = "1"
    workers = max(1, os.cpu_count() or 1)
    done, rounds = 0, 0
    with mp.get_context("spawn").Pool(workers) as pool:
        if warm:  # imports and the first BLAS call in every worker
            pool.map(_oracle_task, [(d, 0.5) for d in warm][:workers] * max(1, workers // max(1, len(warm))))
        t0 = time.perf_counter()
        while True:
            chunk = [cells[(rounds * workers + i) % len(cells)] for i in range(workers)]
            pool.map(_oracle_task, [(d, pe) for d in chunk])
            done += len(chunk)
            rounds += 1
            if time.perf_counter() - t0 >= seconds:
                break
        dt = time.perf_counter() - t0
    return done, dt, rounds, workers


def run_reference(a, rank, world):
    if world > 1 and rank != 0:
        return  # rank 0 alone times the CPU reference
    waves = Waves(a, 0, 1)
    warm = make_cells("c2", 4, 0, 16) if a.workload != "c4" else None
    # a bounded sample: as many rounds as fit the step budget of K steps
    done, dt, rounds, workers = cpu_rounds(waves.queue, a.pe, seconds=a.cpu_seconds + 30.0, warm=warm)
    value = done / dt
    sample = (f"{done} cells of the same queue in {rounds} round(s) of one cell per process ({workers} spawned "
              f"processes, single-threaded BLAS), {dt:.1f} s")
    line = {
        "impl": "reference", "metric": metric_name(a.workload), "value": value, "unit": unit_name(a.workload),
        "n_gpus": a.gpus, "steps": rounds, "warmup": 1 if warm else 0, "ms_per_step": 1e3 * dt / rounds,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
        "data": "synthetic", "config": workload_config(a, a.batch),
        "cpu_baseline": {"value": value, "unit": unit_name(a.workload), "cores": workers, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": unit_name(a.workload), "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def profiled_traffic(family, flops_per_launch):
    """DRAM bytes (read + write) per average launch of the family's main
    kernel, from the committed ncu summary profiles/<family>_traffic.txt
    (`bytes_per_matrix` measured on a smaller launch of the same kernel,
    scaled by the matrices per launch = flops per launch / `flops_per_matrix`),
    or None when no capture is summarised."""
    p = ROOT / "profiles" / f"{family}_traffic.txt"
    if not p.exists() or not flops_per_launch:
        return None
    kv = {}
    for ln in p.read_text().splitlines():
        parts = ln.split()
        if len(parts) == 2:
            try:
                kv[parts[0]] = float(parts[1])
            except ValueError:
                pass
    if "bytes_per_matrix" not in kv or "flops_per_matrix" not in kv:
        return None
    return kv["bytes_per_matrix"] * flops_per_launch / kv["flops_per_matrix"]


def metric_name(workload="c2"):
    if workload == "c4":
        return "batched fwd+adjoint grads/s (FP64 stack solve, per-order T/R and d T(+1,0) / d pixel)"
    return "batched S-matrix solves/s (FP64 varRCWA forward, per-order T/R)"


def unit_name(workload="c2"):
    return "grads/s" if workload == "c4" else "solves/s"


def workload_config(a, batch):
    if a.workload == "c4":
        o = a.orders
        return {"workload": f"config-4 freeform metagrating stacks ({o}x{o} orders, n={2 * o * o}, 4 layers x "
                            f"64x64 pixels, 600 nm period, 633 nm, air -> SiO2)", "batch_per_gpu": batch,
                "n": 2 * o * o,
                "integrator": "Redheffer chain of z-uniform layers (one eigen-solve per layer), star products",
                "output": "per-order R/T (x-polarised incidence) and dT(+1,0)/d(eps) for all 16384 pixels",
                "l2": "per-step working set (GBs of matrices) exceeds the 126 MB L2; no flush needed"}
    names = {"c1": "config-1 2D taper (41 orders, n=82, TE+TM), seeded wavelengths 1.50-1.60 um",
             "c2": "config-2 pillar cells (11x11 orders, n=242, 256x256 raster)",
             "c3": (f"config-3 uneven pillar batch: a queue of {a.queue} cells (orders uniform from 7x7..15x15, "
                    f"n=98..450, lambda U[450,650] nm, 256x256 raster), one wave of {batch} cells per step")}
    n = {"c1": 82, "c2": 242, "c3": "98..450"}.get(a.workload)
    cfg = {"workload": names[a.workload], "batch_per_gpu": batch, "n": n, "pe": a.pe,
           "raster": f"{a.npix}x{a.npix}" if a.workload != "c1" else "2 moving core edges",
           "integrator": "adaptive varRCWA (trisection), Redheffer star products",
           "output": ("the full S-matrix blocks and end bases" if a.workload == "c1" else
                      "per-order R/T, 2 polarisations, incidence from the superstrate"),
           "l2": "per-step working set (GBs of matrices) exceeds the 126 MB L2; no flush needed"}
    if a.workload == "c3":
        cfg["queue"] = a.queue
        cfg["sharding"] = "queue sharded over ranks by cost (n^3), longest first onto the least loaded rank"
    return cfg


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def _busy(v):
    return v.get("busy_ms") or v["ms"]


def breakdown_of(stats):
    busy = {k[1:]: round(v["busy_ms"], 3) for k, v in stats.items() if k.startswith("~")}
    stats = {k: v for k, v in stats.items() if not k.startswith("~")}
    tot = sum(x["ms"] for x in stats.values()) or 1.0
    out = {k: {"ms": round(v["ms"], 3), "busy_ms": round(_busy(v), 3), "share": round(v["ms"] / tot, 4),
               "launches": v["launches"],
               "tflops": round(v["flops"] / (_busy(v) * 1e-3) / 1e12, 3) if v["flops"] and v["ms"] else None}
           for k, v in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])}
    if "host_alloc" in out:  # host time in cudaMalloc / cudaFree (all engines); its byte slot counts the calls
        out["host_alloc"]["calls"] = int(stats["host_alloc"]["bytes"])
    if busy:  # GPU time with at least one kernel of the engines running (all, and per lane)
        out["gpu_busy_ms"] = busy
    return out


def io_bytes(workload, cells):
    """Host-to-device and device-to-host bytes of one step's C-ABI call."""
    import numpy as np
    h2d = sum(len(np.asarray(d.get("eps", [])).tobytes()) for d in cells) + 256 * len(cells)
    if workload == "c1":  # the S-matrix blocks and both end bases come back
        d2h = sum(8 * (2 * d["nx"] * d["ny"]) ** 2 * 16 + 2 * 2 * d["nx"] * d["ny"] * 16 for d in cells)
    elif workload == "c4":  # R, T of one polarisation and the pixel gradient; weights go up
        h2d = sum(sum(np.asarray(x).nbytes for x in d["layers"]) + 8 * len(d["thick"]) + 2 * 8 * d["nx"] * d["ny"]
                  for d in cells)
        d2h = sum(2 * 8 * d["nx"] * d["ny"] + sum(np.asarray(x).nbytes for x in d["layers"]) for d in cells)
    else:  # per-order R and T, both polarisations
        d2h = sum(2 * 2 * d["nx"] * d["ny"] * 8 for d in cells)
    return h2d, d2h


def run_ours(a, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from varrcwa_b200.capi import Context

    dev = local_rank
    torch.cuda.set_device(dev)
    ctx = Context(dev)
    waves = Waves(a, rank, world)
    solve = make_solver(ctx, a.workload, a.pe, a.batch, a.orders)

    def barrier():
        if world > 1:
            dist.barrier()

    fp64_peak = dgemm_peak_tflops(dev) if rank == 0 else None
    for _ in range(a.warmup):
        solve(waves.next())
    ctx.set_profiling(True)
    clocks = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_ms, wall, launches, h2d, d2h, nonzero = 0.0, 0.0, 0, 0, 0, 0
    step_cells = []
    for _ in range(a.steps):
        cells = waves.next()  # host descriptors of the step, built outside its timed call
        step_cells.append(cells)
        t0 = time.perf_counter()
        out, ms, nl = solve(cells)
        wall += time.perf_counter() - t0
        dev_ms += ms
        launches += nl
        bi, bo = io_bytes(a.workload, cells)
        h2d += bi
        d2h += bo
        nonzero += sum(1 for o in out if o["status"])
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    stats = ctx.kernel_stats()
    ctx.set_profiling(False)
    # max over ranks
    if world > 1:
        from varrcwa_b200.replicas import max_over_ranks
        dev_ms, wall = max_over_ranks([dev_ms, wall], device=f"cuda:{dev}")
    if rank != 0:
        return
    from varrcwa_b200.replicas import job_throughput
    value = job_throughput(a.batch, a.steps, world, dev_ms * 1e-3)
    e2e = job_throughput(a.batch, a.steps, world, wall)
    roof = roofline_of(stats, fp64_peak)
    gemm = stats.get("zgemm")
    unit = unit_name(a.workload)
    line = {
        "metric": metric_name(a.workload), "value": value, "unit": unit, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": dev_ms / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
        "config": workload_config(a, a.batch), "parallelism": f"replicas x{world}",
        "e2e": {"value": e2e, "unit": unit, "h2d_bytes_per_step": h2d // a.steps, "d2h_bytes_per_step": d2h // a.steps},
        "gpu_launches": launches, "roofline": roof, "clocks": clk, "kernel_breakdown": breakdown_of(stats),
        "statuses_nonzero": nonzero,
    }
    if a.workload == "c3":
        from collections import Counter
        line["config"]["truncations_timed"] = dict(sorted(Counter(
            f"{d['nx']}x{d['ny']}" for cells in step_cells for d in cells).items()))
    if gemm:
        line["zgemm_tflops"] = gemm["flops"] / (_busy(gemm) * 1e-3) / 1e12
        line["fp64_dgemm_peak_tflops"] = fp64_peak
    # the plain form the metric compares against: the same cells submitted
    # one structure per call on the same GPU (outside the timed region)
    if world == 1 and a.plain_cells > 0:
        cells = step_cells[0][: a.plain_cells]
        torch.cuda.synchronize()
        tp = time.perf_counter()
        for d in cells:
            solve([d])
        torch.cuda.synchronize()
        tpl = time.perf_counter() - tp
        t0 = time.perf_counter()
        solve(cells)  # the same cells in one call, for a like-for-like ratio
        tb = time.perf_counter() - t0
        line["plain_per_solve"] = {"value": len(cells) / tpl, "unit": unit, "cells": len(cells),
                                   "form": "one cell per C-ABI call, same GPU, host buffers"}
        line["batched_over_plain"] = e2e / (len(cells) / tpl)
        line["same_cells_batched_over_plain"] = tpl / tb
    if world == 1 and os.environ.get("VRC_LANES") is None:
        # the same step on one engine, after the timed region: the kernels'
        # uncontended rates (in the timed region the call's cells run on
        # concurrent engines, whose launches share the GPU)
        os.environ["VRC_LANES"] = "1"
        try:
            solve(step_cells[0])  # one engine now holds all cells: let its pools grow first
            ctx.set_profiling(True)
            solve(step_cells[0])
            line["roofline_single_lane"] = roofline_of(ctx.kernel_stats(), fp64_peak)
            line["roofline_single_lane"]["note"] = ("the first timed wave again with the cells on one engine, "
                                                    "outside the timed region")
            ctx.set_profiling(False)
        finally:
            del os.environ["VRC_LANES"]
    if world == 1 and not a.no_sub:
        subs = {}
        if a.workload != "c2":
            subs["c2"] = measure_forward(ctx, "c2", a.pe, batch=64, steps=3)
        if a.workload != "c4":
            subs["fwd_adjoint"] = measure_fwd_adjoint(ctx, 9, batch=128, steps=10, plain=32)
            subs["fwd_adjoint_15x15"] = measure_fwd_adjoint(ctx, 15, batch=64, steps=10, plain=32)
        if not a.no_c5:
            # n = 882 needs large blocks: a fresh context (the pools of the
            # lines above hold their device memory until the context closes)
            ctx.close()
            torch.cuda.empty_cache()
            ctx = Context(dev)
            try:
                subs["c5_fwd_adjoint"] = measure_c5(ctx, fp64_peak, orders=21, batch=1, steps=1,
                                                    cpu=not a.no_cpu_baseline)
            except Exception as e:  # the headline line is printed regardless
                subs["c5_fwd_adjoint"] = {"error": f"{type(e).__name__}: {e}"}
        line.update(subs)
    if world == 1 and not a.no_cpu_baseline:
        done, dt, rounds, workers = cpu_rounds(waves.queue, a.pe, seconds=a.cpu_seconds,
                                               warm=make_cells("c2", 4, 0, 16) if a.workload != "c4" else None)
        line["cpu_baseline"] = {"value": done / dt, "unit": unit, "cores": workers, "kind": "port",
                                "sample": f"{done} cells of the same queue through the numpy oracle, one per "
                                          f"process ({workers} spawned, single-threaded BLAS), {rounds} round(s), "
                                          f"{dt:.1f} s"}
    print(json.dumps(line), flush=True)


def roofline_of(stats, fp64_peak):
    """Roofline of the dominant kernel family of a profiled run."""
    # dominant kernel family and its roofline.  FP64 work on B200 runs either
    # on the DMMA tensor pipe (GEMMs, the inversion's rank-32 updates) or on
    # the FP64 FMA pipe (Hessenberg, QR, back substitution); the two peaks
    # coincide on this part, so both are measured against cuBLAS DGEMM.
    # a family's time is the union of its launches' intervals (busy_ms): a
    # call's cells run on concurrent engines, whose launches overlap
    fam = max((kv for kv in stats.items() if kv[1]["launches"] > 0),  # host_alloc is host time
              key=lambda kv: kv[1].get("busy_ms") or kv[1]["ms"])
    hbm_peak, hbm_src = measured_peaks()
    name, f = fam
    limiter = {"zgemm": "FP64 DMMA tensor pipe", "zinv": "panel reduction (latency) + DMMA rank-32 updates",
               "hessenberg": "cluster barriers per column (latency)",
               "schur_qr": "sequential bulge chase (latency)", "schur_replay": "FP64 pipe / memory latency",
               "trevc": "sequential back substitution (latency)"}.get(name, "HBM bandwidth")
    traffic = profiled_traffic(name, f["flops"] / max(f["launches"], 1))
    busy = f.get("busy_ms") or f["ms"]
    if f["flops"] > 0:
        achieved = f["flops"] / (busy * 1e-3) / 1e12
        roof = {"kernel": name, "bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak if fp64_peak else None,
                "peak_source": "measured cuBLAS DGEMM (FP64) on this GPU, 8192^3, in this run",
                "limiter": limiter, "avg_launch_ms": f["ms"] / max(f["launches"], 1), "busy_ms": busy,
                "achieved_over": "the union of the family's launch intervals on all engines (busy_ms)",
                "traffic": traffic}
    else:
        achieved = f["bytes"] / (busy * 1e-3) / 1e9
        roof = {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved / hbm_peak, "peak_source": f"{hbm_src} MEASURED_PEAKS.json hbm_gbs",
                "limiter": limiter, "avg_launch_ms": f["ms"] / max(f["launches"], 1), "busy_ms": busy,
                "achieved_over": "the union of the family's launch intervals on all engines (busy_ms)",
                "traffic": traffic}
    return roof


def make_solver(ctx, workload, pe, batch, orders=9):
    """One step of the workload through the C ABI: returns (per-cell results,
    device ms, kernel launches) of the call(s)."""
    import numpy as np
    if workload == "c4":
        nx = ny = orders
        k = ny * (1 + (nx - 1) // 2) + (ny - 1) // 2  # order (+1, 0)
        wT = np.zeros((batch, nx * ny))
        wT[:, k] = 1.0
        wR = np.zeros((batch, nx * ny))

        def solve(cells):
            _, _, st = ctx.stack_forward(cells)
            t1 = ctx.timing()
            ctx.stack_backward(wR[: len(cells)], wT[: len(cells)])
            t2 = ctx.timing()
            return ([{"status": int(x)} for x in st], t1["device_ms"] + t2["device_ms"],
                    t1["launches"] + t2["launches"])
        return solve

    def solve(cells):
        # config 1's output is the full S-matrix (its ends are the structure's
        # own cross-sections, so there are no half-space orders to report)
        if workload == "c1":
            out = ctx.redheffer(cells, pe=pe)
        else:
            out = ctx.order_powers(cells, method="redheffer", pe=pe, side=1)
        t = ctx.timing()
        return out, t["device_ms"], t["launches"]
    return solve


def measure_forward(ctx, workload, pe, batch, steps, warmup=1):
    """A short forward sub-line (device and end-to-end solves/s)."""
    import torch
    cells = make_cells(workload, batch, 0, 256)
    solve = make_solver(ctx, workload, pe, batch)
    for _ in range(warmup):
        solve(cells)
    torch.cuda.synchronize()
    dev_ms, t0 = 0.0, time.perf_counter()
    for _ in range(steps):
        dev_ms += solve(cells)[1]
    wall = time.perf_counter() - t0
    return {"metric": metric_name(workload), "value": batch * steps / (dev_ms * 1e-3), "unit": "solves/s",
            "e2e": {"value": batch * steps / wall, "unit": "solves/s"}, "steps": steps, "warmup": warmup,
            "config": {"workload": "config-2 pillar cells (11x11 orders, n=242, 256x256 raster)",
                       "batch_per_gpu": batch, "pe": pe}}


def measure_fwd_adjoint(ctx, orders, batch, steps, plain, warmup=2):
    """Config-4 forward + adjoint: batched stacks against the same stacks one
    forward + backward pair per call (the plain form)."""
    import torch
    cells = make_cells("c4", batch, 0, 64, orders=orders)
    solve = make_solver(ctx, "c4", None, batch, orders)
    for _ in range(warmup):
        solve(cells)
    torch.cuda.synchronize()
    dev_ms, launches = 0.0, 0
    t0 = time.perf_counter()
    for _ in range(steps):
        _, ms, nl = solve(cells)
        dev_ms += ms
        launches += nl
    wall = time.perf_counter() - t0
    solve(cells[:1])  # warm the one-stack shapes
    torch.cuda.synchronize()
    pc = [cells[i % len(cells)] for i in range(plain)]
    tp = time.perf_counter()
    for d in pc:
        solve([d])
    tpl = time.perf_counter() - tp
    return {"metric": metric_name("c4"), "value": batch * steps / (dev_ms * 1e-3), "unit": "grads/s",
            "e2e": {"value": batch * steps / wall, "unit": "grads/s"}, "steps": steps, "warmup": warmup,
            "ms_per_step": dev_ms / steps, "gpu_launches": launches,
            "config": {"workload": f"config-4 freeform metagrating stacks ({orders}x{orders} orders, "
                                   f"n={2 * orders * orders}, 4 layers x 64x64 pixels)", "batch_per_gpu": batch,
                       "output": "per-order R/T and dT(+1,0)/d(eps) for all 16384 pixels"},
            "plain_per_solve": {"value": plain / tpl, "unit": "grads/s", "cells": plain,
                                "form": "one stack per forward+backward C-ABI pair"},
            "batched_over_plain": (batch * steps / wall) / (plain / tpl)}


def measure_c5(ctx, fp64_peak=None, orders=21, batch=2, steps=1, length=20.0, ncontrol=64, cpu=True):
    """Config-5 forward + adjoint: PML mode converters (n = 2 orders^2),
    adaptive varRCWA, the flux-normalised conversion power from the entrance's
    leading mode into the exit's second mode, and its gradient with respect to
    every width control point (spline knots; checkpointed reverse pass).
    With cpu, the oracle's time for the same gradient of one cell is sampled
    on its first one and first two segments of the device's segmentation and
    extrapolated to the cell's segment count."""
    import multiprocessing as mp
    import numpy as np
    import torch
    from varrcwa_b200 import objectives
    from varrcwa_b200 import structures as st
    cells = [st.converter_c5(5000 + i, norders=orders, ncontrol=ncontrol, length=length) for i in range(batch)]

    def one(cs):
        rs = ctx.redheffer_forward(cs, pe=1e-2)
        t1 = ctx.timing()
        cot = []
        for r in rs:
            i0, i1 = int(np.argmax(r["gam0"].real)), int(np.argsort(-r["gam1"].real)[1])
            cot.append(objectives.mode_conversion(r, i0, i1))
        ctx.redheffer_backward([c[1] for c in cot], [c[2] for c in cot])
        t2 = ctx.timing()
        return rs, t1["device_ms"] + t2["device_ms"], t1["launches"] + t2["launches"]

    torch.cuda.synchronize()
    ctx.set_profiling(True)
    dev_ms, launches, segs = 0.0, 0, 0
    t0 = time.perf_counter()
    for _ in range(steps):
        rs, ms, nl = one(cells)
        dev_ms += ms
        launches += nl
        segs += sum(r["N"] for r in rs)
    wall = time.perf_counter() - t0
    stats = ctx.kernel_stats()
    ctx.set_profiling(False)
    leaves = sorted((a_, b_) for (a_, b_, e_, acc) in ctx.tree(0) if acc)
    cuts0 = [leaves[0][0]] + [b_ for (_, b_) in leaves]
    line = {"metric": "batched fwd+adjoint grads/s (FP64 adaptive varRCWA, d(mode conversion) / d(control points))",
            "value": batch * steps / (dev_ms * 1e-3), "unit": "grads/s",
            "e2e": {"value": batch * steps / wall, "unit": "grads/s"}, "steps": steps, "warmup": 0,
            "ms_per_step": dev_ms / steps, "gpu_launches": launches,
            "segments_per_cell": segs / (batch * steps),
            "config": {"workload": f"config-5 PML mode converters ({orders}x{orders} orders, n={2 * orders * orders}, "
                                   f"{ncontrol} spline control points over {length} um, 4 x 2 um cell)",
                       "batch_per_gpu": batch, "pe": 1e-2,
                       "output": "mode-conversion power and its gradient w.r.t. every control point"},
            "kernel_breakdown": breakdown_of(stats)}
    if fp64_peak:
        line["roofline"] = roofline_of(stats, fp64_peak)
    if cpu and len(cuts0) >= 3:
        with mp.get_context("spawn").Pool(2) as pool:
            t1, t2 = pool.map(_c5_oracle_task, [(cells[0], cuts0[:2]), (cells[0], cuts0[:3])])
        nseg = len(cuts0) - 1
        t_cell = t1 + (nseg - 1) * max(t2 - t1, 0.0)
        cores = os.cpu_count() or 1
        line["cpu_baseline"] = {
            "value": cores / t_cell, "unit": "grads/s", "cores": cores, "kind": "port",
            "sample": (f"the oracle's forward replay, conversion adjoint and knot gradient of cell 0 over its first "
                       f"one and two segments of the device's segmentation ({t1:.1f} s, {t2:.1f} s; single-threaded "
                       f"BLAS, two spawned processes), extrapolated to its {nseg} segments ({t_cell:.0f} s per cell) "
                       f"and to {cores} cells at once on {cores} host cores")}
    return line


def run_c5(a):
    """The config-5 forward + adjoint as a line of its own (one GPU): --batch
    converter cells per step, --steps timed steps, the oracle sample for the
    CPU baseline unless --no-cpu-baseline."""
    import torch
    from varrcwa_b200.capi import Context
    ctx = Context(0)
    fp64_peak = dgemm_peak_tflops(0)
    torch.cuda.empty_cache()
    clocks = ClockSampler(0)
    clocks.start()
    line = measure_c5(ctx, fp64_peak, orders=21, batch=a.batch, steps=a.steps, cpu=not a.no_cpu_baseline)
    line["clocks"] = clocks.stop()
    line.update({"n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": "complex128", "data": "synthetic"})
    print(json.dumps(line), flush=True)


def run_kernel(a):
    """One C-ABI kernel entry (vrc_zgemm: batch products of n x n complex
    matrices; vrc_eig: batch eigen-decompositions) on seeded random inputs:
    --warmup untimed calls, then --steps timed ones; device time per call and
    the family's busy time and rate from the engine's counters."""
    import numpy as np
    from varrcwa_b200.capi import Context
    ctx = Context(0)
    n, b = a.n, a.batch
    if a.kernel == "assembly":
        from varrcwa_b200 import structures as st
        cell = st.pillar_config2(seed=2000, npix=a.npix)
        n = 2 * cell["nx"] * cell["ny"]
        zs = np.linspace(cell["z0"], cell["z1"], b)
        call = lambda: ctx.sample_pq(cell, zs)
    else:
        rng = np.random.default_rng(7)
        A = rng.standard_normal((b, n, n)) + 1j * rng.standard_normal((b, n, n))
        B = rng.standard_normal((b, n, n)) + 1j * rng.standard_normal((b, n, n))
        call = (lambda: ctx.zgemm(A, B)) if a.kernel == "zgemm" else (lambda: ctx.eig(A))
    for _ in range(a.warmup):
        call()
    ctx.set_profiling(True)
    ms = []
    for _ in range(a.steps):
        call()
        ms.append(ctx.timing()["device_ms"])
    stats = ctx.kernel_stats()
    ctx.set_profiling(False)
    line = {"kernel": a.kernel, "n": n, "batch": b, "steps": a.steps, "warmup": a.warmup,
            "ms_per_call": sum(ms) / len(ms), "kernel_breakdown": breakdown_of(stats)}
    if a.kernel == "assembly":
        # algorithmic bytes per sample: the eps raster in, fe11, fe22, fe33 and P, Q out
        m = n // 2
        per = 16.0 * (a.npix * a.npix + 3 * m * m + 2 * n * n)
        line["algorithmic_bytes_per_sample"] = per
        fam = stats.get("assembly")
        if fam:  # the assembly family's own busy time, without the copies of P, Q to the host
            busy = _busy(fam) / a.steps
            line["assembly_ms_per_call"] = busy
            line["achieved_gbs"] = per * b / (busy * 1e-3) / 1e9
    else:
        flops = (8.0 if a.kernel == "zgemm" else 80.0) * n ** 3 * b
        line["nominal_tflops"] = flops / (line["ms_per_call"] * 1e-3) / 1e12
        line["nominal_flops"] = "8 n^3 per product" if a.kernel == "zgemm" else "80 n^3 per decomposition"
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "WORLD_SIZE" not in os.environ and a.gpus > 1:
        # one process per GPU: relaunch this command under torchrun
        import socket
        s = socket.socket()
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
        s.close()
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()),
               *sys.argv[1:]]
        sys.exit(subprocess.call(cmd))
    if world != a.gpus:
        sys.exit(f"bench.py: --gpus {a.gpus} but WORLD_SIZE={world}: launch one process per GPU")
    if a.kernel:
        run_kernel(a)
        return
    if a.workload == "c5" and a.impl == "ours":
        run_c5(a)
        return
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
