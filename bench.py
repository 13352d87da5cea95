#!/usr/bin/env python
"""Benchmark of the batched varRCWA S-matrix solve on B200.

Workload (default): a batch of config-2 pillar unit cells -- 400 nm square
period, 532 nm, 11x11 orders (n = 242, complex128), a tapered circular
pillar (eps 5.8) of height 600 nm with seeded base radius U[60,140] nm and
sidewall angle U[85,90] deg, rasterised on 256x256 pixels per z-sample, on
an SiO2 substrate (eps 2.13) under air -- each solved by adaptive varRCWA
(pe = 1e-2) and reduced to per-order reflected/transmitted power for both
polarisations.  A step is one batched call of the C-ABI on `--batch` cells.

Metric: S-matrix solves per second (whole job, all ranks).  `value` is the
device time of the calls (CUDA events on the engine stream); `e2e` is the
wall time of the same C-ABI calls from host structure descriptors to host
order powers.  Multi-GPU runs are independent replicas (one process per
GPU, disjoint cell seeds, no collective on the data path).

`--workload c4` measures the other half of the metric: forward + adjoint
solves of config-4 freeform metagratings (600 nm period, 633 nm, 9x9 orders,
four 150 nm layers of 64x64 permittivity pixels) -- per-order powers and the
gradient of T(+1,0) with respect to all 16384 pixels per stack.  The default
config-2 line carries a short run of it under "fwd_adjoint".

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
                   help="cells per step per GPU (default 128; 8 for c1, whose ~6600 segments per cell are "
                        "all held until the star reduction)")
    p.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4"])
    p.add_argument("--pe", type=float, default=None, help="varRCWA tolerance (default 1e-6 for c1, else 1e-2)")
    p.add_argument("--npix", type=int, default=256)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--cpu-cells", type=int, default=1, help="cells in the bounded CPU sample")
    p.add_argument("--plain-cells", type=int, default=8,
                   help="cells timed one per call (the plain per-solve form of the metric); 0 skips")
    p.add_argument("--no-adjoint", action="store_true", help="skip the fwd_adjoint sub-measurement of the c2 line")
    p.add_argument("--orders", type=int, default=9, help="c4: harmonics per axis (9 = config 4, 15 = 15x15 orders)")
    a = p.parse_args()
    if a.pe is None:
        a.pe = 1e-6 if a.workload == "c1" else 1e-2
    if a.batch is None:
        a.batch = 8 if a.workload == "c1" else 128
    return a


def make_cells(workload, batch, rank, npix, step_seed=0, orders=9):
    from varrcwa_b200.replicas import make_cells as mc
    return mc(workload, batch, rank, npix, step_seed, orders)


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


def cpu_sample(descs, pe):
    """Time the oracle on the given cells with all host threads (BLAS)."""
    t0 = time.perf_counter()
    for d in descs:
        if "layers" in d:
            _oracle_stack(d)
        else:
            _oracle_cell((d, pe))
    return time.perf_counter() - t0


def run_reference(a, rank, world):
    import multiprocessing as mp
    if world > 1 and rank != 0:
        return  # rank 0 alone times the CPU reference
    ncores = os.cpu_count() or 1
    workers = max(1, ncores)
    descs = make_cells(a.workload, workers, rank, a.npix, orders=a.orders)
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    os.environ["OMP_NUM_THREADS"] = "1"
    os.environ["MKL_NUM_THREADS"] = "1"
    ctxm = mp.get_context("spawn")
    with ctxm.Pool(workers) as pool:
        if a.workload == "c4":
            pool.map(_oracle_stack, descs[:workers])  # warm-up: imports, first BLAS call
            t0 = time.perf_counter()
            for _ in range(a.steps):
                pool.map(_oracle_stack, descs)
            dt = time.perf_counter() - t0
        else:
            # warm-up: one small task per worker (imports, first BLAS call)
            for _ in range(a.warmup):
                pool.map(_oracle_cell, [(d, 0.5) for d in make_cells(a.workload, workers, rank, 16)])
            t0 = time.perf_counter()
            for _ in range(a.steps):
                pool.map(_oracle_cell, [(d, a.pe) for d in descs])
            dt = time.perf_counter() - t0
    value = a.steps * len(descs) / dt
    line = {
        "impl": "reference", "metric": metric_name(a.workload), "value": value, "unit": unit_name(a.workload),
        "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * dt / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
        "config": workload_config(a, len(descs)),
        "cpu_baseline": {"value": value, "unit": unit_name(a.workload), "cores": workers, "kind": "port",
                         "sample": f"{len(descs)} cells per step, one per process (spawn), single-threaded BLAS"},
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
             "c3": "config-3 uneven pillar batch (7..15 orders, n=98..450)"}
    n = {"c1": 82, "c2": 242}.get(a.workload)
    return {"workload": names[a.workload], "batch_per_gpu": batch, "n": n, "pe": a.pe,
            "raster": f"{a.npix}x{a.npix}" if a.workload != "c1" else "2 moving core edges",
            "integrator": "adaptive varRCWA (trisection), Redheffer star products",
            "output": ("the full S-matrix blocks and end bases" if a.workload == "c1" else
                       "per-order R/T, 2 polarisations, incidence from the superstrate"),
            "l2": "per-step working set (GBs of matrices) exceeds the 126 MB L2; no flush needed"}


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(a, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    from varrcwa_b200.capi import Context

    dev = local_rank
    torch.cuda.set_device(dev)
    ctx = Context(dev)
    descs = make_cells(a.workload, a.batch, rank, a.npix, orders=a.orders)

    solve = make_solver(ctx, a.workload, a.pe, a.batch, a.orders)

    def barrier():
        if world > 1:
            dist.barrier()

    fp64_peak = dgemm_peak_tflops(dev) if rank == 0 else None
    for _ in range(a.warmup):
        solve(descs)
    adjoint = None
    if a.workload == "c2" and world == 1 and not a.no_adjoint:
        adjoint = measure_fwd_adjoint(ctx, rank, a.no_cpu_baseline)
    ctx.set_profiling(True)
    clocks = ClockSampler(dev)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    dev_ms = 0.0
    launches = 0
    t0 = time.perf_counter()
    for _ in range(a.steps):
        out, ms, nl = solve(descs)
        dev_ms += ms
        launches += nl
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier()
    clk = clocks.stop()
    stats = ctx.kernel_stats()
    ctx.set_profiling(False)
    statuses = [o["status"] for o in out]
    # max over ranks
    if world > 1:
        from varrcwa_b200.replicas import max_over_ranks
        dev_ms, wall = max_over_ranks([dev_ms, wall], device=f"cuda:{dev}")
    if rank != 0:
        return
    from varrcwa_b200.replicas import job_throughput
    value = job_throughput(a.batch, a.steps, world, dev_ms * 1e-3)
    e2e = job_throughput(a.batch, a.steps, world, wall)
    m = 121 if a.workload == "c2" else None
    h2d = sum(len(np.asarray(d.get("eps", [])).tobytes()) for d in descs) + 256 * len(descs)
    if a.workload == "c1":  # the S-matrix blocks and both end bases come back
        d2h = sum(8 * (2 * d["nx"] * d["ny"]) ** 2 * 16 + 2 * 2 * d["nx"] * d["ny"] * 16 for d in descs)
    elif a.workload == "c4":  # R, T of one polarisation and the pixel gradient; weights go up
        h2d = sum(sum(np.asarray(x).nbytes for x in d["layers"]) + 8 * len(d["thick"]) + 2 * 8 * d["nx"] * d["ny"]
                  for d in descs)
        d2h = sum(2 * 8 * d["nx"] * d["ny"] + sum(np.asarray(x).nbytes for x in d["layers"]) for d in descs)
    else:  # per-order R and T, both polarisations
        d2h = sum(2 * 2 * d["nx"] * d["ny"] * 8 for d in descs)
    roof = roofline_of(stats, fp64_peak)
    gemm = stats.get("zgemm")
    def _busy(v):
        return v.get("busy_ms") or v["ms"]
    breakdown = {k: {"ms": round(v["ms"], 3), "busy_ms": round(_busy(v), 3),
                     "share": round(v["ms"] / sum(x["ms"] for x in stats.values()), 4),
                     "launches": v["launches"],
                     "tflops": round(v["flops"] / (_busy(v) * 1e-3) / 1e12, 3) if v["flops"] and v["ms"] else None}
                 for k, v in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])}
    unit = unit_name(a.workload)
    line = {
        "metric": metric_name(a.workload), "value": value, "unit": unit, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": dev_ms / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
        "config": workload_config(a, a.batch), "parallelism": f"replicas x{world}",
        "e2e": {"value": e2e, "unit": unit, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches, "roofline": roof, "clocks": clk, "kernel_breakdown": breakdown,
        "statuses_nonzero": int(sum(1 for s in statuses if s)),
    }
    if gemm:
        line["zgemm_tflops"] = gemm["flops"] / (_busy(gemm) * 1e-3) / 1e12
        line["fp64_dgemm_peak_tflops"] = fp64_peak
    # the plain form the metric compares against: the same cells submitted
    # one structure per call on the same GPU (outside the timed region)
    if world == 1 and a.plain_cells > 0:
        torch.cuda.synchronize()
        tp = time.perf_counter()
        for d in descs[: a.plain_cells]:
            solve([d])
        torch.cuda.synchronize()
        tpl = time.perf_counter() - tp
        plain = min(a.plain_cells, len(descs)) / tpl
        line["plain_per_solve"] = {"value": plain, "unit": unit, "cells": min(a.plain_cells, len(descs)),
                                   "form": "one cell per C-ABI call, same GPU, host buffers"}
        line["batched_over_plain"] = e2e / plain
    if world == 1 and not a.no_cpu_baseline:
        sample = descs[: a.cpu_cells]
        dt = cpu_sample(sample, a.pe)
        line["cpu_baseline"] = {"value": len(sample) / dt, "unit": unit, "cores": os.cpu_count(),
                                "kind": "port",
                                "sample": f"{len(sample)} cell(s) of the same workload through the numpy oracle "
                                          f"(OpenBLAS threads = host cores), {dt:.1f} s"}
    if world == 1 and os.environ.get("VRC_LANES") is None:
        # the same step on one engine, after the timed region: the kernels'
        # uncontended rates (in the timed region the call's cells run on
        # concurrent engines, whose launches share the GPU)
        os.environ["VRC_LANES"] = "1"
        try:
            solve(descs)  # one engine now holds all cells: let its pools grow first
            ctx.set_profiling(True)
            solve(descs)
            line["roofline_single_lane"] = roofline_of(ctx.kernel_stats(), fp64_peak)
            line["roofline_single_lane"]["note"] = ("an extra step with the cells on one engine, outside the "
                                                    "timed region")
            ctx.set_profiling(False)
        finally:
            del os.environ["VRC_LANES"]
    if adjoint is not None:
        line["fwd_adjoint"] = adjoint
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


def measure_fwd_adjoint(ctx, rank, no_cpu, batch=128, steps=3, warmup=3, plain=4):
    """Short config-4 forward+adjoint measurement for the default line."""
    import torch
    cells = make_cells("c4", batch, rank, 64)
    solve = make_solver(ctx, "c4", None, batch)
    for _ in range(warmup):
        solve(cells)
    torch.cuda.synchronize()
    dev_ms = 0.0
    launches = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        _, ms, nl = solve(cells)
        dev_ms += ms
        launches += nl
    wall = time.perf_counter() - t0
    tp = time.perf_counter()
    for d in cells[:plain]:
        solve([d])
    tpl = time.perf_counter() - tp
    out = {"metric": metric_name("c4"), "value": batch * steps / (dev_ms * 1e-3), "unit": "grads/s",
           "e2e": {"value": batch * steps / wall, "unit": "grads/s"}, "steps": steps, "warmup": warmup,
           "ms_per_step": dev_ms / steps, "gpu_launches": launches,
           "config": {"workload": "config-4 freeform metagrating stacks (9x9 orders, n=162, 4 layers x 64x64 "
                                  "pixels)", "batch_per_gpu": batch,
                      "output": "per-order R/T and dT(+1,0)/d(eps) for all 16384 pixels"},
           "plain_per_solve": {"value": plain / tpl, "unit": "grads/s", "cells": plain,
                               "form": "one stack per forward+backward C-ABI pair"},
           "batched_over_plain": (batch * steps / wall) / (plain / tpl)}
    if not no_cpu:
        dt = cpu_sample(cells[:1], None)
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "grads/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"1 stack, oracle forward + adjoint (OpenBLAS threads = host cores), "
                                         f"{dt:.2f} s; central differences would need 2 x 16384 solves"}
    return out


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
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
