"""Benchmark of the gridcalc hot path on B200.

Headline workload: the plain method -- explicit RK4 Cahn-Hilliard, FP64,
order-2 Laplacian applied twice, M = kappa = 1, dx = 1, dt = 0.01, initial
c = U[-0.05, 0.05] from a seed -- on a 2-D periodic 8192 x 8192 grid (each
field 512 MiB, far beyond the 126 MB L2, so every step streams from HBM).
One "step" is one RK4 step (four fused stage kernels).  Metric: Mcell-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): every rank advances its own replica
(the method has no data-path exchange at this size: replicas only, weak
scaling); the time is the max over ranks.

The reference arm (--impl reference) times the reference's own CPU code
(the reference headers compiled into oracle/_ref/libgcref.so; the C oracle
port if that build is absent) on the box's host cores: independent replicas
of a bounded 1024 x 1024 sample, one per host thread, each step one RK4 step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "grid-calculus_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

NX = NY = 8192
DT = 0.01
# Algorithmic HBM bytes per cell-step of the fused RK4 (13 field passes of
# 8-byte doubles: stage 1 reads psi and writes k1, stages 2-3 read psi and
# k_prev and write k_s, stage 4 reads psi, k1, k2, k3 and writes psi').
BYTES_PER_CELL_STEP = 13 * 8
# DRAM bytes (read + write) per RK4 step per cell measured by ncu for the
# four stage kernels on this workload's kernel (profiles/ch_rk4_fp64_8192.md);
# None until a capture exists.
NCU_TRAFFIC_PER_CELL_STEP = None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def cpu_sample(threads: int, n: int = 1024, steps: int = 1):
    """Runs the reference CPU code (or the C port) on `threads` independent
    n x n replicas for `steps` RK4 steps each; returns (Mcell-steps/s, kind, sample)."""
    import numpy as np
    import oracle_lib
    if oracle_lib.reference_available():
        lib, kind = oracle_lib.reference(), "reference"
    else:
        lib, kind = oracle_lib.oracle(), "port"
    rng = np.random.default_rng(7)
    states = [0.05 * (2.0 * rng.random((1, n, n)) - 1.0) for _ in range(threads)]

    def work(i):
        states[i] = lib.ch_integrate(2, 1.0, 1.0, states[i], DT, steps)

    t0 = time.perf_counter()
    ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    dt = time.perf_counter() - t0
    return threads * n * n * steps / dt / 1e6, kind, f"{threads} x RK4 on {n}x{n}, {steps} step(s) each"


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return
    threads = max(1, min(os.cpu_count() or 1, 32))
    for _ in range(args.warmup):
        cpu_sample(threads)
    t0 = time.perf_counter()
    rates = [cpu_sample(threads)[0] for _ in range(args.steps)]
    wall = time.perf_counter() - t0
    _, kind, sample = cpu_sample(1, 256, 1)
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": "Mcell-steps/s (plain FP64 RK4 Cahn-Hilliard)", "value": value,
        "unit": "Mcell-steps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * wall / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "ch2d-rk4-fp64-order2", "grid": f"{NX}x{NY} (CPU sample 1024x1024 per thread)",
                   "dt": DT, "kappa": 1.0, "mobility": 1.0},
        "cpu_baseline": {"value": value, "unit": "Mcell-steps/s", "cores": threads, "kind": kind,
                         "sample": f"{threads} threads x independent 1024x1024 replica, 1 RK4 step per timed step"},
        "e2e": {"value": value, "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local: int):
    import numpy as np
    import torch
    import gridcalc_b200 as gc

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    g = gc.Grid(args.grid, args.grid, 1)
    rhs = gc.CahnHilliardRhs(1.0, 1.0, 2)
    rng = np.random.default_rng(1000 + rank)
    psi0 = 0.05 * (2.0 * rng.random(g.shape) - 1.0)
    psi = torch.from_numpy(psi0).to(f"cuda:{local}")
    ctx = gc.context()

    # Warm-up: W steps, at least one 16-step graph unit so that the step
    # graph is captured before the timed region.
    gc.ch_integrate(psi, g, rhs, DT, max(args.warmup, 16), gc.RK4)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clocks:
        start.record()
        gc.ch_integrate(psi, g, rhs, DT, args.steps, gc.RK4)
        end.record()
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end)
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    cells = g.size
    value = world * cells * args.steps / (ms / 1e3) / 1e6
    ms_per_step = ms / args.steps
    achieved = BYTES_PER_CELL_STEP * cells / (ms_per_step / 1e3) / 1e9
    peak, peak_kind = peaks()

    # e2e: host field in pinned memory -> the C-ABI call -> host field, in
    # chunks of `chunk` steps (one snapshot per chunk), copies inside the timing.
    chunk = min(args.steps, 100)
    n_chunks = max(1, args.steps // chunk)
    host_psi = torch.from_numpy(psi0).pin_memory()
    dev_psi = torch.empty_like(psi)
    gc.ch_integrate(dev_psi.copy_(host_psi), g, rhs, DT, 2, gc.RK4)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(n_chunks):
        dev_psi.copy_(host_psi, non_blocking=True)
        gc.ch_integrate(dev_psi, g, rhs, DT, chunk, gc.RK4)
        host_psi.copy_(dev_psi, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ems], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e = world * cells * chunk * n_chunks / (ems / 1e3) / 1e6

    launches = 4 * args.steps  # four stage kernels per RK4 step
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, kind, sample = cpu_sample(1, 2048, 2)
        cpu = {"value": rate, "unit": "Mcell-steps/s", "cores": 1, "kind": kind,
               "sample": f"1 thread, RK4 on 2048x2048, 2 steps ({sample.split(',')[0]})"}
    if rank == 0:
        traffic = None
        if NCU_TRAFFIC_PER_CELL_STEP is not None:
            traffic = NCU_TRAFFIC_PER_CELL_STEP * cells / 4.0
        line = {
            "metric": "Mcell-steps/s (plain FP64 RK4 Cahn-Hilliard)", "value": value, "unit": "Mcell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "ch2d-rk4-fp64-order2", "grid": f"{g.nx}x{g.ny}", "dt": DT, "kappa": 1.0,
                       "mobility": 1.0, "ic": "U[-0.05,0.05] seeded", "l2": "fields 512 MiB each > L2 (no flush)",
                       "parallelism": f"replicas{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "ch_stage_kernel (4 launches per step, 104 B/cell-step algorithmic)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "Mcell-steps/s", "h2d_bytes_per_step": cells * 8 / chunk,
                    "d2h_bytes_per_step": cells * 8 / chunk,
                    "note": f"pinned host field -> device, {chunk} RK4 steps via gc_ch_integrate, device -> host"},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--grid", type=int, default=NX, help="side of the square grid (default 8192)")
    args = ap.parse_args()
    rank, world, local = dist_setup(args.gpus)
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
