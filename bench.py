#!/usr/bin/env python
"""Benchmark: FP64 red-black SOR pressure solve on the level-3 sphere grid.

Workload (one "step"): FFVILS::RBGS on the FlowPastASphere-shaped grid of
548 leaf blocks of 16^3 cells (2,244,608 cells; domain [-4,12]x[-4,4]x[-4,4],
root grid 4x2x2, refined to level 3 within 0.5 of a unit-diameter sphere),
A and b assembled from a seeded u* = (1,0,0) + N(0, 0.01^2) through the
cut-cell assembly, omega = 1.5, 200 sweeps, a residual after every sweep,
x reset to zero at the start of each step.  Metric: Gcell-sweeps/s =
cells x sweeps / time.

  value  device time (CUDA events on the pool's stream) of K steps with A, b
         resident in HBM;
  e2e    the same solve through the C ABI with host buffers: upload of
         A (7 fields), b, x from pinned host memory in the reference layout
         (vc = 2), the solve, download of x; copies inside the timed region.

--impl reference times the reference's CPU path on this machine's host
cores: the C++ restatement in oracle/ (the reference itself cannot be built
here), OpenMP over blocks, on a bounded sample of sweeps per step.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ffv-hc_b200"))

CELLS_PER_BLOCK = 4096
BYTES_PER_SWEEP_CELL = 80  # 7 coefficients + b + x read, x written (FP64)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ffvgpu", choices=["ffvgpu", "reference"])
    ap.add_argument("--level", type=int, default=3)
    ap.add_argument("--sweeps", type=int, default=200)
    ap.add_argument("--omega", type=float, default=1.5)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU work of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the sweep kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "rbgs_sweep_level3_ncu.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch_full_size:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def build_problem(level, seed):
    import ffvgpu
    g = ffvgpu.SphereGrid(level)
    inp = g.fill(seed=seed, sigma=0.01, vc=2)
    return g, inp


def device_system(g, inp, stream):
    """Pool with A, b assembled on the device (UpdateP P02-P05)."""
    import ffvgpu
    P = ffvgpu.Pool(g.desc())
    P.set_stream(stream)
    for k, v in inp.items():
        P.upload(k, v, 2)
    for u in ("UX", "UY", "UZ"):
        P.exchange(u, ffvgpu.U_BC_TYPE, ffvgpu.U_BC_VALUE[u])
    P.assemble_p(1.0, 0.002)
    P.fold_bc()
    return P


def cpu_baseline(g, inp, sweeps_target, omega, budget_s):
    """The oracle (reference CPU path restated) on all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ffv_oracle as fo
    import ffvgpu
    threads = os.cpu_count() or 1
    O = fo.Oracle.from_grid(g, vc=2, bc_type=ffvgpu.P_BC_TYPE, bc_value=ffvgpu.P_BC_VALUE,
                            threads=threads, reduction=fo.RED_REFERENCE)
    for k, v in inp.items():
        O.field(k)[...] = v
    for u in ("UX", "UY", "UZ"):
        O.exchange(u, ffvgpu.U_BC_TYPE, ffvgpu.U_BC_VALUE[u])
    O.assemble_p(1.0, 0.002)
    O.fold_bc()
    # probe, then size the sample to the budget
    O.field("X")[...] = 0.0
    t = time.perf_counter()
    O.solve_rbgs(omega, 2, 0.0)
    per = (time.perf_counter() - t) / 2
    n = int(max(2, min(sweeps_target, budget_s / max(per, 1e-9))))
    O.field("X")[...] = 0.0
    t = time.perf_counter()
    O.solve_rbgs(omega, n, 0.0)
    dt = time.perf_counter() - t
    O.close()
    value = g.cells * n / dt / 1e9
    return {"value": value, "unit": "Gcell-sweeps/s", "cores": threads, "kind": "port",
            "sample": f"{n} of {sweeps_target} RBSOR sweeps (omega {omega}, residual each sweep) "
                      f"on the {g.nb}-block grid, oracle/ C++ restatement, OpenMP over blocks, "
                      f"{threads} threads, {dt:.2f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    g, inp = build_problem(args.level, args.seed)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ffv_oracle as fo
    import ffvgpu
    threads = os.cpu_count() or 1
    O = fo.Oracle.from_grid(g, vc=2, bc_type=ffvgpu.P_BC_TYPE, bc_value=ffvgpu.P_BC_VALUE,
                            threads=threads, reduction=fo.RED_REFERENCE)
    for k, v in inp.items():
        O.field(k)[...] = v
    for u in ("UX", "UY", "UZ"):
        O.exchange(u, ffvgpu.U_BC_TYPE, ffvgpu.U_BC_VALUE[u])
    O.assemble_p(1.0, 0.002)
    O.fold_bc()
    O.field("X")[...] = 0.0
    t = time.perf_counter()
    O.solve_rbgs(args.omega, 2, 0.0)
    per = (time.perf_counter() - t) / 2
    budget = 120.0 / max(1, args.steps + args.warmup)
    n = int(max(2, min(args.sweeps, budget / max(per, 1e-9))))
    times = []
    for s in range(args.warmup + args.steps):
        O.field("X")[...] = 0.0
        t = time.perf_counter()
        O.solve_rbgs(args.omega, n, 0.0)
        dt = time.perf_counter() - t
        if s >= args.warmup:
            times.append(dt)
    O.close()
    tt = float(np.sum(times))
    value = g.cells * n * args.steps / tt / 1e9
    line = {
        "impl": "reference", "metric": "Gcell-sweeps/s", "value": value, "unit": "Gcell-sweeps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(g, args, extra={"cpu_sweeps_per_step": n}),
        "cpu_baseline": {"value": value, "unit": "Gcell-sweeps/s", "cores": threads,
                         "kind": "port",
                         "sample": f"{n} RBSOR sweeps per step on the {g.nb}-block grid "
                                   f"(oracle/ C++ restatement of the reference CPU path; the "
                                   f"reference needs Fortran/MPI/BCMTools, absent here)"},
        "e2e": {"value": value, "unit": "Gcell-sweeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(g, args, extra=None):
    c = {"workload": f"rbsor-fp64-sphere-level{args.level}", "blocks": int(g.nb),
         "cells": int(g.cells), "sweeps": args.sweeps, "omega": args.omega,
         "residual_every_sweep": True, "grid": "domain [-4,12]x[-4,4]x[-4,4], root 4x2x2, "
         "16^3 leaf blocks, sphere d=1 at origin, margin 0.5, 2:1 balanced",
         "rhs": "div(u*)/dt through bcut_calc_ab_p, u*=(1,0,0)+N(0,0.01^2), dt=0.002, seeded",
         "l2": "inputs larger than L2 (working set ~%d MB)" % (g.cells * 80 // 2 ** 20),
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import ffvgpu
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    stream = torch.cuda.current_stream()
    g, inp = build_problem(args.level, args.seed)
    P = device_system(g, inp, stream.cuda_stream)
    cells = g.cells

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing -------------------------------------------
    sweep_ms, sweep_n, launches = [], [], 0
    for _ in range(args.warmup):
        P.fill("X", 0.0)
        P.solve_rbgs(args.omega, args.sweeps, 0.0, history=False)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            P.fill("X", 0.0)
            r = P.solve_rbgs(args.omega, args.sweeps, 0.0, history=False)
            sweep_ms.append(r["sweep_ms"])
            sweep_n.append(r["sweep_launches"])
            launches += r["kernel_launches"] + 1
        ev1.record(stream)
        torch.cuda.synchronize()
    t_ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([t_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_ms = float(t.item())
    value = world * cells * args.sweeps * args.steps / (t_ms * 1e-3) / 1e9

    # ---- end-to-end through the C ABI with host buffers ---------------------
    w = 20
    per_field = g.nb * w ** 3
    pinned = {}
    for name in ("AP", "AW", "AE", "AS", "AN", "AB", "AT", "B"):
        t = torch.empty(per_field, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = P.download(name, 2).reshape(-1)
        pinned[name] = t
    xin = torch.zeros(per_field, dtype=torch.float64, pin_memory=True)
    xout = torch.empty(per_field, dtype=torch.float64, pin_memory=True)
    h2d = (len(pinned) + 1) * per_field * 8
    d2h = per_field * 8

    def e2e_step():
        for name, t in pinned.items():
            P.upload_ptr(name, t.data_ptr(), 2)
        P.upload_ptr("X", xin.data_ptr(), 2)
        r = P.solve_rbgs(args.omega, args.sweeps, 0.0, history=False)
        P.download_ptr("X", xout.data_ptr(), 2)
        return r

    for _ in range(max(1, args.warmup)):
        e2e_step()
    barrier()
    e2e_launches = 0
    ev0.record(stream)
    for _ in range(args.steps):
        e2e_launches += e2e_step()["kernel_launches"]
    ev1.record(stream)
    torch.cuda.synchronize()
    te_ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([te_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        te_ms = float(t.item())
    e2e_value = world * cells * args.sweeps * args.steps / (te_ms * 1e-3) / 1e9

    # ---- roofline of the dominant kernel (fused residual + RB sweep) ---------
    avg_launch_ms = float(np.sum(sweep_ms) / max(1, np.sum(sweep_n)))
    alg_bytes = BYTES_PER_SWEEP_CELL * cells
    achieved = alg_bytes / (avg_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profile_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": "rbgs_kernel<res,sweep> (fused residual + red-black sweep)",
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_launch_ms,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(g, inp, args.sweeps, args.omega, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": "Gcell-sweeps/s", "value": value, "unit": "Gcell-sweeps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(g, args),
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gcell-sweeps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": te_ms / args.steps},
            "clocks": clk.summary(), "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    P.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
