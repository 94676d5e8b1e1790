#!/usr/bin/env python
"""Benchmark of the FP64 pressure-Poisson path on the sphere-flow grids.

Default form (the headline line): FFVILS::RBGS on the level-5 FlowPastASphere
grid -- 4692 leaf blocks of 16^3 cells (19,218,432 cells; domain
[-4,12]x[-4,4]x[-4,4], root grid 4x2x2, refined to level 5 within 0.5 of a
unit-diameter sphere) -- with A and b assembled from a seeded
u* = (1,0,0) + N(0, 0.01^2) through the cut-cell assembly, omega = 1.5,
200 sweeps, a residual after every sweep, x reset to zero at the start of
each step.  Metric: Gcell-sweeps/s = cells x sweeps / time.

  value  device time (CUDA events on the pool's stream) of K steps with A, b
         resident in HBM;
  e2e    the same solve through the C ABI with host buffers: upload of
         A (7 fields), b, x from pinned host memory in the reference layout
         (vc = 2), the solve, download of x; copies inside the timed region.
  forms  (one GPU) the three forms below in compact form, measured after the
         headline: the level-5 mixed solve, the 64-instance batch and a
         served run of 100 requests at 50 and 500 req/s (--no-forms skips it).

--impl reference times the reference's CPU path on this machine's host
cores: the C++ restatement in oracle/ (the reference itself cannot be built
here), OpenMP over blocks, on a bounded sample of sweeps per step; it loads
only the oracle library (whose copy of the grid generator builds its inputs).

Other forms (--form), each printing one JSON line of its own:
  mixed  solves/s to a 1e-8 relative residual of the mixed-precision solve
         (FP64 BiCGSTAB recurrence, RB-SOR preconditioner on 32-bit data) against the
         plain FP64 GPU solve (FFVILS::BiCGSTAB, Jacobi PreCount 2), with the
         error of p and grad p against a converged FP64 solution;
  batch  64 independent sphere instances (diameter U[0.5,2], centre in the
         inner half of the domain, max level U{2..5}, seeds 0..63) solved to
         1e-8 in one batch pool by the mixed solve under a captured CUDA
         graph, against one-at-a-time plain FP64 GPU solves.
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
# the same for a uniform block, whose seven coefficients are one record: b + x
# read, x written
BYTES_PER_SWEEP_CELL_UNIFORM = 24


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ffvgpu", choices=["ffvgpu", "reference"])
    ap.add_argument("--form", default="rbsor",
                    choices=["rbsor", "mixed", "batch", "serve", "steps"])
    ap.add_argument("--time-steps", type=int, default=20, help="steps form: time steps")
    ap.add_argument("--agree-iterations", type=int, default=3,
                    help="steps form: BiCGSTAB iterations per step of the oracle comparison")
    ap.add_argument("--sigma", type=float, default=0.05, help="steps form: noise of u*")
    ap.add_argument("--agree-steps", type=int, default=0,
                    help="steps form: steps compared with the oracle (0: all)")
    ap.add_argument("--requests", type=int, default=32, help="serve form: requests per rate")
    ap.add_argument("--rates", default="10,20,50,100,200,500", help="serve form: req/s")
    ap.add_argument("--capacity", type=int, default=40000, help="serve form: pool blocks")
    ap.add_argument("--tune", action="store_true",
                    help="batch form: pick the mixed settings with the autotuner first")
    ap.add_argument("--tune-sample", type=int, default=8,
                    help="batch form: instances the autotuner times each candidate on")
    ap.add_argument("--profile-iterations", type=int, default=0,
                    help="mixed form: only run this many iterations once (for ncu)")
    ap.add_argument("--profile-solver", default="mixed", choices=["mixed", "bicgstab"],
                    help="mixed form with --profile-iterations: the solve to run")
    ap.add_argument("--profile-per-exchange", default="4",
                    help="mixed form with --profile-iterations: comma-separated sweeps per "
                         "exchange, each run with two passes per application")
    ap.add_argument("--profile-fp64-data", action="store_true",
                    help="mixed form with --profile-iterations: also the FP64-data variant")
    ap.add_argument("--level", type=int, default=5)
    ap.add_argument("--instances", type=int, default=64, help="batch form: instances")
    ap.add_argument("--fp64-sample", type=int, default=64,
                    help="batch form: instances solved one at a time in FP64 (a sample)")
    ap.add_argument("--sweeps", type=int, default=200)
    ap.add_argument("--omega", type=float, default=1.5)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU work of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="headline line without the compact mixed/batch/serve figures")
    ap.add_argument("--form-requests", type=int, default=100,
                    help="served requests per rate in the headline line's forms")
    ap.add_argument("--form-rates", default="50,500",
                    help="arrival rates (req/s) of the headline line's served run")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(level, cells, fmt_bytes):
    """DRAM bytes per launch of the sweep kernel from the committed ncu summaries:
    the capture of this level, else the level-3 capture scaled by the bytes of
    the pool's format (uniform blocks at 24 B per cell, the others at 80: the
    share of uniform blocks differs between levels), with its provenance."""
    for lv in (level, 3):
        path = os.path.join(ROOT, "profiles", f"rbgs_sweep_level{lv}_ncu.md")
        if not os.path.exists(path):
            continue
        fields = {}
        for line in open(path):
            for key in ("dram_bytes_per_launch_full_size", "cells_per_launch",
                        "format_bytes_per_launch"):
                if line.startswith(key + ":"):
                    try:
                        fields[key] = float(line.split(":", 1)[1].split()[0])
                    except ValueError:
                        pass
        val = fields.get("dram_bytes_per_launch_full_size")
        if val is None:
            continue
        if lv == level:
            return val, f"ncu, {os.path.basename(path)}"
        if fields.get("format_bytes_per_launch"):
            return (val * fmt_bytes / fields["format_bytes_per_launch"],
                    f"ncu level-{lv} capture scaled by the format bytes")
        if fields.get("cells_per_launch"):
            return val * cells / fields["cells_per_launch"], f"ncu level-{lv} capture scaled by cells"
    return None, None


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


def device_system(level, seed, stream):
    """Pool with u*, cuts generated and A, b assembled on the device (UpdateP
    P02-P05); the same values as the host generator + assembly."""
    import ffvgpu
    g = ffvgpu.SphereGrid(level)
    P = ffvgpu.Pool(g.desc())
    P.set_stream(stream)
    P.assemble_sphere(ffvgpu.sphere_problem(level, seed=seed, sigma=0.01))
    return g, P


def host_info():
    """Host cores and CPU model of this machine, for the CPU legs."""
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else None
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "threads_available": threads or os.cpu_count(),
            "cpu_model": model}


def cpu_problem(level, seed, threads):
    """The oracle (the reference's CPU path restated, OpenMP over blocks) with
    the sphere problem assembled; its inputs come from the generator compiled
    into the oracle library, so the device library is never loaded."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ffv_oracle as fo
    return fo.sphere_problem(level, seed=seed, sigma=0.01, threads=threads,
                             reduction=fo.RED_REFERENCE)


def cpu_sweep_seconds(O, omega, n):
    """Wall time of one RBGS solve of n sweeps (residual every sweep) from x = 0."""
    O.field("X")[...] = 0.0
    t = time.perf_counter()
    O.solve_rbgs(omega, n, 0.0)
    return time.perf_counter() - t


def cpu_baseline(level, seed, sweeps_target, omega, budget_s):
    """Bounded sample of the same solve on the oracle, all host threads: one
    warm-up, then the best of 5 timed repetitions of n sweeps, n sized so the
    repetitions take about budget_s."""
    info = host_info()
    threads = info["threads_available"]
    g, O = cpu_problem(level, seed, threads)
    per = cpu_sweep_seconds(O, omega, 2) / 2  # warm-up and probe
    n = int(max(2, min(sweeps_target, budget_s / 5 / max(per, 1e-9))))
    times = [cpu_sweep_seconds(O, omega, n) for _ in range(5)]
    O.close()
    best = min(times)
    return {"value": g.cells * n / best / 1e9, "unit": "Gcell-sweeps/s", "cores": threads,
            "kind": "port",
            "sample": f"{n} of {sweeps_target} RBSOR sweeps (omega {omega}, residual each sweep) "
                      f"on the {g.nb}-block grid, best of 5 after a warm-up "
                      f"({', '.join(f'{t:.2f}' for t in times)} s); oracle/ C++ restatement, "
                      f"OpenMP over blocks, {threads} threads",
            "host": info}


def run_reference(args):
    """The reference's CPU path on this machine's host cores: the oracle/ C++
    restatement (the reference itself needs Fortran, MPI and BCMTools, none
    of which exist here), OpenMP over blocks on every available thread.  Each
    step is a bounded sample of the workload -- the same grid, problem and
    sweep, with fewer sweeps than the GPU arm's 200 -- sized so that the whole
    --warmup + --steps run takes about four minutes; the rate per sweep does
    not depend on how many sweeps a step runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    info = host_info()
    threads = info["threads_available"]
    g, O = cpu_problem(args.level, args.seed, threads)
    per = cpu_sweep_seconds(O, args.omega, 2) / 2
    budget = 240.0 / max(1, args.steps + args.warmup)
    n = int(max(2, min(args.sweeps, budget / max(per, 1e-9))))
    times = []
    for s in range(args.warmup + args.steps):
        dt = cpu_sweep_seconds(O, args.omega, n)
        if s >= args.warmup:
            times.append(dt)
    O.close()
    tt = float(np.sum(times))
    value = g.cells * n * args.steps / tt / 1e9
    sample = (f"{n} of the {args.sweeps} RBSOR sweeps per step on the {g.nb}-block grid, "
              f"{args.steps} timed steps after {args.warmup} warm-up steps (oracle/ C++ "
              f"restatement of the reference CPU path, OpenMP over blocks, {threads} threads)")
    line = {
        "impl": "reference", "metric": "Gcell-sweeps/s", "value": value, "unit": "Gcell-sweeps/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(g, args),
        "cpu_baseline": {"value": value, "unit": "Gcell-sweeps/s", "cores": threads,
                         "kind": "port", "sample": sample,
                         "best_step_value": g.cells * n / min(times) / 1e9, "host": info},
        "sweeps_per_step": n,
        "e2e": {"value": value, "unit": "Gcell-sweeps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(ms, dist, device):
    """The slowest rank's time (ms): every rank's device-timed region, max-reduced."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms):
    """Whole-job throughput in G units/s: every rank processes units_per_rank
    (weak scaling), all within the slowest rank's time."""
    return world * units_per_rank / (ms * 1e-3) / 1e9


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


# ---------------------------------------------------------------------------
# Other forms
# ---------------------------------------------------------------------------
MIXED = dict(omega=1.5, sweeps=8, sweeps_per_exchange=4)
FP64_SOLVER = dict(omega=1.0, pre_count=2)  # FFV's pbicgstabP (sphere.tpp)


def field_errors(pa, pb, level, root_length=4.0):
    """Relative L2 and max errors of p and of its in-block face differences
    (grad p, divided by each block's cell size) of interiors [nb][k][j][i]."""
    dx = root_length / np.exp2(np.asarray(level, np.float64)) / 16.0
    d = pa - pb
    out = {"p_rel_l2": float(np.linalg.norm(d) / np.linalg.norm(pb)),
           "p_max_rel": float(np.abs(d).max() / np.abs(pb).max())}
    ga, gb = [], []
    for ax in (1, 2, 3):
        ga.append((np.diff(pa, axis=ax) / dx[:, None, None, None]).reshape(-1))
        gb.append((np.diff(pb, axis=ax) / dx[:, None, None, None]).reshape(-1))
    ga, gb = np.concatenate(ga), np.concatenate(gb)
    out["gradp_rel_l2"] = float(np.linalg.norm(ga - gb) / np.linalg.norm(gb))
    out["gradp_max_rel"] = float(np.abs(ga - gb).max() / np.abs(gb).max())
    return out


def timed(stream, fn):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    r = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return r, e0.elapsed_time(e1)


def run_form(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    line = {"mixed": run_mixed, "batch": run_batch, "serve": run_serve,
            "steps": run_steps}[args.form](args)
    print(json.dumps(line), flush=True)
    return 0


def size_table():
    """(level, radius) -> leaf blocks of the sphere grid centred at (4, 0, 0)."""
    import ffvgpu
    table = []
    for L in range(2, 6):
        for r in np.geomspace(0.1, 1.6, 20):
            g = ffvgpu.SphereGrid(L, center=(4.0, 0.0, 0.0), radius=float(r))
            table.append((g.nb, L, float(r)))
    return table


def serve_requests(n, seed, table):
    """Config-5 requests: target block count log-uniform in [100, 8000], met by
    the (max level, radius) of the table whose count is nearest; centre
    uniform in the inner half of the domain; seeded RHS."""
    r = np.random.default_rng(seed)
    out = []
    for k in range(n):
        target = float(np.exp(r.uniform(np.log(100.0), np.log(8000.0))))
        nb, L, rad = min(table, key=lambda t: abs(np.log(t[0] / target)))
        c = r.uniform([0.0, -2.0, -2.0], [8.0, 2.0, 2.0])
        out.append((L, dict(center=tuple(float(v) for v in c), radius=rad), 1000 + k))
    return out


def fifo_latencies(arrivals, service):
    """One server, first come first served: completion - arrival per request."""
    t, lat = 0.0, []
    for a, s_ in zip(arrivals, service):
        t = max(t, a) + s_
        lat.append(t - a)
    return lat


def run_serve(args):
    import torch
    import ffvgpu
    stream = torch.cuda.current_stream()
    table = size_table()
    reqs = serve_requests(args.requests, args.seed, table)
    probs = [ffvgpu.sphere_problem(L, seed=s, sigma=0.01, **kw) for (L, kw, s) in reqs]
    blocks = [ffvgpu.SphereGrid(L, **kw).nb for (L, kw, _) in reqs]
    rates = [float(v) for v in args.rates.split(",")]
    B = ffvgpu.Batch(args.capacity, 64)
    B.set_stream(stream.cuda_stream)
    B.serve([0.0], probs[:1], iterations_per_step=8, count_max=5000)  # warm-up
    per_rate = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for rate in rates:
            rng = np.random.default_rng(int(rate))
            arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(probs)))
            arrivals -= arrivals[0]
            out = B.serve(arrivals, probs, iterations_per_step=8, count_max=5000)
            lat = np.array([o["finish_s"] - o["arrival_s"] for o in out])
            span = max(o["finish_s"] for o in out)
            per_rate.append({"rate": rate, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                             "p99_ms": float(np.percentile(lat, 99) * 1e3),
                             "solves_per_s": len(out) / span,
                             "worst_residual": max(o["residual"] for o in out),
                             "iterations_max": max(o["count"] for o in out)})
    B.close()
    # one-at-a-time plain FP64 GPU solves of the same requests: service times
    service = []
    for (L, kw, s), p in zip(reqs, probs):
        t0 = time.perf_counter()
        g = ffvgpu.SphereGrid(L, **kw)
        P = ffvgpu.Pool(g.desc())
        P.set_stream(stream.cuda_stream)
        P.assemble_sphere(p)
        r = P.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"], 50000, 1e-8,
                             history=False, restart_drop=1e-3)
        P.download("X", 1)
        torch.cuda.synchronize()
        service.append(time.perf_counter() - t0)
        P.close()
    fp64 = []
    for rate in rates:
        rng = np.random.default_rng(int(rate))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(probs)))
        arrivals -= arrivals[0]
        lat = np.array(fifo_latencies(arrivals, service))
        fp64.append({"rate": rate, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                     "p99_ms": float(np.percentile(lat, 99) * 1e3),
                     "solves_per_s": len(service) / float(max(arrivals[i] + lat[i]
                                                              for i in range(len(lat))))})
    top = per_rate[-1]
    line = {
        "form": "serve", "metric": "served solves/s and p50/p99 latency at 1e-8",
        "value": top["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": "f64 arithmetic, 32-bit sweep data", "data": "synthetic",
        "config": {"workload": f"serve-{len(probs)}-requests-per-rate", "rates": rates,
                   "blocks_min_max": [int(min(blocks)), int(max(blocks))],
                   "blocks_total": int(sum(blocks)), "capacity_blocks": args.capacity,
                   "mixed": MIXED, "iterations_per_replay": 8, "epsilon": 1e-8,
                   "requests_rule": "block count log-uniform [100, 8000] via (max level, "
                                    "radius) table, centre U([0,8]x[-2,2]x[-2,2]), Poisson "
                                    "arrivals per rate"},
        "per_rate": per_rate,
        "fp64_one_at_a_time": {"service_s_mean": float(np.mean(service)),
                               "solves_per_s": len(service) / float(np.sum(service)),
                               "solver": "BiCGSTAB omega 1, PreCount 2, restarts 1e-3",
                               "per_rate_fifo": fp64},
        "clocks": clk.summary(),
    }
    return line


def run_mixed(args):
    import torch
    import ffvgpu
    stream = torch.cuda.current_stream()
    g, P = device_system(args.level, args.seed, stream.cuda_stream)
    peak, peak_kind = measured_peaks()
    if args.profile_iterations > 0:  # a fixed, short run for profilers
        P.fill("X", 0.0)
        if args.profile_solver == "bicgstab":
            r = P.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"],
                                 args.profile_iterations, 0.0, history=False)
        else:
            for per in (int(v) for v in args.profile_per_exchange.split(",")):
                for d64 in ((False, True) if args.profile_fp64_data else (False,)):
                    P.fill("X", 0.0)
                    r = P.solve_mixed(MIXED["omega"], 2 * per, per, args.profile_iterations,
                                      0.0, history=False, check_every=args.profile_iterations,
                                      fp64_data=d64)
        P.close()
        return {"form": f"{args.profile_solver}-profile", "level": args.level,
                "blocks": int(g.nb), "iterations": args.profile_iterations,
                "ms": r["elapsed_ms"], "bytes_moved": r["bytes_moved"]}

    def fp64_ref():  # the reference's recurrence, no restarts
        P.fill("X", 0.0)
        return P.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"], 20000, 1e-8,
                                history=False)

    def fp64():  # with the restart option, so that it reaches 1e-8 where the above stalls
        P.fill("X", 0.0)
        return P.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"], 50000, 1e-8,
                                history=False, restart_drop=1e-3)

    def mixed():
        P.fill("X", 0.0)
        return P.solve_mixed(MIXED["omega"], MIXED["sweeps"], MIXED["sweeps_per_exchange"],
                             5000, 1e-8, history=False)

    def rbsor64():  # the same preconditioner on FP64 data: what the 32-bit data buy
        P.fill("X", 0.0)
        return P.solve_mixed(MIXED["omega"], MIXED["sweeps"], MIXED["sweeps_per_exchange"],
                             5000, 1e-8, history=False, fp64_data=True)

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        res = {}
        for name, fn in (("fp64_ref", fp64_ref), ("fp64", fp64), ("rbsor64", rbsor64),
                         ("mixed", mixed)):
            for _ in range(max(1, args.warmup)):
                fn()
            ms, runs = [], []
            for _ in range(args.steps):
                r, t = timed(stream, fn)
                ms.append(t)
                runs.append(r)
            res[name] = (runs[-1], float(np.mean(ms)), runs)
    # errors against a converged FP64 solution of the same system
    P.fill("X", 0.0)
    rref = P.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"], 50000, 1e-11,
                            history=False, restart_drop=1e-3)
    pref = P.download("X", 2)[:, 2:18, 2:18, 2:18].copy()
    mixed()
    pm = P.download("X", 2)[:, 2:18, 2:18, 2:18].copy()
    fp64()
    pf = P.download("X", 2)[:, 2:18, 2:18, 2:18].copy()
    P.close()
    rf, tf, _ = res["fp64"]
    rr_, tr_, _ = res["fp64_ref"]
    rm, tm, _ = res["mixed"]
    rd, td, _ = res["rbsor64"]
    achieved = rm["bytes_moved"] / (tm * 1e-3) / 1e9
    line = {
        "form": "mixed", "metric": "solves/s to 1e-8 relative residual",
        "value": 1e3 / tm, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tm, "higher_is_better": True,
        "dtype": "f64 arithmetic, 32-bit sweep data", "data": "synthetic",
        "config": {"workload": f"mixed-vs-fp64-sphere-level{args.level}", "blocks": int(g.nb),
                   "cells": int(g.cells), "epsilon": 1e-8, "mixed": MIXED,
                   "fp64": dict(FP64_SOLVER, solver="BiCGSTAB (FFVILS.h:793-974)")},
        "fp64": {"solves_per_s": 1e3 / tf, "ms": tf, "iterations": rf["count"],
                 "residual": rf["residual"], "restart_drop": 1e-3},
        "fp64_reference_recurrence": {
            "ms": tr_, "iterations": rr_["count"], "residual": rr_["residual"],
            "reached_1e-8": bool(rr_["status"] == 0 and rr_["count"] > 0 and
                                 rr_["residual"] <= 1e-8),
            "note": "FFVILS::BiCGSTAB as the reference runs it (no restarts); count 0 is its "
                    "|r.r0| < FLT_MIN exit"},
        "mixed": {"solves_per_s": 1e3 / tm, "ms": tm, "iterations": rm["count"],
                  "residual": rm["residual"], "kernel_launches": rm["kernel_launches"]},
        "speedup_vs_fp64": tf / tm,
        "fp64_bicgstab_rbsor": {"solves_per_s": 1e3 / td, "ms": td, "iterations": rd["count"],
                                "residual": rd["residual"],
                                "what": "the same BiCGSTAB and RB-SOR preconditioner with FP64 "
                                        "coefficients, iterate and preconditioned vectors",
                                "achieved_gbs": rd["bytes_moved"] / (td * 1e-3) / 1e9},
        "speedup_vs_fp64_bicgstab_rbsor": td / tm,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "what": "algorithmic bytes of the whole mixed solve "
                     "/ its device time", "peak_source": f"{peak_kind} hbm_gbs"},
        "error_vs_fp64_converged": {"mixed": field_errors(pm, pref, g.level),
                                    "fp64_at_1e-8": field_errors(pf, pref, g.level),
                                    "reference_solution": f"FP64 BiCGSTAB with restarts to "
                                                          f"1e-11 ({rref['count']} iterations, "
                                                          f"residual {rref['residual']:.2e})"},
        "clocks": clk.summary(),
    }
    return line


def run_steps(args):
    """The at-scale workload's time-step loop: --time-steps fractional steps on
    the level-args.level sphere grid, each the pressure part of a step on the
    device in Solver::UpdateP / UpdateU's order (ffvgpu_update_p /
    ffvgpu_update_u: remove_p with the previous pressure, u exchange,
    assembly, BC folding, FP64 BiCGSTAB from the previous pressure to 1e-8,
    p exchange, corr_u, u and p exchanges), with u* = (1,0,0) + N(0, sigma^2)
    regenerated on the device from a per-step seed (the reference's
    convection/diffusion, which would produce u*, is not on this path).
    Then the same steps with --agree-iterations BiCGSTAB iterations per step
    on the device and on the oracle (the reference's CPU path restated, same
    sums), with the per-step pressure agreement."""
    import torch
    import ffvgpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ffv_oracle as fo
    stream = torch.cuda.current_stream()
    level, nsteps, sigma = args.level, args.time_steps, args.sigma
    g = ffvgpu.SphereGrid(level)
    peak, peak_kind = measured_peaks()

    def device_pool():
        P = ffvgpu.Pool(g.desc())
        P.set_stream(stream.cuda_stream)
        P.assemble_sphere(ffvgpu.sphere_problem(level, seed=args.seed, sigma=sigma))
        P.fill("X", 0.0)
        return P

    def step(P, n, count_max, eps, restart):
        P.generate_sphere(ffvgpu.sphere_problem(level, seed=args.seed + n, sigma=sigma))
        r = P.update_p(ffvgpu.SOLVER_BICGSTAB, omega=FP64_SOLVER["omega"],
                       pre_count=FP64_SOLVER["pre_count"], count_max=count_max, epsilon=eps,
                       restart_drop=restart)
        P.update_u()
        return r

    # ---- timed: every step solved to 1e-8 --------------------------------
    P = device_pool()
    for n in range(max(1, args.warmup)):  # warm-up steps on a separate history
        step(P, 1000 + n, 50000, 1e-8, 1e-3)
    P.close()
    P = device_pool()
    per_step = []
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for n in range(nsteps):
            r, t = timed(stream, lambda: step(P, n, 50000, 1e-8, 1e-3))
            per_step.append({"step": n, "ms": t, "solve_ms": r["elapsed_ms"],
                             "iterations": r["count"], "residual": r["residual"],
                             "solve_gbs": r["bytes_moved"] / (r["elapsed_ms"] * 1e-3) / 1e9})
    P.close()
    tot = float(sum(x["ms"] for x in per_step))
    solve_gbs = [x["solve_gbs"] for x in per_step]

    # ---- agreement with the oracle, a bounded solve per step ---------------
    K = args.agree_iterations
    P = device_pool()
    O = fo.sphere_problem(level, seed=args.seed, sigma=sigma, threads=host_info()["threads_available"],
                          reduction=fo.RED_CANONICAL)[1]
    O.field("X")[...] = 0.0
    go = fo.SphereGrid(level)
    agree = []
    t0 = time.perf_counter()
    for n in range(args.agree_steps if args.agree_steps > 0 else nsteps):
        rg = step(P, n, K, 0.0, 0.0)
        ro = fo.time_step(O, go.fill_u(seed=args.seed + n, sigma=sigma, vc=2),
                          lambda o: o.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"],
                                                     K, 0.0))
        pg = P.download("X", 2)[:, 2:18, 2:18, 2:18]
        po = O.field("X")[:, 2:18, 2:18, 2:18]
        d = float(np.abs(pg - po).max() / max(np.abs(po).max(), 1e-300))
        agree.append({"step": n, "p_max_rel_diff": d, "bitwise": bool(np.array_equal(pg, po)),
                      "residual_gpu": rg["residual"], "residual_oracle": ro["residual"]})
    oracle_s = time.perf_counter() - t0
    P.close()
    O.close()
    line = {
        "form": "steps", "metric": "fractional steps/s (pressure part, FP64 BiCGSTAB to 1e-8)",
        "value": 1e3 * nsteps / tot, "unit": "steps/s", "n_gpus": 1, "steps": nsteps,
        "warmup": max(1, args.warmup), "ms_per_step": tot / nsteps, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"time-steps-sphere-level{level}", "blocks": int(g.nb),
                   "cells": int(g.cells), "sigma": sigma, "seeds": [args.seed, args.seed + nsteps - 1],
                   "dt": 0.002, "rhof": 1.0,
                   "solver": dict(FP64_SOLVER, solver="BiCGSTAB", epsilon=1e-8, restart_drop=1e-3),
                   "sequence": "generate u*; remove_p; exchange u; assemble; fold BCs; solve; "
                               "exchange p; corr_u; exchange u; exchange p"},
        "per_step": per_step,
        "solve_hbm": {"achieved_gbs_median": float(np.median(solve_gbs)), "peak": peak,
                      "frac_median": float(np.median(solve_gbs)) / peak,
                      "peak_source": f"{peak_kind} hbm_gbs"},
        "oracle_agreement": {"iterations_per_step": K, "steps": agree,
                             "all_bitwise": all(a["bitwise"] for a in agree),
                             "max_p_rel_diff": max(a["p_max_rel_diff"] for a in agree),
                             "oracle_seconds": oracle_s,
                             "oracle": "reference CPU path restated (oracle/), canonical sums"},
        "clocks": clk.summary(),
    }
    return line


def batch_instances(n):
    """Config-4 instances: diameter U[0.5,2], centre U([0,8]x[-2,2]x[-2,2]),
    max level U{2..5}, seeds 0..n-1."""
    out = []
    for seed in range(n):
        r = np.random.default_rng(seed)
        d = r.uniform(0.5, 2.0)
        c = r.uniform([0.0, -2.0, -2.0], [8.0, 2.0, 2.0])
        L = int(r.integers(2, 6))
        out.append((L, dict(center=tuple(float(v) for v in c), radius=d / 2.0), seed))
    return out


def run_batch(args):
    import torch
    import ffvgpu
    stream = torch.cuda.current_stream()
    insts = batch_instances(args.instances)
    grids = [ffvgpu.SphereGrid(L, **kw) for (L, kw, _) in insts]
    blocks = [gr.nb for gr in grids]
    total = int(sum(blocks))
    peak, peak_kind = measured_peaks()
    B = ffvgpu.Batch(total, len(insts))
    B.set_stream(stream.cuda_stream)
    t0 = time.perf_counter()
    ids = [B.admit_sphere(ffvgpu.sphere_problem(L, seed=s, sigma=0.01, **kw))
           for (L, kw, s) in insts]
    torch.cuda.synchronize()
    admit_s = time.perf_counter() - t0
    assert all(i is not None for i in ids)

    setting = dict(MIXED, iterations_per_replay=8, threads_per_block=256, stage_depth=1,
                   sweep_threads=256, matvec_form=0)
    tune = None
    if args.tune:
        # a sample spread over the instance sizes (every k-th by block count)
        order = sorted(range(len(ids)), key=lambda k: blocks[k])
        step = max(1, len(order) // max(1, args.tune_sample))
        sample = [ids[k] for k in order[::step][:args.tune_sample]]
        t0 = time.perf_counter()
        recs, best = B.autotune(sample)
        tune = {"sample_instances": len(sample),
                "sample_blocks": int(sum(B.blocks(i) for i in sample)),
                "candidates": len(recs), "seconds": time.perf_counter() - t0,
                "converged_candidates": sum(r["converged"] for r in recs),
                "best": recs[best] if best >= 0 else None,
                "default": next((r for r in recs if r["omega"] == MIXED["omega"] and
                                 r["sweeps"] == MIXED["sweeps"] and
                                 r["sweeps_per_exchange"] == MIXED["sweeps_per_exchange"] and
                                 r["iterations_per_replay"] == 8 and
                                 r["threads_per_block"] == 256 and r["stage_depth"] == 1 and
                                 r["sweep_threads"] == 256 and r["matvec_form"] == 0), None)}
        if best >= 0:
            b = recs[best]
            setting = dict(omega=b["omega"], sweeps=b["sweeps"],
                           sweeps_per_exchange=b["sweeps_per_exchange"],
                           iterations_per_replay=b["iterations_per_replay"],
                           threads_per_block=b["threads_per_block"],
                           stage_depth=b["stage_depth"], sweep_threads=b["sweep_threads"],
                           matvec_form=b["matvec_form"])

    def batched():
        for i in ids:
            B.fill(i, "X", 0.0)
        return B.solve_mixed(setting["omega"], setting["sweeps"], setting["sweeps_per_exchange"],
                             5000, 1e-8, check_every=setting["iterations_per_replay"],
                             threads_per_block=setting["threads_per_block"],
                             stage_depth=setting["stage_depth"],
                             sweep_threads=setting["sweep_threads"],
                             matvec_form=setting["matvec_form"])

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(max(1, args.warmup)):
            batched()
        ms, r = [], None
        for _ in range(args.steps):
            r, t = timed(stream, batched)
            ms.append(t)
    tb = float(np.mean(ms))
    results = [B.result(i) for i in ids]
    iters = [x["count"] for x in results]
    worst = max(x["residual"] for x in results)
    achieved = r["bytes_moved"] / (tb * 1e-3) / 1e9
    # the same batched solve with the preconditioner on FP64 data: what the
    # 32-bit data buy, on the same instances, batch and graph
    for i in ids:
        B.fill(i, "X", 0.0)
    r64, t64b = timed(stream, lambda: B.solve_mixed(
        setting["omega"], setting["sweeps"], setting["sweeps_per_exchange"], 5000, 1e-8,
        check_every=setting["iterations_per_replay"], fp64_data=True,
        threads_per_block=setting["threads_per_block"], stage_depth=setting["stage_depth"],
        sweep_threads=setting["sweep_threads"], matvec_form=setting["matvec_form"]))
    res64 = [B.result(i) for i in ids]
    rbsor64 = {"solves_per_s": 1e3 * len(ids) / t64b, "ms": t64b,
               "iterations_min_max": [int(min(x["count"] for x in res64)),
                                      int(max(x["count"] for x in res64))],
               "worst_residual": max(x["residual"] for x in res64),
               "achieved_gbs": r64["bytes_moved"] / (t64b * 1e-3) / 1e9,
               "what": "the same batched BiCGSTAB and RB-SOR preconditioner with FP64 "
                       "coefficients, iterate and preconditioned vectors"}
    dev_gb = B.device_bytes / 1e9
    B.close()
    # one-at-a-time plain FP64 GPU solves (and mixed, alone) of a sample
    n_s = min(args.fp64_sample, len(insts))
    sample = list(range(len(insts)))[:: max(1, len(insts) // n_s)][:n_s]
    t64, tmix, it64 = 0.0, 0.0, []
    for k in sample:
        L, kw, s = insts[k]
        P = ffvgpu.Pool(grids[k].desc())
        P.set_stream(stream.cuda_stream)
        P.assemble_sphere(ffvgpu.sphere_problem(L, seed=s, sigma=0.01, **kw))

        def f64():
            P.fill("X", 0.0)
            return P.solve_bicgstab(FP64_SOLVER["omega"], FP64_SOLVER["pre_count"], 50000, 1e-8,
                                    history=False, restart_drop=1e-3)

        def mx():
            P.fill("X", 0.0)
            return P.solve_mixed(MIXED["omega"], MIXED["sweeps"], MIXED["sweeps_per_exchange"],
                                 5000, 1e-8, history=False)

        f64()
        rr, t = timed(stream, f64)
        t64 += t
        it64.append(rr["count"])
        mx()
        _, t = timed(stream, mx)
        tmix += t
        P.close()
    fp64_sps = len(sample) / (t64 * 1e-3)
    alone_sps = len(sample) / (tmix * 1e-3)
    line = {
        "form": "batch", "metric": "solves/s to 1e-8 relative residual", "value": 1e3 * len(ids) / tb,
        "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tb, "higher_is_better": True, "dtype": "f64 arithmetic, 32-bit sweep data",
        "data": "synthetic",
        "config": {"workload": f"batch-{len(ids)}-sphere-instances", "instances": len(ids),
                   "blocks": total, "cells": total * CELLS_PER_BLOCK,
                   "blocks_min_max": [int(min(blocks)), int(max(blocks))], "epsilon": 1e-8,
                   "mixed": setting, "autotuned": bool(args.tune),
                   "instances_rule": "diameter U[0.5,2], centre U([0,8]x[-2,2]x[-2,2]), "
                                     "max level U{2..5}, seed = index"},
        "iterations_min_max": [int(min(iters)), int(max(iters))], "worst_residual": worst,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "what": "algorithmic bytes of the batched solve / "
                     "its device time", "peak_source": f"{peak_kind} hbm_gbs"},
        "fp64_one_at_a_time": {"solves_per_s": fp64_sps, "sample": len(sample),
                               "iterations_min_max": [int(min(it64)), int(max(it64))],
                               "solver": "BiCGSTAB omega 1, PreCount 2"},
        "mixed_one_at_a_time": {"solves_per_s": alone_sps, "sample": len(sample)},
        "speedup_vs_fp64_one_at_a_time": (1e3 * len(ids) / tb) / fp64_sps,
        "fp64_rbsor_batched": rbsor64,
        "speedup_vs_fp64_rbsor_batched": t64b / tb,
        "admission_s": admit_s, "device_gb": dev_gb, "autotune": tune, "clocks": clk.summary(),
    }
    return line


def forms_summary(args):
    """The three forms in compact form for the headline line (one GPU, rank 0):
    the level-5 mixed solve against the plain FP64 GPU solve, the 64-instance
    batch, and a served run of args.form_requests requests at two arrival
    rates.  Each entry keeps the figures of its own --form line; a form that
    fails records its error instead of stopping the line."""
    import copy
    out = {}
    t_all = time.perf_counter()
    plans = (
        ("mixed_level5", run_mixed, dict(level=5, steps=2, warmup=1, profile_iterations=0)),
        ("batch64", run_batch, dict(instances=64, steps=1, warmup=1, tune=False, fp64_sample=64)),
        ("serve", run_serve, dict(requests=args.form_requests, rates=args.form_rates,
                                  capacity=40000)),
        ("steps_level5", run_steps, dict(level=5, time_steps=20, warmup=1, agree_steps=3,
                                         agree_iterations=3, sigma=0.05)),
    )
    for name, fn, over in plans:
        a = copy.copy(args)
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        try:
            ln = fn(a)
        except Exception as e:  # recorded, the headline stands
            out[name] = {"error": f"{type(e).__name__}: {e}"}
            continue
        sec = time.perf_counter() - t0
        if name == "mixed_level5":
            out[name] = {
                "solves_per_s": ln["value"], "ms": ln["ms_per_step"],
                "iterations": ln["mixed"]["iterations"], "residual": ln["mixed"]["residual"],
                "fp64_bicgstab_jacobi": {k: ln["fp64"][k] for k in ("solves_per_s", "ms",
                                                                     "iterations")},
                "speedup_vs_fp64_bicgstab_jacobi": ln["speedup_vs_fp64"],
                "hbm_frac": ln["roofline"]["frac"], "achieved_gbs": ln["roofline"]["achieved"],
                "error_vs_fp64_converged": ln["error_vs_fp64_converged"]["mixed"],
                "clocks": ln["clocks"], "seconds": sec}
            for k in ("fp64_bicgstab_rbsor", "speedup_vs_fp64_bicgstab_rbsor"):
                if k in ln:
                    out[name][k] = ln[k]
        elif name == "batch64":
            out[name] = {
                "solves_per_s": ln["value"], "ms": ln["ms_per_step"],
                "blocks": ln["config"]["blocks"], "iterations_min_max": ln["iterations_min_max"],
                "worst_residual": ln["worst_residual"], "hbm_frac": ln["roofline"]["frac"],
                "achieved_gbs": ln["roofline"]["achieved"],
                "fp64_one_at_a_time": ln["fp64_one_at_a_time"],
                "speedup_vs_fp64_one_at_a_time": ln["speedup_vs_fp64_one_at_a_time"],
                "clocks": ln["clocks"], "seconds": sec}
            for k in ("fp64_rbsor_batched", "speedup_vs_fp64_rbsor_batched"):
                if k in ln:
                    out[name][k] = ln[k]
        elif name == "steps_level5":
            out[name] = {
                "steps_per_s": ln["value"], "ms_per_step": ln["ms_per_step"],
                "iterations_per_step": [x["iterations"] for x in ln["per_step"]],
                "solve_hbm_frac_median": ln["solve_hbm"]["frac_median"],
                "solve_gbs_median": ln["solve_hbm"]["achieved_gbs_median"],
                "oracle_agreement": {k: ln["oracle_agreement"][k] for k in
                                     ("iterations_per_step", "all_bitwise", "max_p_rel_diff")},
                "oracle_steps_compared": len(ln["oracle_agreement"]["steps"]),
                "clocks": ln["clocks"], "seconds": sec}
        else:
            out[name] = {
                "requests_per_rate": args.form_requests,
                "blocks_min_max": ln["config"]["blocks_min_max"],
                "per_rate": [{k: r[k] for k in ("rate", "p50_ms", "p99_ms", "solves_per_s")}
                             for r in ln["per_rate"]],
                "fp64_one_at_a_time_fifo": [{k: r[k] for k in ("rate", "p50_ms", "p99_ms")}
                                            for r in ln["fp64_one_at_a_time"]["per_rate_fifo"]],
                "fp64_one_at_a_time_solves_per_s": ln["fp64_one_at_a_time"]["solves_per_s"],
                "clocks": ln["clocks"], "seconds": sec}
    out["seconds"] = time.perf_counter() - t_all
    return out


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
    if args.form != "rbsor":
        if world > 1:
            raise SystemExit("--form mixed/batch run on one GPU")
        return run_form(args)
    stream = torch.cuda.current_stream()
    g, P = device_system(args.level, args.seed, stream.cuda_stream)
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
    t_ms = max_over_ranks(t_ms, dist, "cuda")
    value = whole_job_rate(world, cells * args.sweeps * args.steps, t_ms)

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
    # The host buffers hold the reference layout ((16+2vc)^3 per block); from
    # pinned memory the pack kernel reads across the link only the interior
    # (and for x its first guide layer): those are the bytes moved up.  The
    # download writes the whole layout (interior, guide layers, zeros).
    host_bytes = (len(pinned) + 1) * per_field * 8
    h2d = (len(pinned) * CELLS_PER_BLOCK + CELLS_PER_BLOCK + 6 * 256) * g.nb * 8
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
    te_ms = max_over_ranks(te_ms, dist, "cuda")
    e2e_value = whole_job_rate(world, cells * args.sweeps * args.steps, te_ms)

    # ---- roofline of the dominant kernel (fused residual + RB sweep) ---------
    # achieved: the fixed algorithmic bytes of an RB sweep with its residual,
    # 80 B per interior cell (7 coefficients + b + x read, x written), over
    # the kernel's average launch; 'traffic' is what the kernel moves from
    # DRAM (ncu), below the algorithmic bytes because a uniform block's seven
    # coefficients come from one record (its pass moves 24 B per cell)
    avg_launch_ms = float(np.sum(sweep_ms) / max(1, np.sum(sweep_n)))
    ublocks = int(r.get("uniform_blocks", 0))
    alg_bytes = BYTES_PER_SWEEP_CELL * cells
    fmt_bytes = CELLS_PER_BLOCK * ((g.nb - ublocks) * BYTES_PER_SWEEP_CELL +
                                   ublocks * BYTES_PER_SWEEP_CELL_UNIFORM)
    achieved = alg_bytes / (avg_launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic, traffic_src = profile_traffic(args.level, cells, fmt_bytes)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                "kernel": "rbgs_pipelined_kernel<res,sweep> (fused residual + red-black sweep)",
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_launch_ms,
                "bytes_per_cell": BYTES_PER_SWEEP_CELL, "uniform_blocks": ublocks,
                "format_bytes_per_launch": fmt_bytes,
                "format_bytes_per_cell": f"{BYTES_PER_SWEEP_CELL} (per-cell coefficients), "
                                         f"{BYTES_PER_SWEEP_CELL_UNIFORM} (uniform block)",
                "format_gbs": fmt_bytes / (avg_launch_ms * 1e-3) / 1e9,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.level, args.seed, args.sweeps, args.omega, args.cpu_seconds)

    P.close()
    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        forms = forms_summary(args)

    if rank == 0:
        line = {
            "metric": "Gcell-sweeps/s", "value": value, "unit": "Gcell-sweeps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(g, args),
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gcell-sweeps/s", "h2d_bytes_per_step": h2d,
                    "h2d_host_buffer_bytes": host_bytes,
                    "d2h_bytes_per_step": d2h, "ms_per_step": te_ms / args.steps},
            "clocks": clk.summary(), "gpu_launches": launches,
        }
        if forms is not None:
            line["forms"] = forms
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
