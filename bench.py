#!/usr/bin/env python
"""Benchmark of the PDHG-for-OT hot path on B200.

Workload: one OT instance with m = 20000 sources and n = 15000 targets, points
drawn from a 2-D mixture of 8 isotropic Gaussians (sigma 0.05, means U[0,1]^2,
seeded, not clipped), C = squared Euclidean distance / max (FP64, 2.4 GB),
marginals U(0.1, 1) normalised; the FP64 drop-in solver with the reference
script's parameters (tolerance 1e-4).

A step is one PDHG iteration (one loop body of optimize(): the fused primal
pass, the dual step and, on the reference's schedule, an evaluation). The
metric is iterations per second with the problem resident in HBM; the inputs
(7.2 GB of C, X, Xavg) are far larger than L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU runs are replicas (one independent solve per GPU, weak scaling):
a single OT solve has one all-reduce per iteration and is not sharded here.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "pdot.jl_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "time-to-KKT≤1e-4 and PDHG iters/s at n=20000 (plain vs MP+warm-start); % HBM roofline"
UNIT = "iters/s"
M_ROWS, N_COLS, SEED, TOL = 20000, 15000, 0, 1e-4
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes per matrix entry of one fused primal pass, from the ncu capture
# summarised in profiles/k1_primal_fp64.md (None until captured).
K1_DRAM_BYTES_PER_ENTRY = None
CPU_SAMPLE_ROWS = 500  # row slice of the instance timed on the host cores


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--m", type=int, default=M_ROWS)
    ap.add_argument("--n", type=int, default=N_COLS)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ttk", action="store_true", help="skip the time-to-KKT solve")
    return ap.parse_args()


def host_instance(m, n, seed):
    """Points and marginals (host, seeded), as pdot.instances.gauss_mixture draws them."""
    import numpy as np

    from pdot import instances

    rng = np.random.default_rng(seed)
    xs = instances.gauss_mixture_points(rng, m)
    ys = instances.gauss_mixture_points(rng, n)
    a = rng.uniform(0.1, 1.0, size=m)
    b = rng.uniform(0.1, 1.0, size=n)
    return xs, ys, a / a.sum(), b / b.sum()


def device_cost(xs, ys, device):
    """C (column-major m x n) built on the device: a (n, m) row-major tensor
    whose row j is column j of C."""
    import torch

    x = torch.from_numpy(xs).to(device)
    y = torch.from_numpy(ys).to(device)
    Ct = (y[:, 0:1] - x[None, :, 0]).square_()
    for k in range(1, xs.shape[1]):
        Ct.add_((y[:, k : k + 1] - x[None, :, k]).square_())
    Ct.div_(Ct.max())
    return Ct


def is_eval(it, freq=128, limit=2**31 - 1):
    return (it - 1) % freq == 0 or it == limit + 1 or it <= 10


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i",
                 str(self.gpu), "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def read_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def cpu_sample_problem(xs, ys, a, b, rows):
    """Rows [0, rows) of the instance (the same cost entries, source marginal
    renormalised), for timing on the host cores."""
    import numpy as np

    from pdot import api

    x, y = xs[:rows], ys
    C = np.zeros((rows, y.shape[0]), order="F")
    for k in range(x.shape[1]):
        C += (x[:, k : k + 1] - y[None, :, k]) ** 2
    full_max = 0.0
    for k0 in range(0, xs.shape[0], 2000):  # max over the full instance, in blocks
        blk = np.zeros((min(2000, xs.shape[0] - k0), y.shape[0]))
        for k in range(x.shape[1]):
            blk += (xs[k0 : k0 + 2000, k : k + 1] - y[None, :, k]) ** 2
        full_max = max(full_max, float(blk.max()))
    C /= full_max
    return api.OptimalTransportProblem(C, a[:rows] / a[:rows].sum(), b)


def cpu_baseline(xs, ys, a, b, m, n, steps):
    import oracle
    import pdot

    prob = cpu_sample_problem(xs, ys, a, b, CPU_SAMPLE_ROWS)
    cores = os.cpu_count() or 1
    sec = oracle.time_steps(pdot.default_parameters(TOL), prob, steps, cores)
    scale = (CPU_SAMPLE_ROWS * n) / float(m * n)
    return {"value": steps / sec * scale, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} PDHG iterations of the FP64 oracle on rows 0..{CPU_SAMPLE_ROWS - 1} of the "
                      f"{m}x{n} instance ({CPU_SAMPLE_ROWS * n} entries), per-iteration time scaled by "
                      f"{m}/{CPU_SAMPLE_ROWS} to the full size",
            "seconds": sec}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def run_reference(args, world, rank):
    """CPU implementation of the path on the host cores (the oracle port; the
    reference is Julia and no Julia toolchain is installed)."""
    if rank != 0:
        return None
    import oracle
    import pdot

    xs, ys, a, b = host_instance(args.m, args.n, SEED)
    prob = cpu_sample_problem(xs, ys, a, b, CPU_SAMPLE_ROWS)
    cores = os.cpu_count() or 1
    params = pdot.default_parameters(TOL)
    if args.warmup > 0:
        oracle.time_steps(params, prob, args.warmup, cores)
    sec = oracle.time_steps(params, prob, args.steps, cores)
    scale = (CPU_SAMPLE_ROWS * args.n) / float(args.m * args.n)
    value = args.steps / sec * scale
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"PDHG-OT m={args.m} n={args.n} gauss-mixture sq-euclid/max FP64, tol {TOL}",
                   "implementation": "FP64 CPU restatement of the reference algorithm (OpenMP), "
                                     "the reference itself is Julia and cannot run here"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"each step one PDHG iteration on rows 0..{CPU_SAMPLE_ROWS - 1} of the "
                                   f"instance, time scaled by {args.m}/{CPU_SAMPLE_ROWS}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import pdot

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    m, n = args.m, args.n
    N = m * n
    xs, ys, a_h, b_h = host_instance(m, n, SEED)
    Ct = device_cost(xs, ys, device)
    a = torch.from_numpy(a_h).to(device)
    b = torch.from_numpy(b_h).to(device)
    torch.cuda.synchronize()
    dev_problem = (m, n, Ct.data_ptr(), a.data_ptr(), b.data_ptr())
    params = pdot.default_parameters(TOL)
    params.termination_criteria.time_sec_limit = 300.0

    # ---- timed region: K iterations, problem resident, CUDA graphs ----
    solver = pdot.Solver(params, device_problem=dev_problem, device=local)
    s0 = solver.iterate(args.warmup)
    stream = torch.cuda.ExternalStream(solver.stream, device=device)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        ev0.record(stream)
        s1 = solver.iterate(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, device)
    iters = s1["iteration"] - s0["iteration"]
    evals = sum(1 for it in range(s0["iteration"], s1["iteration"]) if is_eval(it))
    launches = 2 * iters + 2 * evals

    # ---- time to KKT <= 1e-4 from the zero start ----
    ttk = None
    if not args.no_ttk:
        solver.reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = solver.finish()
        e1.record(stream)
        e1.synchronize()
        ci = out.iteration_stats[-1].convergence_information[0]
        ttk = {"seconds": e0.elapsed_time(e1) / 1000.0, "iterations": out.iteration_count,
               "termination": out.termination_string,
               "relative_l2_primal_residual": ci.relative_l2_primal_residual,
               "relative_l2_dual_residual": ci.relative_l2_dual_residual,
               "relative_optimality_gap": ci.relative_optimality_gap,
               "primal_objective": ci.primal_objective,
               "solver_time_sec": out.iteration_stats[-1].cumulative_time_sec}
    solver.close()
    del solver

    # ---- per-launch kernel times (CUDA events around every launch) ----
    tsolver = pdot.Solver(params, device_problem=dev_problem, device=local, use_cuda_graph=False,
                          time_kernels=True)
    t0 = tsolver.iterate(args.warmup)
    t1 = tsolver.iterate(args.steps)
    tsolver.close()
    del tsolver
    passes = t1["primal_passes"] - t0["primal_passes"]
    fresh = t1["primal_passes_fresh_average"] - t0["primal_passes_fresh_average"]
    k1_launches = t1["timed_primal_passes"] - t0["timed_primal_passes"]
    k1_ms = t1["primal_pass_ms"] - t0["primal_pass_ms"]
    region_kernel_ms = (t1["primal_pass_ms"] + t1["dual_step_ms"] + t1["evaluation_ms"]
                        - t0["primal_pass_ms"] - t0["dual_step_ms"] - t0["evaluation_ms"])
    # algorithmic bytes: read C, X, Xavg and write X, Xavg (8 B each in FP64);
    # a pass that starts a new average does not read Xavg
    alg_bytes = N * (40.0 * (passes - fresh) + 32.0 * fresh)
    per_launch_bytes = alg_bytes / max(passes, 1)
    k1_avg_s = k1_ms / 1000.0 / max(k1_launches, 1)
    achieved = per_launch_bytes / k1_avg_s / 1e9
    peak, peak_kind = read_peak()
    traffic = (K1_DRAM_BYTES_PER_ENTRY * N) if K1_DRAM_BYTES_PER_ENTRY else None

    # ---- end to end through the public API, host buffers ----
    e2e = None
    if not args.no_e2e:
        C_host = torch.empty((n, m), dtype=torch.float64, pin_memory=True)
        C_host.copy_(Ct)
        prob = pdot.OptimalTransportProblem(C_host.numpy().T, a_h, b_h)
        eparams = pdot.default_parameters(TOL, iteration_limit=args.steps)
        torch.cuda.synchronize()
        barrier(world)
        w0 = time.perf_counter()
        out = pdot.optimize(eparams, prob, device=local)
        torch.cuda.synchronize()
        w1 = time.perf_counter()
        e_sec = max_over_ranks(w1 - w0, world, device)
        vec_bytes = 8 * (m + n)
        e2e = {"value": world * out.iteration_count / e_sec, "unit": UNIT,
               "h2d_bytes_per_step": (8 * N + vec_bytes) / max(out.iteration_count, 1),
               "d2h_bytes_per_step": (8 * N + vec_bytes) / max(out.iteration_count, 1),
               "iterations_per_call": out.iteration_count, "seconds_per_call": e_sec,
               "note": "one pdot.optimize call: H2D of C, a, b from pinned memory, the solve, "
                       "D2H of the returned plan and duals; bytes amortised per iteration"}
        del C_host

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline(xs, ys, a_h, b_h, m, n, steps=20)

    value = world * iters / (ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": iters,
        "warmup": args.warmup, "ms_per_step": ms / max(iters, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"PDHG-OT m={m} n={n} gauss-mixture(8, sigma 0.05) sq-euclid/max FP64 drop-in, "
                               f"reference script parameters, tol {TOL}",
                   "l2": "inputs larger than L2 (C, X, Xavg = 7.2 GB), no flush",
                   "parallelism": "replicas" if world > 1 else "1 GPU",
                   "cuda_graph_chunks": True},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "k1_primal (fused primal pass)",
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "avg_launch_ms": k1_avg_s * 1000.0, "launches_timed": k1_launches,
                     "share_of_kernel_time": k1_ms / region_kernel_ms if region_kernel_ms > 0 else None},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "time_to_kkt": ttk,
    }
    return line


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    else:
        line = run_ours(args, world, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
