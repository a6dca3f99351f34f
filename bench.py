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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "pdot.jl_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "time-to-KKT≤1e-4 and PDHG iters/s at n=20000 (plain vs MP+warm-start); % HBM roofline"
UNIT = "iters/s"
M_ROWS, N_COLS, SEED, TOL = 20000, 15000, 0, 1e-4
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes over algorithmic bytes of one full-size fused primal pass, from a
# one-pass ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) on B200:
# 9.578 GB measured for 9.600 GB algorithmic (FP64), 3.554 GB for 3.600 GB
# (FP32 plan with the coordinate cost).
K1_TRAFFIC_RATIO = {"f64": 9578004224 / 9.6e9, "sqeuclid": 3554418944 / 3.6e9}
C1_SIZE, C2_SIZE = 1000, 10000  # the square configurations: U[0,1]^2 and U[0,1]^3 points


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
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-solver line (512 instances)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start line (64 instances)")
    ap.add_argument("--batched-only", action="store_true", help="run only the batched-solver line and print it")
    ap.add_argument("--no-mp", action="store_true", help="skip the mixed-precision variants")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the m=n=1000 and m=n=10000 configuration blocks (c1, c2)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling runs)")
    ap.add_argument("--precision", choices=["f64", "f32"], default="f64",
                    help="plan precision of the primary workload (f64: the drop-in)")
    ap.add_argument("--cost", choices=["f64", "f32", "bf16", "sqeuclid"], default=None,
                    help="cost source of the primary workload (default: f64, or f32 with --precision f32)")
    return ap.parse_args()


def host_instance(m, n, seed):
    """Points and marginals (host, seeded): pdot.instances.gauss_mixture_instance."""
    from pdot import instances

    return instances.gauss_mixture_instance(m, n, seed)


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


def full_problem_host(xs, ys, a, b):
    """The full FP64 instance on the host (C column-major, 2.4 GB at
    20000 x 15000): the same entries the device cost builder writes."""
    from pdot import api, instances

    return api.OptimalTransportProblem(instances.sqeuclid_cost(xs, ys), a, b)


def time_oracle_steps(prob, steps, warmup):
    """Full-size PDHG iterations of the FP64 oracle on all host cores: `warmup`
    untimed iterations, then `steps` timed ones in the same state."""
    import oracle
    import pdot

    cores = os.cpu_count() or 1
    sec = oracle.time_steps(pdot.default_parameters(TOL), prob, steps, cores, warmup=warmup)
    return sec, cores


def cpu_baseline(prob, m, n, steps, warmup):
    sec, cores = time_oracle_steps(prob, steps, warmup)
    return {"value": steps / float(sec.sum()), "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} full-size PDHG iterations (take_step!) of the FP64 oracle on the {m}x{n} "
                      f"instance after {warmup} untimed ones in the same state; no extrapolation",
            "seconds": float(sec.sum()), "step_seconds": [round(float(x), 4) for x in sec]}
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
    reference is Julia and no Julia toolchain is installed): each step is one
    full-size PDHG iteration of the FP64 oracle on the benchmark instance."""
    if rank != 0:
        return None
    xs, ys, a, b = host_instance(args.m, args.n, SEED)
    prob = full_problem_host(xs, ys, a, b)
    sec, cores = time_oracle_steps(prob, args.steps, args.warmup)
    total = float(sec.sum())
    value = args.steps / total
    sample = (f"each step one full-size PDHG iteration (take_step!) of the FP64 oracle on the "
              f"{args.m}x{args.n} instance, after {args.warmup} untimed iterations in the same state")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / max(args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"PDHG-OT m={args.m} n={args.n} gauss-mixture(8, sigma 0.05) sq-euclid/max, "
                               f"FP64 drop-in, reference script parameters, tol {TOL}",
                   "implementation": "FP64 CPU restatement of the reference algorithm (OpenMP), "
                                     "the reference itself is Julia and cannot run here"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                         "seconds": total, "step_seconds": [round(float(x), 4) for x in sec]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    return line


def fp64_kkt_device(Ct, a, b, X_t, u, v):
    """Relative L2 KKT error of a solution on the FP64 problem, on the device.
    Ct is the (n, m) row-major view of C; X_t the plan in the same layout."""
    import torch

    pres = torch.sqrt(((a - X_t.sum(dim=0)) ** 2).sum() + ((b - X_t.sum(dim=1)) ** 2).sum()).item()
    G = Ct - u[None, :] - v[:, None]
    dres = torch.linalg.vector_norm(torch.clamp(G, max=0.0)).item()
    del G
    pobj = float((Ct * X_t).sum().item())
    dobj = float((a @ u + b @ v).item())
    rp = pres / (1 + math.sqrt(float((a @ a + b @ b).item())))
    rd = dres / (1 + torch.linalg.vector_norm(Ct).item())
    rg = abs(pobj - dobj) / (1 + abs(pobj) + abs(dobj))
    return {"primal_objective": pobj, "relative_l2_primal_residual": rp, "relative_l2_dual_residual": rd,
            "relative_optimality_gap": rg, "relative_kkt": max(rp, rd, rg)}


def time_iterations(solver, warmup, steps, device):
    import torch

    s0 = solver.iterate(warmup)
    stream = torch.cuda.ExternalStream(solver.stream, device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s1 = solver.iterate(steps)
    e1.record(stream)
    e1.synchronize()
    return s1["iteration"] - s0["iteration"], e0.elapsed_time(e1), s0, s1


def run_mixed(args, params, m, n, Ct, a, b, xs_d, ys_d, device, local, fp64_obj):
    """Mixed-precision variants: FP32 plan with the cost from FP32 or BF16
    storage or computed from FP32 coordinates (16 B per entry)."""
    import torch

    import pdot

    N = m * n
    out = {}
    dev_problem = (m, n, Ct.data_ptr(), a.data_ptr(), b.data_ptr())
    pts = (xs_d.data_ptr(), ys_d.data_ptr(), xs_d.shape[1])
    bytes_per_entry = {"sqeuclid": 16.0, "f32": 20.0, "bf16": 18.0}
    for cost in ("sqeuclid", "f32", "bf16"):
        kw = {"points": pts} if cost == "sqeuclid" else {}
        prob = (m, n, 0, a.data_ptr(), b.data_ptr()) if cost == "sqeuclid" else dev_problem
        solver = pdot.Solver(params, device_problem=prob, device=local, precision="f32", cost=cost, **kw)
        iters, ms, _, _ = time_iterations(solver, args.warmup, args.steps, device)
        entry = {"iters_per_sec": iters / (ms / 1000.0), "ms_per_iter": ms / max(iters, 1)}
        if cost == "sqeuclid" and not args.no_ttk:
            solver.reset()
            stream = torch.cuda.ExternalStream(solver.stream, device=device)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            res = solver.finish()
            e1.record(stream)
            e1.synchronize()
            X_t = torch.from_numpy(np.ascontiguousarray(res.primal_solution.T)).to(device)
            u = torch.from_numpy(res.dual_source_solution).to(device)
            v = torch.from_numpy(res.dual_target_solution).to(device)
            k64 = fp64_kkt_device(Ct, a, b, X_t, u, v)
            del X_t
            entry["time_to_kkt"] = {"seconds": e0.elapsed_time(e1) / 1000.0, "iterations": res.iteration_count,
                                    "termination": res.termination_string,
                                    "internal_relative_gap":
                                        res.iteration_stats[-1].convergence_information[0].relative_optimality_gap,
                                    "fp64_evaluation": k64,
                                    "objective_vs_fp64_solve": (k64["primal_objective"] - fp64_obj) / fp64_obj
                                    if fp64_obj else None}
        solver.close()
        if cost == "sqeuclid":
            ts = pdot.Solver(params, device_problem=prob, device=local, use_cuda_graph=False, time_kernels=True,
                             precision="f32", cost=cost, **kw)
            t0 = ts.iterate(args.warmup)
            t1 = ts.iterate(min(args.steps, 200))
            ts.close()
            passes = t1["primal_passes"] - t0["primal_passes"]
            fresh = t1["primal_passes_fresh_average"] - t0["primal_passes_fresh_average"]
            k1_ms = t1["primal_pass_ms"] - t0["primal_pass_ms"]
            launches = t1["timed_primal_passes"] - t0["timed_primal_passes"]
            alg = N * (16.0 * (passes - fresh) + 12.0 * fresh) / max(passes, 1)
            avg_s = k1_ms / 1000.0 / max(launches, 1)
            peak, _ = read_peak()
            ratio = K1_TRAFFIC_RATIO["sqeuclid"] if (m, n) == (M_ROWS, N_COLS) else None
            entry["roofline"] = {"achieved": alg / avg_s / 1e9, "peak": peak, "unit": "GB/s",
                                 "frac": alg / avg_s / 1e9 / peak, "algorithmic_bytes_per_launch": alg,
                                 "avg_launch_ms": avg_s * 1000.0, "traffic": alg * ratio if ratio else None}
        entry["bytes_per_entry"] = bytes_per_entry[cost]
        out[cost] = entry
    return out


def solve_timed(params, dev_problem, local, device, **variant):
    """A full solve from the zero start on a resident problem, timed with CUDA
    events on the solver's stream; returns (seconds, output)."""
    import torch

    import pdot

    solver = pdot.Solver(params, device_problem=dev_problem, device=local, **variant)
    stream = torch.cuda.ExternalStream(solver.stream, device=device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = solver.finish()
    e1.record(stream)
    e1.synchronize()
    solver.close()
    return e0.elapsed_time(e1) / 1000.0, out


def ttk_record(sec, out):
    ci = out.iteration_stats[-1].convergence_information[0]
    return {"seconds": sec, "iterations": out.iteration_count, "termination": out.termination_string,
            "iters_per_sec": out.iteration_count / sec if sec > 0 else None,
            "relative_l2_primal_residual": ci.relative_l2_primal_residual,
            "relative_l2_dual_residual": ci.relative_l2_dual_residual,
            "relative_optimality_gap": ci.relative_optimality_gap, "primal_objective": ci.primal_objective}


def square_instance(k, dim, seed, device):
    """The square configurations (pdot.instances.uniform_sqeuclid): points
    U[0,1]^dim, C = ||x - y||^2 / max built on the device, marginals
    U(0.1, 1) normalised. Returns the host problem's vectors and device tensors."""
    import torch

    rng = np.random.default_rng(seed)
    xs = rng.uniform(0.0, 1.0, size=(k, dim))
    ys = rng.uniform(0.0, 1.0, size=(k, dim))
    a = rng.uniform(0.1, 1.0, size=k)
    b = rng.uniform(0.1, 1.0, size=k)
    a, b = a / a.sum(), b / b.sum()
    Ct = device_cost(xs, ys, device)
    return xs, ys, a, b, Ct, torch.from_numpy(a).to(device), torch.from_numpy(b).to(device)


def run_c1(args, device, local, cpu_too):
    """m = n = 1000 (points U[0,1]^2), FP64, tol 1e-4: a full solve on the GPU
    (resident problem, device time) and, beside it, the FP64 oracle's full solve
    on the host cores (wall time)."""
    import oracle
    import pdot
    from pdot import api, instances

    xs, ys, a, b, Ct, ad, bd = square_instance(C1_SIZE, 2, 0, device)
    params = pdot.default_parameters(TOL)
    dev_problem = (C1_SIZE, C1_SIZE, Ct.data_ptr(), ad.data_ptr(), bd.data_ptr())
    solve_timed(params, dev_problem, local, device)  # first-call set-up outside the timing
    sec, out = solve_timed(params, dev_problem, local, device)
    res = {"workload": "m=n=1000, U[0,1]^2 points, sq-euclid/max, FP64 drop-in, tol 1e-4",
           "gpu": ttk_record(sec, out)}
    if cpu_too:
        prob = api.OptimalTransportProblem(instances.sqeuclid_cost(xs, ys), a, b)
        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        r = oracle.optimize(params, prob, num_threads=cores)
        wall = time.perf_counter() - t0
        rec = ttk_record(wall, r)
        rec.update({"cores": cores, "kind": "port", "timing": "wall time of the oracle's whole optimize call"})
        res["cpu_oracle"] = rec
        res["gpu_speedup_over_cpu"] = wall / sec
    return res


def run_c2(args, device, local):
    """m = n = 10000 (points U[0,1]^3), the FP64 drop-in: iterations/s with the
    fused pass's roofline, and time to relative KKT 1e-4 and 1e-6."""
    import pdot

    k = C2_SIZE
    _, _, _, _, Ct, ad, bd = square_instance(k, 3, 0, device)
    dev_problem = (k, k, Ct.data_ptr(), ad.data_ptr(), bd.data_ptr())
    params = pdot.default_parameters(TOL)
    solver = pdot.Solver(params, device_problem=dev_problem, device=local)
    iters, ms, _, _ = time_iterations(solver, args.warmup, args.steps, device)
    solver.close()
    ts = pdot.Solver(params, device_problem=dev_problem, device=local, use_cuda_graph=False, time_kernels=True)
    t0 = ts.iterate(args.warmup)
    t1 = ts.iterate(args.steps)
    ts.close()
    passes = t1["primal_passes"] - t0["primal_passes"]
    fresh = t1["primal_passes_fresh_average"] - t0["primal_passes_fresh_average"]
    launches = t1["timed_primal_passes"] - t0["timed_primal_passes"]
    alg = k * k * (40.0 * (passes - fresh) + 32.0 * fresh) / max(passes, 1)
    avg_s = (t1["primal_pass_ms"] - t0["primal_pass_ms"]) / 1000.0 / max(launches, 1)
    peak, _ = read_peak()
    res = {"workload": "m=n=10000, U[0,1]^3 points, sq-euclid/max, FP64 drop-in",
           "iters_per_sec": iters / (ms / 1000.0), "ms_per_iter": ms / max(iters, 1),
           "roofline": {"kernel": "k1_primal", "achieved": alg / avg_s / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": alg / avg_s / 1e9 / peak, "algorithmic_bytes_per_launch": alg,
                        "avg_launch_ms": avg_s * 1000.0}}
    for tol in (1e-4, 1e-6):
        sec, out = solve_timed(pdot.default_parameters(tol), dev_problem, local, device)
        res[f"tol_{tol:.0e}"] = ttk_record(sec, out)
    return res


WARM_GRID, WARM_EPS, WARM_ROUNDS = 128, 3e-4, 100  # coarse-to-fine warm start of the 20000 x 15000 solve


def run_warm_mixed(args, params, m, n, xs, ys, a_h, b_h, Ct, a, b, xs_d, ys_d, device, local, fp64_ttk,
                   learned=False):
    """The mixed-precision solve (FP32 plan, cost from FP32 coordinates) from
    the coarse-to-fine warm start: points binned on a 128 x 128 grid, the binned
    problem solved, its duals extended to every point by the c-transform, a
    plan recovered from them by 100 balancing rounds (eps 3e-4), then PDHG to
    relative KKT 1e-4. With `learned`, the coarse solve itself starts from the
    packaged network's 32 x 32 prediction (multiscale.learned_coarse_to_fine_duals;
    loading the network is outside the region). One wall-clock region covers
    all of it, from the host points to the plan back on the host; the answer is
    judged on the FP64 problem."""
    import torch

    import pdot
    from pdot import multiscale

    starter = None
    if learned:
        from pdot import learned as learned_mod

        starter = learned_mod.WarmStarter(device=local)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if learned:
        u, v, info = multiscale.learned_coarse_to_fine_duals(xs, ys, a_h, b_h, starter, G=WARM_GRID)
    else:
        u, v, info = multiscale.coarse_to_fine_duals(xs, ys, a_h, b_h, G=WARM_GRID, device=local)
    t1 = time.perf_counter()
    ud = torch.from_numpy(u).to(device)
    vd = torch.from_numpy(v).to(device)
    solver = pdot.Solver(params, device_problem=(m, n, 0, a.data_ptr(), b.data_ptr()), device=local,
                         precision="f32", cost="sqeuclid", points=(xs_d.data_ptr(), ys_d.data_ptr(), xs_d.shape[1]),
                         warm_start=(ud.data_ptr(), vd.data_ptr()), recover_plan=(WARM_EPS, WARM_ROUNDS))
    res = solver.finish()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    solver.close()
    X_t = torch.from_numpy(np.ascontiguousarray(res.primal_solution.T)).to(device)
    k64 = fp64_kkt_device(Ct, a, b, X_t, torch.from_numpy(res.dual_source_solution).to(device),
                          torch.from_numpy(res.dual_target_solution).to(device))
    del X_t
    total = t2 - t0
    kind = "learned coarse-to-fine warm start (the network's 32 x 32 duals start the " if learned else \
        "coarse-to-fine warm start ("
    return {"workload": f"FP32 plan, cost from FP32 coordinates, {kind}grid {WARM_GRID} coarse solve, "
                        f"plan recovered with eps {WARM_EPS}, {WARM_ROUNDS} rounds), tol {TOL}",
            "seconds": total, "prep_seconds": t1 - t0, "coarse": info, "iterations": res.iteration_count,
            "termination": res.termination_string, "fp64_evaluation": k64,
            "speedup_over_fp64_time_to_kkt": (fp64_ttk / total) if fp64_ttk else None,
            "timing": "wall clock from the host points to the plan on the host (binning, coarse solve, "
                      "c-transforms, solver set-up and plan recovery, the solve, the copy back)"}


def run_batched(args, device):
    """The batched solver on 512 uneven instances (m, n log-uniform in
    [64, 2048], points U[0,1]^2, L1 cost / max, Dirichlet(1) marginals, FP32
    plan), all to relative KKT 1e-4 in one lockstep solve. Effective bandwidth:
    16 B per entry per iteration (plan and average read and written; the cost
    comes from the coordinates) summed over the iterations each instance ran,
    divided by the device time of the whole solve."""
    import pdot
    from pdot import instances

    probs, pts = instances.batched_l1(512, 64, 2048, seed=SEED)
    params = pdot.default_parameters(TOL, iteration_limit=200_000)
    # the autotuner picks the launch configuration from the first 256 iterations
    best, timings = pdot.tune_batched(params, probs, cost="l1", points=pts, device=device.index)
    outs, sec = pdot.optimize_batched(params, probs, cost="l1", points=pts, device=device.index,
                                      return_primal=False, **best)
    its = np.array([o.iteration_count for o in outs], dtype=float)
    mn = np.array([p.source_distribution.size * p.target_distribution.size for p in probs], dtype=float)
    alg = float(np.sum(its * mn) * 16.0)
    peak, _ = read_peak()
    opt = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL
    return {"workload": "512 instances, m,n log-uniform [64,2048], L1 cost from U[0,1]^2 points, Dirichlet(1), "
                        "FP32 plan, tol 1e-4",
            "seconds": sec, "instances_per_sec": len(probs) / sec, "optimal": int(sum(o.termination_reason == opt
                                                                                        for o in outs)),
            "mean_iterations": float(its.mean()), "max_iterations": float(its.max()),
            "total_entries": float(mn.sum()), "effective_gbs": alg / sec / 1e9, "peak": peak,
            "effective_frac": alg / sec / 1e9 / peak, "configuration": best,
            "autotune_256_iterations": [{**c, "seconds": t} for c, t in timings]}


def run_learned(args, device):
    """The learned warm start on 64 grid instances outside its training,
    validation and evaluation seeds: one batched cold solve, and one batched
    solve of the network's warm starts each raced against a cold start of the
    same instance (a cold start is the fallback). Both to relative KKT 1e-4."""
    import time

    import pdot
    from pdot import learned

    seeds = list(range(9_200_000, 9_200_064))
    params = pdot.default_parameters(TOL, iteration_limit=400_000)
    pairs = [learned.grid_pair(s) for s in seeds]
    A = np.asarray([p[0] for p in pairs])
    B = np.asarray([p[1] for p in pairs])
    cold, cold_sec = learned.solve_grid_batch(seeds, params, device=device.index)
    ws = learned.WarmStarter(device=device.index, max_batch=128)
    ws.predict(A[:1], B[:1])  # first-call setup outside the timing
    t0 = time.perf_counter()
    u, v = ws.predict(A, B)
    pred_sec = time.perf_counter() - t0
    warm, warm_sec, won = ws.solve(A, B, params, race=True)
    ci = np.array([o.iteration_count for o in cold], dtype=float)
    wi = np.array([o.iteration_count for o in warm], dtype=float)
    opt = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL
    return {"workload": "64 held-out 32x32 grid instances (C5 distribution), sq-euclid grid cost, FP32 plan, tol 1e-4",
            "cold_seconds": cold_sec, "learned_seconds": warm_sec + pred_sec, "network_seconds": pred_sec,
            "speedup": cold_sec / (warm_sec + pred_sec),
            "cold_mean_iterations": float(ci.mean()), "learned_mean_iterations": float(wi.mean()),
            "cold_median_iterations": float(np.median(ci)), "learned_median_iterations": float(np.median(wi)),
            "warm_won": int(sum(won)), "all_optimal": bool(all(o.termination_reason == opt for o in cold + warm))}


def run_ours(args, world, rank, local):
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
    params = pdot.default_parameters(TOL)
    params.termination_criteria.time_sec_limit = 300.0
    precision = args.precision
    cost = args.cost or ("f64" if precision == "f64" else "f32")
    variant = {"precision": precision, "cost": cost}
    xs_d = torch.from_numpy(xs.astype(np.float32)).to(device)
    ys_d = torch.from_numpy(ys.astype(np.float32)).to(device)
    if cost == "sqeuclid":
        dev_problem = (m, n, 0, a.data_ptr(), b.data_ptr())
        variant["points"] = (xs_d.data_ptr(), ys_d.data_ptr(), xs.shape[1])
    else:
        dev_problem = (m, n, Ct.data_ptr(), a.data_ptr(), b.data_ptr())
    # algorithmic bytes per entry of the fused pass: read cost, plan, average;
    # write plan, average (the average is not read after a reset)
    xb = 8.0 if precision == "f64" else 4.0
    cb = {"f64": 8.0, "f32": 4.0, "bf16": 2.0, "sqeuclid": 0.0}[cost]
    full_bytes, fresh_bytes = cb + 4 * xb, cb + 3 * xb

    # ---- timed region: K iterations, problem resident, CUDA graphs ----
    solver = pdot.Solver(params, device_problem=dev_problem, device=local, **variant)
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
                          time_kernels=True, **variant)
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
    alg_bytes = N * (full_bytes * (passes - fresh) + fresh_bytes * fresh)
    per_launch_bytes = alg_bytes / max(passes, 1)
    k1_avg_s = k1_ms / 1000.0 / max(k1_launches, 1)
    achieved = per_launch_bytes / k1_avg_s / 1e9
    peak, peak_kind = read_peak()
    ratio = K1_TRAFFIC_RATIO.get("f64" if precision == "f64" else cost) if (m, n) == (M_ROWS, N_COLS) else None
    traffic = per_launch_bytes * ratio if ratio else None

    # ---- end to end through the public API, host buffers ----
    e2e = None
    if not args.no_e2e:
        C_host = torch.empty((n, m), dtype=torch.float64, pin_memory=True)
        C_host.copy_(Ct)
        ekw = {"precision": precision, "cost": cost}
        if cost == "sqeuclid":
            prob = pdot.OptimalTransportProblem(None, a_h, b_h)
            ekw["points"] = (xs.astype(np.float32), ys.astype(np.float32))
        else:
            prob = pdot.OptimalTransportProblem(C_host.numpy().T, a_h, b_h)
        eparams = pdot.default_parameters(TOL, iteration_limit=args.steps)
        # the caller's output arrays, page-locked like the input and reused by every call
        X_pin = torch.empty((n, m), dtype=torch.float64, pin_memory=True)
        u_pin = torch.empty(m, dtype=torch.float64, pin_memory=True)
        v_pin = torch.empty(n, dtype=torch.float64, pin_memory=True)
        out_arrays = (X_pin.numpy().T, u_pin.numpy(), v_pin.numpy())
        # one untimed call first, as the warm-up steps of the primary region
        pdot.optimize(pdot.default_parameters(TOL, iteration_limit=max(args.warmup, 1)), prob, device=local,
                      out=out_arrays, **ekw)

        def timed_calls(**kw):
            # three timed calls, the median reported (each allocates on the device, copies in, solves,
            # copies out, frees)
            calls = []
            res = None
            for _ in range(3):
                torch.cuda.synchronize()
                barrier(world)
                w0 = time.perf_counter()
                res = pdot.optimize(eparams, prob, device=local, **ekw, **kw)
                torch.cuda.synchronize()
                w1 = time.perf_counter()
                calls.append(max_over_ranks(w1 - w0, world, device))
            return res, calls

        out, calls = timed_calls(out=out_arrays)
        e_sec = statistics.median(calls)
        fresh, fresh_calls = timed_calls()
        assert np.array_equal(fresh.primal_solution, out.primal_solution)
        vec_bytes = 8 * (m + n)
        h2d = (8 * (m + n) * xs.shape[1] // 2 if cost == "sqeuclid" else 8 * N) + vec_bytes
        e2e = {"value": world * out.iteration_count / e_sec, "unit": UNIT,
               "h2d_bytes_per_step": h2d / max(out.iteration_count, 1),
               "d2h_bytes_per_step": (8 * N + vec_bytes) / max(out.iteration_count, 1),
               "iterations_per_call": out.iteration_count, "seconds_per_call": e_sec,
               "seconds_of_the_three_calls": calls,
               "note": "the median of three pdot.optimize calls after one untimed call: H2D of C, a, b "
                       "from pinned memory, the solve, D2H of the plan and duals into the caller's pinned "
                       "output arrays (out=); bytes amortised per iteration",
               "fresh_host_arrays": {
                   "value": world * fresh.iteration_count / statistics.median(fresh_calls),
                   "seconds_of_the_three_calls": fresh_calls,
                   "note": "the same calls returning fresh numpy arrays (allocated and first touched per call)"}}
        del C_host, X_pin, u_pin, v_pin, out_arrays

    mixed = None
    if not args.no_mp and precision == "f64":
        fp64_obj = ttk["primal_objective"] if ttk else None
        mixed = run_mixed(args, params, m, n, Ct, a, b, xs_d, ys_d, device, local, fp64_obj)
        if not args.no_ttk:
            mixed["sqeuclid"]["warm_start"] = run_warm_mixed(args, params, m, n, xs, ys, a_h, b_h, Ct, a, b, xs_d,
                                                             ys_d, device, local, ttk["seconds"] if ttk else None)
            mixed["sqeuclid"]["learned_warm_start"] = run_warm_mixed(
                args, params, m, n, xs, ys, a_h, b_h, Ct, a, b, xs_d, ys_d, device, local,
                ttk["seconds"] if ttk else None, learned=True)

    batched = run_batched(args, device) if not args.no_batched else None
    learned_ws = run_learned(args, device) if not args.no_learned else None

    c1 = run_c1(args, device, local, cpu_too=(rank == 0 and world == 1)) if not args.no_configs else None
    c2 = run_c2(args, device, local) if not args.no_configs else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(full_problem_host(xs, ys, a_h, b_h), m, n, steps=5, warmup=2)

    value = world * iters / (ms / 1000.0)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": iters,
        "warmup": args.warmup, "ms_per_step": ms / max(iters, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": precision, "data": "synthetic",
        "config": {"workload": f"PDHG-OT m={m} n={n} gauss-mixture(8, sigma 0.05) sq-euclid/max, "
                               + ("FP64 drop-in" if precision == "f64" else f"FP32 plan, {cost} cost")
                               + f", reference script parameters, tol {TOL}",
                   "l2": "inputs larger than L2 (C, X, Xavg = 7.2 GB), no flush",
                   "parallelism": "replicas" if world > 1 else "1 GPU",
                   "cuda_graph_chunks": True},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one full-size launch "
                                       "on B200: measured/algorithmic ratio times this region's algorithmic "
                                       "bytes per launch" if traffic else None,
                     "kernel": "k1_primal (fused primal pass)",
                     "algorithmic_bytes_per_entry": full_bytes,
                     "algorithmic_bytes_per_launch": per_launch_bytes,
                     "avg_launch_ms": k1_avg_s * 1000.0, "launches_timed": k1_launches,
                     "share_of_kernel_time": k1_ms / region_kernel_ms if region_kernel_ms > 0 else None},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "time_to_kkt": ttk,
        "mixed_precision": mixed, "batched": batched, "learned_warm_start": learned_ws,
        "c1": c1, "c2": c2,
    }
    return line


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    elif args.batched_only:
        import torch

        line = run_batched(args, torch.device("cuda", local))
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
