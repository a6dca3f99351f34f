"""A coarse-to-fine warm start for point-cloud instances with the squared
Euclidean cost (an addition; the reference has none).

    1. bin the source and target points on a G x G grid over their common
       bounding square; the masses of a cell add up
    2. solve the binned problem (empty cells dropped) with the cell centres'
       cost, scaled as the fine cost is (1 / max fine distance^2)
    3. extend the coarse duals to every point by the exact semi-discrete
       c-transform: u_i = min_J (s ||x_i - c_J||^2 - V_J), v_j likewise
    4. solve the fine problem from (u, v) with a plan recovered from them
       (pdot.optimize(..., warm_start=(u, v), recover_plan=(eps, rounds)))

On the mixed-precision benchmark instance (20000 x 15000, points from a
mixture of 8 Gaussians) this warm start does not reduce the iterations of the
fine solve; `python -m pdot.multiscale` measures it against the cold start.
"""
from __future__ import annotations

import json
import time

import numpy as np

from . import api, instances


def bounding_square(xs: np.ndarray, ys: np.ndarray):
    pts = np.concatenate([xs, ys])
    lo = pts.min(axis=0)
    side = float((pts.max(axis=0) - lo).max()) * (1.0 + 1e-9)
    return lo, side if side > 0 else 1.0


def bin_masses(points: np.ndarray, masses: np.ndarray, lo, side: float, G: int):
    """Masses of the G x G cells (index row * G + column) and the cell of each point."""
    cell = np.minimum(((points - lo) / side * G).astype(np.int64), G - 1)
    idx = cell[:, 1] * G + cell[:, 0]
    out = np.zeros(G * G)
    np.add.at(out, idx, masses)
    return out, idx


def cell_centres(lo, side: float, G: int) -> np.ndarray:
    gy, gx = np.mgrid[0:G, 0:G]
    return lo + (np.stack([gx.ravel(), gy.ravel()], axis=1) + 0.5) * (side / G)


def max_sq_distance(xs: np.ndarray, ys: np.ndarray, chunk: int = 4096) -> float:
    mx = 0.0
    for k in range(0, xs.shape[0], chunk):
        d = ((xs[k:k + chunk, None, :] - ys[None, :, :]) ** 2).sum(-1)
        mx = max(mx, float(d.max()))
    return mx


def coarse_problem(xs, ys, a, b, G: int, scale: float):
    """The binned problem: (cost, source masses, target masses, source centres,
    target centres) over the non-empty cells, cost = scale * ||c_I - c_J||^2."""
    lo, side = bounding_square(xs, ys)
    A, _ = bin_masses(xs, a, lo, side, G)
    B, _ = bin_masses(ys, b, lo, side, G)
    cent = cell_centres(lo, side, G)
    ia, ib = np.nonzero(A > 0)[0], np.nonzero(B > 0)[0]
    ca, cb = cent[ia], cent[ib]
    Cc = scale * ((ca[:, None, :] - cb[None, :, :]) ** 2).sum(-1)
    return np.asfortranarray(Cc), A[ia], B[ib], ca, cb


def c_transform(points: np.ndarray, centres: np.ndarray, dual: np.ndarray, scale: float,
                chunk: int = 4096) -> np.ndarray:
    """min_J (scale * ||p - c_J||^2 - dual_J) for every point p."""
    out = np.empty(points.shape[0])
    for k in range(0, points.shape[0], chunk):
        d = scale * ((points[k:k + chunk, None, :] - centres[None, :, :]) ** 2).sum(-1) - dual[None, :]
        out[k:k + chunk] = d.min(axis=1)
    return out


def learned_to_fine_duals(xs, ys, a, b, starter, *, scale: float | None = None, floor: float = 1e-6):
    """Warm-start duals (u, v) for the fine problem from the learned network
    instead of a coarse solve: both point sets are binned on the network's
    32 x 32 grid over their common bounding square, the network predicts the
    grid problem's duals (its cost is the squared grid distance divided by its
    maximum, 2 * 31^2), they are rescaled to the fine cost between cell centres,
    scale * (side / 32)^2 * |g_I - g_J|^2, and extended to every point by the
    c-transform over the non-empty cells. `starter` is a learned.WarmStarter;
    empty cells get `floor` mass before the histograms are renormalised, as the
    training histograms carry a small floor."""
    from .learned import SIDE

    G = SIDE
    s = scale if scale is not None else 1.0 / max_sq_distance(xs, ys)
    lo, side = bounding_square(xs, ys)
    A, _ = bin_masses(xs, a, lo, side, G)
    B, _ = bin_masses(ys, b, lo, side, G)
    ha = (A + floor) / (A + floor).sum()
    hb = (B + floor) / (B + floor).sum()
    U, V = starter.predict(ha[None, :], hb[None, :])
    kappa = s * (side / G) ** 2 * 2.0 * (G - 1) ** 2
    cent = cell_centres(lo, side, G)
    ia, ib = np.nonzero(A > 0)[0], np.nonzero(B > 0)[0]
    u = c_transform(xs, cent[ib], kappa * V[0][ib], s)
    v = c_transform(ys, cent[ia], kappa * U[0][ia], s)
    return u, v, {"cells": [int(ia.size), int(ib.size)]}


def coarse_to_fine_duals(xs, ys, a, b, *, G: int = 32, tol: float = 1e-4, iteration_limit: int = 100_000,
                         scale: float | None = None, device: int = 0):
    """Warm-start duals (u, v) for the fine problem, and facts about the coarse solve."""
    s = scale if scale is not None else 1.0 / max_sq_distance(xs, ys)
    Cc, A, B, ca, cb = coarse_problem(xs, ys, a, b, G, s)
    from .solve import default_parameters

    params = default_parameters(tol, iteration_limit=iteration_limit)
    out = api.optimize(params, api.OptimalTransportProblem(Cc, A, B), device=device)
    u = c_transform(xs, cb, out.dual_target_solution, s)
    v = c_transform(ys, ca, out.dual_source_solution, s)
    info = {"cells": [int(A.size), int(B.size)], "coarse_iterations": out.iteration_count,
            "coarse_termination": out.termination_string,
            "coarse_seconds": out.iteration_stats[-1].cumulative_time_sec}
    return u, v, info


def main(argv=None):
    import argparse

    from .solve import default_parameters

    ap = argparse.ArgumentParser(prog="python -m pdot.multiscale")
    ap.add_argument("--m", type=int, default=20000)
    ap.add_argument("--n", type=int, default=15000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--grids", type=int, nargs="+", default=[32, 64])
    ap.add_argument("--eps", type=float, nargs="+", default=[1e-4, 3e-4, 1e-3])
    ap.add_argument("--rounds", type=int, nargs="+", default=[30, 100])
    ap.add_argument("--iteration-limit", type=int, default=40_000)
    ap.add_argument("--out")
    args = ap.parse_args(argv)
    xs, ys, a, b = instances.gauss_mixture_instance(args.m, args.n, args.seed)
    xs32, ys32 = xs.astype(np.float32), ys.astype(np.float32)
    prob = api.OptimalTransportProblem(None, a, b)
    params = default_parameters(1e-4, iteration_limit=args.iteration_limit)
    kw = {"precision": "f32", "cost": "sqeuclid", "points": (xs32, ys32)}
    cold = api.optimize(params, prob, **kw)
    rows = [{"start": "cold", "iterations": cold.iteration_count,
             "seconds": cold.iteration_stats[-1].cumulative_time_sec}]
    print(json.dumps(rows[-1]), flush=True)
    scale = 1.0 / max_sq_distance(xs32.astype(np.float64), ys32.astype(np.float64))
    for G in args.grids:
        t0 = time.perf_counter()
        u, v, info = coarse_to_fine_duals(xs32.astype(np.float64), ys32.astype(np.float64), a, b, G=G, scale=scale)
        prep = time.perf_counter() - t0
        for eps in args.eps:
            for rounds in args.rounds:
                w = api.optimize(params, prob, warm_start=(u, v), recover_plan=(eps, rounds), **kw)
                rows.append({"start": f"coarse-to-fine G={G}", "eps": eps, "rounds": rounds,
                             "iterations": w.iteration_count, "termination": w.termination_string,
                             "seconds": w.iteration_stats[-1].cumulative_time_sec, "prep_seconds": prep, **info})
                print(json.dumps(rows[-1]), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(rows, f, indent=1)


if __name__ == "__main__":
    main()
