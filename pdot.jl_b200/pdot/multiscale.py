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

import numpy as np

from . import _abi, api


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


def _device_points(p, device: int):
    import torch

    t = p if isinstance(p, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(p, dtype=np.float32))
    return t.to(device=torch.device("cuda", device), dtype=torch.float32).contiguous()


def max_sq_distance(xs, ys, *, device: int = 0) -> float:
    """max_ij ||x_i - y_j||^2 over the two point sets, on the GPU
    (pdot_points_max_sqdist; coordinates rounded to FP32 as the solver reads
    them, distances in FP64)."""
    import torch

    lib = _abi.load()
    x, y = _device_points(xs, device), _device_points(ys, device)
    out = torch.zeros(1, dtype=torch.float64, device=x.device)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    _abi.check(lib, lib.pdot_points_max_sqdist(x.shape[0], y.shape[0], x.shape[1], x.data_ptr(), y.data_ptr(),
                                               out.data_ptr(), stream), "pdot_points_max_sqdist")
    return float(out.item())


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


def c_transform(points, centres: np.ndarray, dual: np.ndarray, scale: float, *, device: int = 0) -> np.ndarray:
    """min_J (scale * ||p - c_J||^2 - dual_J) for every point p, on the GPU
    (pdot_points_c_transform)."""
    import torch

    lib = _abi.load()
    p = _device_points(points, device)
    c = torch.from_numpy(np.ascontiguousarray(centres, dtype=np.float64)).to(p.device)
    d = torch.from_numpy(np.ascontiguousarray(dual, dtype=np.float64)).to(p.device)
    out = torch.empty(p.shape[0], dtype=torch.float64, device=p.device)
    stream = torch.cuda.current_stream(p.device).cuda_stream
    _abi.check(lib, lib.pdot_points_c_transform(p.shape[0], c.shape[0], p.shape[1], p.data_ptr(), c.data_ptr(),
                                                d.data_ptr(), float(scale), out.data_ptr(), stream),
               "pdot_points_c_transform")
    return out.cpu().numpy()


def _grid_prediction(xs, ys, a, b, starter, scale: float, floor: float):
    """The network's duals of the binned problem on its 32 x 32 grid over the
    common bounding square of the two point sets (empty cells get `floor` mass
    before the histograms are renormalised, as the training histograms carry a
    small floor), rescaled to the cost scale * ||c_I - c_J||^2 between cell
    centres: (centres, non-empty source cells, non-empty target cells, source
    duals, target duals)."""
    from .learned import SIDE

    G = SIDE
    lo, side = bounding_square(xs, ys)
    A, _ = bin_masses(xs, a, lo, side, G)
    B, _ = bin_masses(ys, b, lo, side, G)
    ha = (A + floor) / (A + floor).sum()
    hb = (B + floor) / (B + floor).sum()
    U, V = starter.predict(ha[None, :], hb[None, :])
    # the network's cost is the squared grid distance divided by its maximum, 2 * 31^2
    kappa = scale * (side / G) ** 2 * 2.0 * (G - 1) ** 2
    return cell_centres(lo, side, G), np.nonzero(A > 0)[0], np.nonzero(B > 0)[0], kappa * U[0], kappa * V[0]


def learned_to_fine_duals(xs, ys, a, b, starter, *, scale: float | None = None, floor: float = 1e-6):
    """Warm-start duals (u, v) for the fine problem from the learned network
    instead of a coarse solve: the network predicts the duals of the problem
    binned on its 32 x 32 grid (_grid_prediction), and they are extended to
    every point by the c-transform over the non-empty cells. `starter` is a
    learned.WarmStarter."""
    xs, ys = np.asarray(xs, dtype=np.float64), np.asarray(ys, dtype=np.float64)
    s = scale if scale is not None else 1.0 / max_sq_distance(xs, ys, device=starter.device)
    cent, ia, ib, U, V = _grid_prediction(xs, ys, a, b, starter, s, floor)
    u = c_transform(xs, cent[ib], V[ib], s, device=starter.device)
    v = c_transform(ys, cent[ia], U[ia], s, device=starter.device)
    return u, v, {"cells": [int(ia.size), int(ib.size)]}


def learned_coarse_to_fine_duals(xs, ys, a, b, starter, *, G: int = 128, tol: float = 1e-4,
                                 iteration_limit: int = 200_000, floor: float = 1e-6,
                                 recover_plan=(3e-4, 100), warm_restart: str = "zero"):
    """Warm-start duals (u, v) for the fine problem through a learned coarse
    solve: the network's 32 x 32 duals (_grid_prediction), extended by the
    c-transform to the non-empty cells of a G x G binning, warm-start the G x G
    coarse solve (a plan recovered from them, the zero point's restart record
    as the network's grid warm starts use); its duals are then extended to
    every point, as coarse_to_fine_duals does. Returns (u, v, facts)."""
    from .solve import default_parameters

    xs, ys = np.asarray(xs, dtype=np.float64), np.asarray(ys, dtype=np.float64)
    dev = starter.device
    s = 1.0 / max_sq_distance(xs, ys, device=dev)
    Cc, A, B, ca, cb = coarse_problem(xs, ys, a, b, G, s)
    cent, ia, ib, U, V = _grid_prediction(xs, ys, a, b, starter, s, floor)
    u0 = c_transform(ca, cent[ib], V[ib], s, device=dev)
    v0 = c_transform(cb, cent[ia], U[ia], s, device=dev)
    params = default_parameters(tol, iteration_limit=iteration_limit)
    out = api.optimize(params, api.OptimalTransportProblem(Cc, A, B), device=dev, warm_start=(u0, v0),
                       recover_plan=recover_plan, warm_restart=warm_restart)
    u = c_transform(xs, cb, out.dual_target_solution, s, device=dev)
    v = c_transform(ys, ca, out.dual_source_solution, s, device=dev)
    info = {"cells": [int(A.size), int(B.size)], "coarse_iterations": out.iteration_count,
            "coarse_termination": out.termination_string,
            "coarse_seconds": out.iteration_stats[-1].cumulative_time_sec}
    return u, v, info


def coarse_to_fine_duals(xs, ys, a, b, *, G: int = 128, tol: float = 1e-4, iteration_limit: int = 200_000,
                         scale: float | None = None, device: int = 0, precision: str = "f64"):
    """Warm-start duals (u, v) for the fine problem, and facts about the coarse
    solve. The binning and the coarse cost are host work on at most G^2 cells;
    the normaliser, the coarse solve and the c-transforms run on the GPU.
    `precision` is the coarse solve's plan precision ("f64", or "f32" with an
    FP32 copy of the coarse cost)."""
    xs, ys = np.asarray(xs, dtype=np.float64), np.asarray(ys, dtype=np.float64)
    s = scale if scale is not None else 1.0 / max_sq_distance(xs, ys, device=device)
    Cc, A, B, ca, cb = coarse_problem(xs, ys, a, b, G, s)
    from .solve import default_parameters

    params = default_parameters(tol, iteration_limit=iteration_limit)
    out = api.optimize(params, api.OptimalTransportProblem(Cc, A, B), device=device, precision=precision)
    u = c_transform(xs, cb, out.dual_target_solution, s, device=device)
    v = c_transform(ys, ca, out.dual_source_solution, s, device=device)
    info = {"cells": [int(A.size), int(B.size)], "coarse_iterations": out.iteration_count,
            "coarse_termination": out.termination_string,
            "coarse_seconds": out.iteration_stats[-1].cumulative_time_sec}
    return u, v, info
