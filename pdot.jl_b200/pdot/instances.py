"""Seeded synthetic OT instances with the shapes and distributions of the
benchmark workloads (the reference ships no dataset; these stand in for it).

    uniform_sqeuclid   points i.i.d. U[0,1]^d, C_ij = ||x_i - y_j||^2 / max(C),
                       marginals U(0.1, 1) normalised to sum 1
    gauss_mixture      points from a 2-D mixture of 8 isotropic Gaussians
                       (sigma = 0.05, means U[0,1]^2, equal weights, not clipped),
                       squared-Euclidean cost / max, marginals U(0.1, 1) normalised
    l1_dirichlet       points U[0,1]^2, C = ||x - y||_1 / max, marginals Dirichlet(1)
    grid_histograms    32x32 grid histograms, mixtures of 1-5 isotropic Gaussians
                       (sigma in [1, 6] px) plus a 1e-4 floor, normalised;
                       C = squared grid distance / max
"""
from __future__ import annotations

import numpy as np

from .api import OptimalTransportProblem


def _marginal(rng, k):
    w = rng.uniform(0.1, 1.0, size=k)
    return w / w.sum()


def sqeuclid_cost(xs: np.ndarray, ys: np.ndarray) -> np.ndarray:
    """C_ij = ||x_i - y_j||^2 / max(C), as an m x n Fortran-ordered float64 matrix."""
    xs = np.asarray(xs, dtype=np.float64)
    ys = np.asarray(ys, dtype=np.float64)
    C = np.zeros((xs.shape[0], ys.shape[0]), dtype=np.float64, order="F")
    for k in range(xs.shape[1]):
        C += (xs[:, k : k + 1] - ys[None, :, k]) ** 2
    mx = C.max()
    if mx > 0:
        C /= mx
    return C


def uniform_sqeuclid(m: int, n: int, dim: int = 2, seed: int = 0) -> OptimalTransportProblem:
    rng = np.random.default_rng(seed)
    xs = rng.uniform(0.0, 1.0, size=(m, dim))
    ys = rng.uniform(0.0, 1.0, size=(n, dim))
    return OptimalTransportProblem(sqeuclid_cost(xs, ys), _marginal(rng, m), _marginal(rng, n))


def gauss_mixture_points(rng, k: int, components: int = 8, sigma: float = 0.05):
    means = rng.uniform(0.0, 1.0, size=(components, 2))
    lab = rng.integers(0, components, size=k)
    return means[lab] + sigma * rng.standard_normal(size=(k, 2))


def gauss_mixture_instance(m: int, n: int, seed: int = 0):
    """(xs, ys, a, b) of the mixed-precision benchmark instance: points from a
    2-D mixture of 8 Gaussians (sigma 0.05, means U[0,1]^2), marginals
    U(0.1, 1) normalised; C = ||x - y||^2 / max, built from the points."""
    rng = np.random.default_rng(seed)
    xs = gauss_mixture_points(rng, m)
    ys = gauss_mixture_points(rng, n)
    a = rng.uniform(0.1, 1.0, size=m)
    b = rng.uniform(0.1, 1.0, size=n)
    return xs, ys, a / a.sum(), b / b.sum()


def gauss_mixture(m: int, n: int, seed: int = 0) -> OptimalTransportProblem:
    rng = np.random.default_rng(seed)
    xs = gauss_mixture_points(rng, m)
    ys = gauss_mixture_points(rng, n)
    return OptimalTransportProblem(sqeuclid_cost(xs, ys), _marginal(rng, m), _marginal(rng, n))


def l1_dirichlet(m: int, n: int, seed: int = 0) -> OptimalTransportProblem:
    rng = np.random.default_rng(seed)
    xs = rng.uniform(0.0, 1.0, size=(m, 2))
    ys = rng.uniform(0.0, 1.0, size=(n, 2))
    C = np.abs(xs[:, None, 0] - ys[None, :, 0]) + np.abs(xs[:, None, 1] - ys[None, :, 1])
    C = np.asfortranarray(C / C.max())
    return OptimalTransportProblem(C, rng.dirichlet(np.ones(m)), rng.dirichlet(np.ones(n)))


def grid_histogram(rng, side: int = 32) -> np.ndarray:
    yy, xx = np.mgrid[0:side, 0:side].astype(np.float64)
    h = np.zeros((side, side))
    for _ in range(int(rng.integers(1, 6))):
        cx, cy = rng.uniform(0, side, size=2)
        s = rng.uniform(1.0, 6.0)
        h += rng.uniform(0.2, 1.0) * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * s * s))
    h = h.ravel() + 1e-4
    return h / h.sum()


def grid_cost(side: int = 32) -> np.ndarray:
    yy, xx = np.mgrid[0:side, 0:side]
    pts = np.stack([xx.ravel(), yy.ravel()], axis=1).astype(np.float64)
    return sqeuclid_cost(pts, pts)


def grid_histograms(seed: int = 0, side: int = 32) -> OptimalTransportProblem:
    rng = np.random.default_rng(seed)
    return OptimalTransportProblem(grid_cost(side), grid_histogram(rng, side), grid_histogram(rng, side))


def batched_l1(count: int = 512, lo: int = 64, hi: int = 2048, seed: int = 0):
    """`count` instances with m, n each log-uniform in [lo, hi], points U[0,1]^2,
    marginals Dirichlet(1). Returns (problems without cost matrices, points):
    the L1 cost |x - y|_1 / max is computed from the points."""
    rng = np.random.default_rng(seed)
    probs, pts = [], []
    for _ in range(count):
        m = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        n = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        xs = rng.uniform(0.0, 1.0, size=(m, 2))
        ys = rng.uniform(0.0, 1.0, size=(n, 2))
        probs.append(OptimalTransportProblem(None, rng.dirichlet(np.ones(m)), rng.dirichlet(np.ones(n))))
        pts.append((xs, ys))
    return probs, pts


def l1_cost(xs: np.ndarray, ys: np.ndarray) -> np.ndarray:
    """C_ij = ||x_i - y_j||_1 / max(C), Fortran-ordered float64."""
    C = np.zeros((xs.shape[0], ys.shape[0]), order="F")
    for k in range(xs.shape[1]):
        C += np.abs(xs[:, k : k + 1] - ys[None, :, k])
    mx = C.max()
    if mx > 0:
        C /= mx
    return C
