"""The coarse-to-fine warm start's host steps (pdot/multiscale.py): binning,
the coarse problem and the semi-discrete c-transform, against direct
computation on small point sets."""
import numpy as np
import pytest

from pdot import instances, multiscale


def test_binning_conserves_mass_and_places_points_in_their_cells():
    xs, ys, a, b = instances.gauss_mixture_instance(300, 200, seed=3)
    lo, side = multiscale.bounding_square(xs, ys)
    G = 8
    A, idx = multiscale.bin_masses(xs, a, lo, side, G)
    assert A.sum() == pytest.approx(1.0, abs=1e-12)
    cent = multiscale.cell_centres(lo, side, G)
    h = side / G
    assert np.all(np.abs(xs - cent[idx]) <= h / 2 + 1e-9)


def test_coarse_problem_keeps_nonempty_cells_and_scaled_cost():
    xs, ys, a, b = instances.gauss_mixture_instance(120, 90, seed=4)
    s = 1.0 / multiscale.max_sq_distance(xs, ys)
    C, A, B, ca, cb = multiscale.coarse_problem(xs, ys, a, b, 6, s)
    assert np.all(A > 0) and np.all(B > 0)
    assert A.sum() == pytest.approx(1.0) and B.sum() == pytest.approx(1.0)
    assert C.shape == (A.size, B.size)
    np.testing.assert_allclose(C[1, 2], s * np.sum((ca[1] - cb[2]) ** 2), rtol=1e-14)


def test_c_transform_matches_brute_force():
    rng = np.random.default_rng(0)
    pts = rng.uniform(0, 1, (50, 2))
    cen = rng.uniform(0, 1, (17, 2))
    dual = rng.normal(0, 0.1, 17)
    got = multiscale.c_transform(pts, cen, dual, 0.7, chunk=8)
    ref = np.array([min(0.7 * np.sum((p - c) ** 2) - d for c, d in zip(cen, dual)) for p in pts])
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-15)


def test_max_sq_distance():
    xs = np.array([[0.0, 0.0], [1.0, 0.0]])
    ys = np.array([[0.0, 2.0], [3.0, 0.0]])
    assert multiscale.max_sq_distance(xs, ys, chunk=1) == 9.0
