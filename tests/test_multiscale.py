"""The coarse-to-fine warm start's host steps (pdot/multiscale.py): binning and
the coarse problem, against direct computation on small point sets (the device
passes, the normaliser and the c-transform, are checked in
tests/test_gpu_multiscale.py)."""
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
    s = 1.0 / float((((xs[:, None, :] - ys[None, :, :]) ** 2).sum(-1)).max())
    C, A, B, ca, cb = multiscale.coarse_problem(xs, ys, a, b, 6, s)
    assert np.all(A > 0) and np.all(B > 0)
    assert A.sum() == pytest.approx(1.0) and B.sum() == pytest.approx(1.0)
    assert C.shape == (A.size, B.size)
    np.testing.assert_allclose(C[1, 2], s * np.sum((ca[1] - cb[2]) ** 2), rtol=1e-14)
