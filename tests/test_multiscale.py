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


def test_grid_prediction_feeds_floored_histograms_and_rescales_the_duals():
    """The learned warm starts' host step: both point sets binned on the
    network's 32 x 32 grid over their common square, `floor` added to every
    cell and each histogram renormalised before the network sees it; the
    network's duals (of the grid cost |g_I - g_J|^2 / (2 * 31^2)) come back in
    the fine cost's units, scale * (side / 32)^2 * |g_I - g_J|^2."""
    from pdot import learned

    xs, ys, a, b = instances.gauss_mixture_instance(500, 400, seed=5)
    seen = {}

    class FakeStarter:
        def predict(self, ha, hb):
            seen["ha"], seen["hb"] = ha, hb
            return np.arange(1024.0)[None, :], -np.arange(1024.0)[None, :]

    floor, scale = 1e-6, 0.37
    cent, ia, ib, U, V = multiscale._grid_prediction(xs, ys, a, b, FakeStarter(), scale, floor)
    G = learned.SIDE
    lo, side = multiscale.bounding_square(xs, ys)
    A, _ = multiscale.bin_masses(xs, a, lo, side, G)
    B, _ = multiscale.bin_masses(ys, b, lo, side, G)
    np.testing.assert_allclose(seen["ha"][0], (A + floor) / (A + floor).sum(), rtol=1e-15)
    np.testing.assert_allclose(seen["hb"][0], (B + floor) / (B + floor).sum(), rtol=1e-15)
    assert np.array_equal(ia, np.nonzero(A > 0)[0]) and np.array_equal(ib, np.nonzero(B > 0)[0])
    kappa = scale * (side / G) ** 2 * 2.0 * (G - 1) ** 2
    np.testing.assert_allclose(U, kappa * np.arange(1024.0), rtol=1e-15)
    np.testing.assert_allclose(V, -kappa * np.arange(1024.0), rtol=1e-15)
    np.testing.assert_allclose(cent, multiscale.cell_centres(lo, side, G))
    # the cost units: one grid step between adjacent cell centres costs scale * (side / G)^2
    d2 = ((cent[1] - cent[0]) ** 2).sum()
    assert scale * d2 == pytest.approx(kappa / (2.0 * (G - 1) ** 2), rel=1e-12)
