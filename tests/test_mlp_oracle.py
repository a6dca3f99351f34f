"""The learned warm start on the CPU: the network oracle's backward pass is
the gradient of its forward pass, and the symmetry augmentation of solved
instances gives exact solutions of the images."""
import numpy as np
import pytest

import mlp_oracle as mo
import oracle
import pdot
from pdot import learned


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    I, H, O, B = 6, 5, 4, 3
    P = H * I + H + H * H + H + O * H + O
    theta = rng.standard_normal(P) * 0.5
    x = rng.standard_normal((B, I))
    t = rng.standard_normal((B, O))
    loss, g = mo.loss_and_gradients(theta, x, t, I, H, O, round_bf16=False)
    fd = np.zeros(P)
    h = 1e-6
    for k in range(P):
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd[k] = (mo.loss_and_gradients(tp, x, t, I, H, O, False)[0] - mo.loss_and_gradients(tm, x, t, I, H, O, False)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-5, atol=1e-8)


def test_bf16_rounding_is_nearest_even():
    # BF16 keeps 8 significant bits: neighbours of 1 are 1 and 1 + 2^-7
    vals = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-9, 1.0 + 2**-9, 1.0 + 3 * 2**-8, 3.14159], dtype=np.float32)
    got = mo.bf16(vals)
    # ties (1 + 2^-8, 1 + 3 * 2^-8) go to the even neighbour
    np.testing.assert_array_equal(got[:5], [1.0, 1.0, 1.0 + 2**-7, 1.0, 1.0 + 2**-6])
    assert got[5] == 3.140625


def test_grid_symmetries_preserve_the_cost():
    side = 5
    pts = learned.grid_points(side).astype(np.float64)
    D = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    maps = learned.grid_symmetries(side)
    assert len({tuple(p) for p in maps}) == 8
    for p in maps:
        np.testing.assert_array_equal(D[np.ix_(p, p)], D)


def test_augmented_duals_solve_the_images():
    """Solve a small grid instance with the oracle; each of its 16 images has
    the image duals as an optimal dual solution (same objective, feasible)."""
    side = 6
    rng = np.random.default_rng(3)
    a = pdot.instances.grid_histogram(rng, side)
    b = pdot.instances.grid_histogram(rng, side)
    C = pdot.instances.grid_cost(side)
    out = oracle.optimize(pdot.default_parameters(1e-8), pdot.OptimalTransportProblem(C, a, b))
    u, v = learned.canonical_duals(out.dual_source_solution, out.dual_target_solution)
    obj = a @ u + b @ v
    imgs = learned.augment(a, b, u, v, side)
    assert len(imgs) == 16
    for aa, bb, uu, vv in imgs:
        assert aa @ uu + bb @ vv == pytest.approx(obj, rel=1e-12)
        assert np.min(C - uu[:, None] - vv[None, :]) >= np.min(C - u[:, None] - v[None, :]) - 1e-15


def test_symmetrized_prediction_maps_images_back(monkeypatch):
    """With an equivariant stand-in for the network (its 'duals' are the
    input histograms), the prediction averaged over the 16 images returns
    exactly that equivariant answer for the original instance."""
    rng = np.random.default_rng(5)
    a = rng.dirichlet(np.ones(learned.BINS), size=3)
    b = rng.dirichlet(np.ones(learned.BINS), size=3)
    monkeypatch.setattr(learned, "forward_rows", lambda mlp, hist: hist.astype(np.float32))
    model = learned.WarmStartModel(np.zeros(1, np.float32), 0.0, 1.0)
    u, v = learned.predict(None, model, a, b, symmetrize=True)
    np.testing.assert_allclose(u, a.astype(np.float32), rtol=1e-6)
    np.testing.assert_allclose(v, b.astype(np.float32), rtol=1e-6)


def test_packaged_model_loads():
    model = learned.WarmStartModel.load(learned.MODEL_PATH)
    I, H, O = 2 * learned.BINS, model.hidden_dim, 2 * learned.BINS
    assert model.parameters.size == H * I + H + H * H + H + O * H + O
    assert np.all(np.isfinite(model.parameters))
    assert 0 < model.target_scale < 1
