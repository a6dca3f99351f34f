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


def test_tight_duals_are_feasible_and_c_conjugate():
    side = 6
    rng = np.random.default_rng(11)
    C = pdot.instances.grid_cost(side)
    u = rng.normal(0, 0.1, side * side)
    v = rng.normal(0, 0.1, side * side)
    v[3] = -50.0  # a loose dual, as PDHG leaves them on rows of tiny mass
    ut, vt = learned.tight_duals(u, v, C)
    G = C - ut[:, None] - vt[None, :]
    assert G.min() >= -1e-12                                   # feasible
    np.testing.assert_allclose(ut, (C - vt[None, :]).min(axis=1), atol=1e-12)  # u = v^c
    np.testing.assert_allclose(vt, (C - ut[:, None]).min(axis=0), atol=1e-12)  # v = u^c
    assert abs(ut.mean() - vt.mean()) < 1e-12                  # canonical shift
    assert np.abs(np.concatenate([ut, vt])).max() <= C.max() + 1.0


def test_dataset_expands_each_optimal_instance_into_16_images():
    data = {"seeds": np.array([5, 6, 7]), "reasons": np.array([1, 3, 1]),
            "u": np.zeros((3, learned.BINS)), "v": np.zeros((3, learned.BINS)),
            "iterations": np.array([1, 2, 3]), "seconds": 0.0}
    hist, duals = learned.dataset(data)
    assert hist.shape == (32, 2 * learned.BINS) and duals.shape == (32, 2 * learned.BINS)  # instance 6 dropped
    a, b = learned.grid_pair(5)
    np.testing.assert_array_equal(hist[0], np.concatenate([a, b]))
    np.testing.assert_array_equal(hist[1], np.concatenate([b, a]))


def test_model_save_load_roundtrip(tmp_path):
    I, H, O = 2 * learned.BINS, 128, 2 * learned.BINS
    P = H * I + H + H * H + H + O * H + O
    rng = np.random.default_rng(0)
    theta = rng.standard_normal(P).astype(np.float32) * 0.02
    model = learned.WarmStartModel(theta, -0.03, 0.11, hidden_dim=H)
    path = str(tmp_path / "m.npz")
    model.save(path)
    back = learned.WarmStartModel.load(path)
    assert back.hidden_dim == H and back.target_mean == -0.03 and back.target_scale == 0.11
    sizes = [H * I, H, H * H, H, O * H, O]
    off = 0
    for k, s in enumerate(sizes):
        seg, got = theta[off:off + s], back.parameters[off:off + s]
        if k % 2 == 0:  # weights: their BF16 values
            np.testing.assert_array_equal(got, mo.bf16(seg).astype(np.float32))
        else:           # biases: FP32 as they were
            np.testing.assert_array_equal(got, seg)
        off += s


def test_summarize_counts_race_results():
    res = {"cold_iterations": [100, 200, 300, 400], "warm_iterations": [50, 250, 100, 400],
           "cold_seconds": 2.0, "warm_seconds": 1.0, "predict_seconds": 0.1,
           "cold_reasons": [1, 1, 1, 1], "warm_reasons": [1, 1, 1, 3],
           "dual_rel_error": [0.1, 0.2, 0.3, 0.4], "warm_work_iterations": [100, 400, 200, 800],
           "race_winner_warm": [True, False, True, False]}
    s = learned.summarize(res)
    assert s["cold_mean_iterations"] == 250 and s["warm_mean_iterations"] == 200
    assert s["warm_better_fraction"] == 0.5 and s["race_warm_wins"] == 2
    assert s["warm_optimal"] == 3 and s["warm_work_mean_iterations"] == 375
