"""The learned warm start's network on the GPU against its CPU oracle
(oracle/mlp_oracle.py): the tcgen05 products, the forward pass, the
gradients, AdamW, and a plan recovered from warm duals.

Tolerances: both sides round the same operands to BF16; the GPU accumulates
in FP32 and the oracle in FP64, which moves a handful of BF16 roundings of
intermediate activations by one unit (2^-8 relative). The outputs and the
gradients therefore agree to ~1e-4 in relative 2-norm; the tests allow 1e-3
(outputs) and 1e-2 (gradients)."""
import numpy as np
import pytest

import mlp_oracle as mo
import oracle
import pdot
from pdot import instances, learned

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def _net_and_inputs(I, H, O, batch, seed=0, max_batch=None):
    torch = _torch()
    net = learned.MLP(I, H, O, max_batch=max_batch or batch, seed=seed)
    rng = np.random.default_rng(seed)
    hist = rng.dirichlet(np.ones(I // 2), size=(batch, 2)).reshape(batch, I)
    target = rng.standard_normal((batch, O)).astype(np.float32)
    h_dev = torch.from_numpy(hist).cuda()
    t_dev = torch.from_numpy(target).cuda()
    torch.cuda.synchronize()
    return net, hist, target, h_dev, t_dev


@pytest.mark.parametrize("batch", [128, 100, 256])
def test_forward_matches_oracle(cuda, batch):
    torch = _torch()
    I, H, O = 256, 128, 384
    net, hist, _, h_dev, _ = _net_and_inputs(I, H, O, batch, seed=1, max_batch=256)
    theta = net.get_parameters()
    y = torch.zeros((batch, O), dtype=torch.float32, device="cuda")
    net.set_input(h_dev.data_ptr(), batch)
    net.forward(y.data_ptr())
    x = mo.features(hist, learned.FEATURE_SHIFT, learned.FEATURE_SCALE)
    ref, _ = mo.forward(theta, x, I, H, O)
    got = y.cpu().numpy()
    assert np.all(np.isfinite(got))
    assert _rel(got, ref) < 1e-3


def test_gradients_match_oracle_full_size(cuda):
    """2048 -> 1024 -> 1024 -> 2048 at batch 256: every parameter block."""
    I, H, O, B = 2048, 1024, 2048, 256
    net, hist, target, h_dev, t_dev = _net_and_inputs(I, H, O, B, seed=2)
    theta = net.get_parameters()
    net.set_input(h_dev.data_ptr(), B)
    net.forward()
    loss = net.backward(t_dev.data_ptr())
    g = net.gradients()
    x = mo.features(hist, learned.FEATURE_SHIFT, learned.FEATURE_SCALE)
    ref_loss, ref_g = mo.loss_and_gradients(theta, x, target, I, H, O)
    assert loss == pytest.approx(ref_loss, rel=1e-4)
    sizes = [H * I, H, H * H, H, O * H, O]
    off = 0
    for name, s in zip(["W1", "b1", "W2", "b2", "W3", "b3"], sizes):
        assert _rel(g[off:off + s], ref_g[off:off + s]) < 1e-2, name
        off += s


def test_adamw_step_matches_oracle(cuda):
    I, H, O, B = 256, 128, 256, 128
    net, hist, target, h_dev, t_dev = _net_and_inputs(I, H, O, B, seed=3)
    theta = net.get_parameters().astype(np.float64)
    net.set_input(h_dev.data_ptr(), B)
    net.forward()
    net.backward(t_dev.data_ptr())
    g = net.gradients().astype(np.float64)
    net.adamw(1e-3, 0.9, 0.999, 1e-8, 0.01)
    got = net.get_parameters()
    m = np.zeros_like(theta)
    v = np.zeros_like(theta)
    mo.adamw(theta, g, m, v, 1, 1e-3, 0.9, 0.999, 1e-8, 0.01, I, H, O)
    np.testing.assert_allclose(got, theta, rtol=1e-5, atol=1e-8)


def test_training_reduces_the_loss(cuda):
    I, H, O, B = 256, 256, 256, 128
    net, hist, _, h_dev, _ = _net_and_inputs(I, H, O, B, seed=4)
    # a learnable target: a fixed smooth function of the input
    x = mo.features(hist, learned.FEATURE_SHIFT, learned.FEATURE_SCALE)
    target = np.tanh(x[:, :O] - x[:, O - 1::-1][:, :O]).astype(np.float32)
    torch = _torch()
    t_dev = torch.from_numpy(target).cuda()
    torch.cuda.synchronize()
    net.set_input(h_dev.data_ptr(), B)
    first = net.train_step(t_dev.data_ptr(), 1e-3, 0.0, True)
    for _ in range(200):
        last = net.train_step(t_dev.data_ptr(), 1e-3, 0.0, True)
    assert last < 0.2 * first


def test_saved_model_reproduces_the_outputs(cuda, tmp_path):
    """The saved form keeps the BF16 weights the kernels use and the FP32
    biases, so a network loaded from it computes the same outputs bit for bit."""
    torch = _torch()
    I, H, O, B = 2048, 1024, 2048, 128
    net, hist, _, h_dev, _ = _net_and_inputs(I, H, O, B, seed=5)
    model = learned.WarmStartModel(net.get_parameters(), 0.1, 0.05, hidden_dim=H)
    path = str(tmp_path / "model.npz")
    model.save(path)
    loaded = learned.WarmStartModel.load(path)
    assert loaded.target_mean == 0.1 and loaded.target_scale == 0.05
    net2 = learned.MLP(I, H, O, max_batch=B, seed=99)
    net2.set_parameters(loaded.parameters)
    y1 = torch.zeros((B, O), dtype=torch.float32, device="cuda")
    y2 = torch.zeros((B, O), dtype=torch.float32, device="cuda")
    net.set_input(h_dev.data_ptr(), B)
    net.forward(y1.data_ptr())
    net2.set_input(h_dev.data_ptr(), B)
    net2.forward(y2.data_ptr())
    assert torch.equal(y1, y2)


def test_recovered_plan_matches_oracle(cuda):
    prob = instances.uniform_sqeuclid(70, 50, seed=6)
    params = pdot.default_parameters(1e-4)
    cold = pdot.optimize(params, prob)
    rng = np.random.default_rng(0)
    u0 = cold.dual_source_solution + 0.01 * rng.standard_normal(70)
    v0 = cold.dual_target_solution + 0.01 * rng.standard_normal(50)
    eps, rounds = 1e-2, 20
    X, _, _ = oracle.warm_plan(prob.cost_matrix, prob.source_distribution, prob.target_distribution, u0, v0, eps,
                               rounds)
    res = np.sqrt(np.sum((prob.source_distribution - X.sum(1)) ** 2) + np.sum((prob.target_distribution - X.sum(0)) ** 2))
    pobj = float(np.vdot(prob.cost_matrix, X))
    p0 = pdot.default_parameters(1e-4, iteration_limit=0)
    for precision, cost in [("f64", None), ("f32", "f32")]:
        out = pdot.optimize(p0, prob, precision=precision, cost=cost, warm_start=(u0, v0), recover_plan=(eps, rounds))
        c0 = out.iteration_stats[0].convergence_information[0]
        assert c0.primal_objective == pytest.approx(pobj, rel=1e-3)
        assert c0.l2_primal_residual == pytest.approx(res, rel=1e-2, abs=1e-9)
        np.testing.assert_allclose(out.primal_solution, X, rtol=1e-3, atol=1e-9)
    # the batched solver, with the coordinate cost
    probs, pts = instances.batched_l1(3, 40, 90, seed=7)
    cold_b, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts)
    warm = [(o.dual_source_solution, o.dual_target_solution) for o in cold_b]
    outs, _ = pdot.optimize_batched(p0, probs, cost="l1", points=pts, warm_starts=warm, recover_plan=(eps, rounds))
    for k, o in enumerate(outs):
        C = instances.l1_cost(*pts[k])
        Xk, _, _ = oracle.warm_plan(C, probs[k].source_distribution, probs[k].target_distribution, warm[k][0],
                                    warm[k][1], eps, rounds)
        np.testing.assert_allclose(o.primal_solution, Xk, rtol=2e-3, atol=1e-8)
