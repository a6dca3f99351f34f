"""Warm starts on the GPU: initial duals and an initial plan (this
implementation's addition; the reference always starts at zero,
src/solver_gpu.jl:428-441).

A warm start sets u, v, X, the sums r = X 1 and c = X^T 1, and the stored
gradient C - u - v. The oracle's warm start does the same, so the early
evaluation records of the two agree as the cold ones do (the per-eval scalars
within ~1e-9 relative)."""
import numpy as np
import pytest

import oracle
import pdot
from pdot import instances

pytestmark = pytest.mark.gpu

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


def _perturbed(cold, rng, scale):
    u, v = cold.dual_source_solution, cold.dual_target_solution
    return (u + scale * np.std(u) * rng.standard_normal(u.shape),
            v + scale * np.std(v) * rng.standard_normal(v.shape),
            np.maximum(cold.primal_solution * (1 + scale * rng.standard_normal(cold.primal_solution.shape)), 0))


def test_exact_warm_start_stops_at_the_first_evaluation(cuda):
    prob = instances.uniform_sqeuclid(120, 90, seed=2)
    params = pdot.default_parameters(1e-4)
    cold = pdot.optimize(params, prob)
    assert cold.termination_reason == OPTIMAL
    warm = pdot.optimize(params, prob, warm_start=(cold.dual_source_solution, cold.dual_target_solution,
                                                   cold.primal_solution))
    assert warm.termination_reason == OPTIMAL
    assert warm.iteration_count == 0
    np.testing.assert_array_equal(warm.primal_solution, cold.primal_solution)


@pytest.mark.parametrize("m,n", [(64, 48), (257, 130)])
def test_warm_start_matches_the_oracle_early(cuda, m, n):
    """Records of iterations 1-10 and the forced one at 129: past the
    artificial restarts of the first iterations, the adaptive restart test
    compares against the last restart point, which a warm start sets to its
    own start point (its residuals, gap and norms), on both sides."""
    prob = instances.uniform_sqeuclid(m, n, seed=m)
    params = pdot.default_parameters(1e-4)
    cold = oracle.optimize(params, prob)
    u0, v0, X0 = _perturbed(cold, np.random.default_rng(1), 0.05)
    p128 = pdot.default_parameters(1e-4, iteration_limit=128)
    g = pdot.optimize(p128, prob, warm_start=(u0, v0, X0))
    o = oracle.optimize_warm(p128, prob, u0, v0, X0)
    assert len(g.iteration_stats) == len(o.iteration_stats)
    for a, b in zip(g.iteration_stats, o.iteration_stats):
        assert a.restart_used == b.restart_used
        assert a.step_size == pytest.approx(b.step_size, rel=1e-9)
        assert a.primal_weight == pytest.approx(b.primal_weight, rel=1e-9)
        ca, cb = a.convergence_information[0], b.convergence_information[0]
        for f in ("primal_objective", "dual_objective", "l2_primal_residual", "l2_dual_residual"):
            assert getattr(ca, f) == pytest.approx(getattr(cb, f), rel=1e-9, abs=1e-14), f


def test_warm_start_with_fp32_plan(cuda):
    prob = instances.uniform_sqeuclid(200, 150, seed=4)
    params = pdot.default_parameters(1e-4)
    cold = pdot.optimize(params, prob)
    u0, v0, X0 = _perturbed(cold, np.random.default_rng(2), 0.02)
    w = pdot.optimize(params, prob, precision="f32", cost="f32", warm_start=(u0, v0, X0))
    assert w.termination_reason == OPTIMAL
    c0 = w.iteration_stats[0].convergence_information[0]
    X32 = X0.astype(np.float32).astype(np.float64)
    res = np.sqrt(np.sum((prob.source_distribution - X32.sum(1)) ** 2)
                  + np.sum((prob.target_distribution - X32.sum(0)) ** 2))
    assert c0.l2_primal_residual == pytest.approx(res, rel=1e-9, abs=1e-15)


def test_warm_plan_requires_duals(cuda):
    prob = instances.uniform_sqeuclid(20, 20, seed=1)
    opts, keep = pdot.api._options(0, True, warm_start=(np.zeros(20), np.zeros(20), np.zeros((20, 20))))
    opts.warm_dual_source = None
    opts.warm_dual_target = None
    lib = pdot._abi.load()
    mp = pdot.api.MarshalledProblem(prob)
    cp = pdot.api.marshal_params(pdot.default_parameters(1e-4))
    ob = pdot.api.OutputBuffers(20, 20, 16)
    import ctypes as ct
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(opts), ct.byref(ob.c))
    assert rc == pdot._abi.PDOT_ERR_INVALID_ARGUMENT
    del keep


def test_batched_warm_and_cold_instances(cuda):
    """Exact warm starts end at the first evaluation; cold instances in the
    same batch solve to the same optimum as in an all-cold batch (not bit for
    bit: the batched reductions are partitioned over the instances still
    active, and the warm ones leave at once)."""
    probs, pts = instances.batched_l1(6, 40, 120, seed=3)
    params = pdot.default_parameters(1e-4)
    cold, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts)
    warm = [None if k % 2 else (o.dual_source_solution, o.dual_target_solution, o.primal_solution)
            for k, o in enumerate(cold)]
    again, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, warm_starts=warm)
    for k, (c, w) in enumerate(zip(cold, again)):
        assert w.termination_reason == OPTIMAL
        if k % 2:
            ow = w.iteration_stats[-1].convergence_information[0].primal_objective
            oc = c.iteration_stats[-1].convergence_information[0].primal_objective
            assert abs(ow - oc) <= 2e-4 * (1 + abs(oc))
        else:
            assert w.iteration_count == 0


def test_race_groups_stop_the_slower_member(cuda):
    """An exact warm start and a cold start of the same problem in one race
    group: the warm one is optimal at the first evaluation and the cold one
    stops there (reason OTHER); an instance outside the group is unaffected."""
    probs, pts = instances.batched_l1(2, 50, 90, seed=11)
    params = pdot.default_parameters(1e-4)
    cold, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts)
    o = cold[0]
    batch = [probs[0], probs[0], probs[1]]
    bpts = [pts[0], pts[0], pts[1]]
    warm = [(o.dual_source_solution, o.dual_target_solution, o.primal_solution), None, None]
    out, _ = pdot.optimize_batched(params, batch, cost="l1", points=bpts, warm_starts=warm,
                                   race_groups=[0, 0, -1])
    assert out[0].termination_reason == OPTIMAL and out[0].iteration_count == 0
    assert out[1].termination_reason == pdot.TerminationReason.TERMINATION_REASON_OTHER
    assert out[1].iteration_count == 0
    # the stopped member keeps its last evaluation record (the first one here)
    assert out[1].iteration_stats[-1].iteration_number == 1
    assert out[1].iteration_stats[-1].convergence_information[0].l2_primal_residual > 0
    assert out[2].termination_reason == OPTIMAL and out[2].iteration_count == cold[1].iteration_count
    with pytest.raises(pdot._abi.PdotError):
        pdot.optimize_batched(params, batch, cost="l1", points=bpts, race_groups=[0, 3, -1])


def test_warm_primal_weight_is_the_initial_weight(cuda):
    prob = instances.uniform_sqeuclid(60, 50, seed=6)
    params = pdot.default_parameters(1e-4, iteration_limit=3)
    cold = oracle.optimize(pdot.default_parameters(1e-4), prob)
    u0, v0, X0 = _perturbed(cold, np.random.default_rng(4), 0.05)
    g = pdot.optimize(params, prob, warm_start=(u0, v0, X0), warm_primal_weight=7.5)
    o = oracle.optimize_warm(params, prob, u0, v0, X0, omega0=7.5)
    assert g.iteration_stats[0].primal_weight == 7.5
    for a, b in zip(g.iteration_stats, o.iteration_stats):
        assert a.primal_weight == pytest.approx(b.primal_weight, rel=1e-9)
        assert a.step_size == pytest.approx(b.step_size, rel=1e-9)


@pytest.mark.parametrize("m,n", [(64, 48)])
def test_warm_restart_at_zero_matches_the_oracle(cuda, m, n):
    """With warm_restart="zero" the restart information starts at the zero
    point, as a cold start's, on both sides."""
    prob = instances.uniform_sqeuclid(m, n, seed=m + 1)
    cold = oracle.optimize(pdot.default_parameters(1e-4), prob)
    u0, v0, X0 = _perturbed(cold, np.random.default_rng(3), 0.05)
    p128 = pdot.default_parameters(1e-4, iteration_limit=128)
    g = pdot.optimize(p128, prob, warm_start=(u0, v0, X0), warm_restart="zero")
    o = oracle.optimize_warm(p128, prob, u0, v0, X0, restart_at_zero=True)
    w = oracle.optimize_warm(p128, prob, u0, v0, X0)
    assert len(g.iteration_stats) == len(o.iteration_stats)
    for a, b in zip(g.iteration_stats, o.iteration_stats):
        assert a.restart_used == b.restart_used
        assert a.step_size == pytest.approx(b.step_size, rel=1e-9)
        assert a.primal_weight == pytest.approx(b.primal_weight, rel=1e-9)
        ca, cb = a.convergence_information[0], b.convergence_information[0]
        assert ca.primal_objective == pytest.approx(cb.primal_objective, rel=1e-9, abs=1e-14)
    # the two records differ: the first primal-weight update measures from a different point
    assert [s.primal_weight for s in o.iteration_stats] != [s.primal_weight for s in w.iteration_stats]
