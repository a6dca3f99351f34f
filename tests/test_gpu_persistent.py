"""Persistent chunks: a regular chunk of loop bodies (the evaluation and the
steps up to the next one) as one cooperative launch with grid barriers between
the phases (k_chunk) instead of a CUDA graph of separate launches.

Each phase runs the body of its own kernel over the same CTA ranges of the
matrix passes and the same blocks of the vector passes, with the same
last-block elections, so every result must be bit-identical to the graph
path's: iterates, duals and every iteration-stats record.
"""
import numpy as np
import pytest

import pdot
from pdot import instances

pytestmark = pytest.mark.gpu

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


def _records(o):
    out = []
    for s in o.iteration_stats:
        c = s.convergence_information[0]
        out.append((s.iteration_number, s.step_size, s.primal_weight, int(s.restart_used),
                    s.cumulative_kkt_matrix_passes, c.primal_objective, c.dual_objective,
                    c.l2_primal_residual, c.l2_dual_residual))
    return out


def _assert_same(a, b):
    assert a.iteration_count == b.iteration_count
    assert a.termination_reason == b.termination_reason
    assert np.array_equal(a.primal_solution, b.primal_solution)
    assert np.array_equal(a.dual_source_solution, b.dual_source_solution)
    assert np.array_equal(a.dual_target_solution, b.dual_target_solution)
    assert _records(a) == _records(b)


def test_persistent_chunks_match_the_graph_path_to_tolerance(cuda):
    """m = n = 1000 (4 panels, 296 CTA ranges), FP64, solved to 1e-4: the
    termination found inside a chunk's evaluation, the restarts and the
    step-size retries all go the same way."""
    prob = instances.uniform_sqeuclid(1000, 1000, seed=11)
    params = pdot.default_parameters(1e-4, iteration_limit=20_000)
    g = pdot.optimize(params, prob, persistent=False)
    p = pdot.optimize(params, prob, persistent=True)
    auto = pdot.optimize(params, prob)
    assert g.termination_reason == OPTIMAL
    _assert_same(g, p)
    _assert_same(g, auto)


@pytest.mark.parametrize("m,n,limit", [(4000, 4000, 300), (2050, 300, 700), (256, 4096, 500), (68, 40, 900)])
def test_persistent_chunks_match_the_graph_path_on_shapes(cuda, m, n, limit):
    """Shapes where the dual step has more blocks than the chunk has CTAs
    (4000 x 4000: a warp per row, 516 blocks), a ragged last panel, a single
    panel with many columns, and fewer units than CTAs; iteration limits that
    end inside a chunk."""
    prob = instances.uniform_sqeuclid(m, n, seed=m + n)
    params = pdot.default_parameters(1e-8, iteration_limit=limit)
    g = pdot.optimize(params, prob, persistent=False)
    p = pdot.optimize(params, prob, persistent=True)
    _assert_same(g, p)


@pytest.mark.parametrize("cost", ["f32", "bf16", "sqeuclid", "l1"])
def test_persistent_chunks_match_the_graph_path_mixed_precision(cuda, cost):
    """FP32 plans with every cost source, through the direct 16-byte pass (the
    staged pass has no persistent form)."""
    rng = np.random.default_rng(5)
    m, n = 1200, 900
    xs = rng.uniform(0, 1, (m, 2)).astype(np.float32)
    ys = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    base = instances.uniform_sqeuclid(m, n, seed=5)
    kw = {"precision": "f32", "cost": cost, "primal_pass": "direct"}
    if cost in ("sqeuclid", "l1"):
        kw["points"] = (xs, ys)
        prob = pdot.OptimalTransportProblem(None, base.source_distribution, base.target_distribution)
    else:
        prob = base
    params = pdot.default_parameters(1e-4, iteration_limit=3000)
    g = pdot.optimize(params, prob, persistent=False, **kw)
    p = pdot.optimize(params, prob, persistent=True, **kw)
    _assert_same(g, p)


def test_persistent_chunks_with_a_warm_start(cuda):
    """A warm start (start-point evaluation, stored gradient C - u - v) runs
    its regular chunks persistently too."""
    prob = instances.uniform_sqeuclid(600, 500, seed=8)
    params = pdot.default_parameters(1e-4, iteration_limit=20_000)
    cold = pdot.optimize(params, prob)
    u = cold.dual_source_solution * 0.9
    v = cold.dual_target_solution * 0.9
    g = pdot.optimize(params, prob, warm_start=(u, v), persistent=False)
    p = pdot.optimize(params, prob, warm_start=(u, v), persistent=True)
    assert g.termination_reason == OPTIMAL
    _assert_same(g, p)


def test_persistent_solver_iterates_in_pieces(cuda):
    """The stepwise Solver: chunks issued by iterate() calls of odd lengths
    (regular chunks persistent, the rest as single loop bodies) give the same
    state as one optimize call."""
    prob = instances.uniform_sqeuclid(700, 650, seed=4)
    params = pdot.default_parameters(1e-4, iteration_limit=5000)
    ref = pdot.optimize(params, prob, persistent=False)
    s = pdot.Solver(params, prob, persistent=True)
    try:
        for k in (3, 70, 129, 1, 256, 5000):
            s.iterate(k)
        out = s.finish()
    finally:
        s.close()
    _assert_same(ref, out)
