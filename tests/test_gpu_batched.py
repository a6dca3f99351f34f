"""The batched solver (pdot_optimize_batched): many instances of uneven sizes,
each with its own step size, restarts and termination, in one lockstep solve.

Each instance is checked against the FP64 problem built from the same
coordinates: OPTIMAL, FP64 relative KKT of its returned solution within 2x the
tolerance (FP32 plans), objective within the tolerance band of the FP64
single-instance solve. Sizes cover a single row/column, rows that are not a
multiple of 4 (padded plan storage) and more than one row panel.
"""
import math

import numpy as np
import pytest

import pdot
from pdot import instances

pytestmark = pytest.mark.gpu

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


def fp64_kkt(C, a, b, X, u, v):
    pres = math.sqrt(np.sum((a - X.sum(axis=1)) ** 2) + np.sum((b - X.sum(axis=0)) ** 2))
    dres = float(np.linalg.norm(np.minimum(C - u[:, None] - v[None, :], 0.0)))
    pobj, dobj = float(np.vdot(C, X)), float(a @ u + b @ v)
    return pobj, max(pres / (1 + np.linalg.norm(np.concatenate([a, b]))), dres / (1 + np.linalg.norm(C)),
                     abs(pobj - dobj) / (1 + abs(pobj) + abs(dobj)))


SIZES = [(1, 1), (1, 17), (13, 1), (7, 5), (64, 64), (130, 77), (257, 300), (511, 129), (600, 601)]


@pytest.mark.parametrize("cost, panel_rows", [("l1", 256), ("sqeuclid", 256), ("f32", 256), ("l1", 128),
                                              ("f32", 128)])
def test_batched_instances_solve_their_fp64_problems(cuda, cost, panel_rows):
    tol = 1e-4
    rng = np.random.default_rng(7)
    probs, pts, fp64 = [], [], []
    for m, n in SIZES:
        xs, ys = rng.uniform(0, 1, (m, 2)).astype(np.float32), rng.uniform(0, 1, (n, 2)).astype(np.float32)
        a, b = rng.dirichlet(np.ones(m)), rng.dirichlet(np.ones(n))
        C = (instances.l1_cost if cost == "l1" else instances.sqeuclid_cost)(xs.astype(np.float64),
                                                                             ys.astype(np.float64))
        fp64.append(pdot.OptimalTransportProblem(C, a, b))
        probs.append(pdot.OptimalTransportProblem(C if cost == "f32" else None, a, b))
        pts.append((xs, ys))
    params = pdot.default_parameters(tol)
    outs, seconds = pdot.optimize_batched(params, probs, cost=cost, points=None if cost == "f32" else pts,
                                          panel_rows=panel_rows)
    assert seconds > 0
    for (m, n), o, p64 in zip(SIZES, outs, fp64):
        assert o.termination_reason == OPTIMAL, (m, n, o.termination_string)
        pobj, kkt = fp64_kkt(p64.cost_matrix, p64.source_distribution, p64.target_distribution,
                             o.primal_solution, o.dual_source_solution, o.dual_target_solution)
        assert kkt <= 2 * tol, (m, n, kkt)
        ref = pdot.optimize(params, p64)
        ref_obj = ref.iteration_stats[-1].convergence_information[0].primal_objective
        assert abs(pobj - ref_obj) <= 2 * tol * (1 + abs(ref_obj)), (m, n)


@pytest.mark.parametrize("panel_rows", [256, 128])
def test_batched_matches_single_instance_mixed_precision_early(cuda, panel_rows):
    """Same arithmetic per entry as the single-instance FP32 solve of one
    instance, with either tile: the first evaluations agree to rounding of the
    sums."""
    rng = np.random.default_rng(3)
    m, n = 300, 200
    xs, ys = rng.uniform(0, 1, (m, 2)).astype(np.float32), rng.uniform(0, 1, (n, 2)).astype(np.float32)
    a, b = rng.dirichlet(np.ones(m)), rng.dirichlet(np.ones(n))
    prob = pdot.OptimalTransportProblem(None, a, b)
    params = pdot.default_parameters(1e-4, iteration_limit=9)
    single = pdot.optimize(params, prob, precision="f32", cost="l1", points=(xs, ys))
    outs, _ = pdot.optimize_batched(params, [prob], cost="l1", points=[(xs, ys)], panel_rows=panel_rows)
    assert outs[0].iteration_count == single.iteration_count
    cs = single.iteration_stats[-1].convergence_information[0]
    cb = outs[0].iteration_stats[-1].convergence_information[0]
    assert cb.primal_objective == pytest.approx(cs.primal_objective, rel=1e-7, abs=1e-12)
    assert cb.l2_primal_residual == pytest.approx(cs.l2_primal_residual, rel=1e-7)
    np.testing.assert_allclose(outs[0].dual_source_solution, single.dual_source_solution, rtol=1e-7, atol=1e-12)


def test_batched_invalid_instance_does_not_stop_the_others(cuda):
    rng = np.random.default_rng(1)
    probs = []
    for m, n in [(40, 30), (20, 25), (33, 33)]:
        C = np.asfortranarray(rng.uniform(0, 1, (m, n)))
        probs.append(pdot.OptimalTransportProblem(C, rng.dirichlet(np.ones(m)), rng.dirichlet(np.ones(n))))
    probs[1].cost_matrix[3, 4] = math.nan
    outs, _ = pdot.optimize_batched(pdot.default_parameters(1e-4), probs, cost="f32")
    assert outs[1].termination_reason == pdot.TerminationReason.TERMINATION_REASON_INVALID_PROBLEM
    assert outs[0].termination_reason == OPTIMAL and outs[2].termination_reason == OPTIMAL


@pytest.mark.parametrize("panel_rows", [256, 128])
def test_batched_is_deterministic(cuda, panel_rows):
    probs, pts = instances.batched_l1(count=24, lo=16, hi=300, seed=5)
    params = pdot.default_parameters(1e-4)
    o1, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, panel_rows=panel_rows)
    o2, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, panel_rows=panel_rows)
    for x, y in zip(o1, o2):
        assert x.iteration_count == y.iteration_count
        assert np.array_equal(x.primal_solution, y.primal_solution)


@pytest.mark.parametrize("cost, panel_rows", [("l1", 256), ("f32", 256), ("l1", 128), ("f32", 128)])
def test_batched_staged_and_direct_passes_agree(cuda, cost, panel_rows):
    """The bulk-copy staged pass and the direct pass do the same arithmetic in
    the same order over the same CTA partition (the same tile, the same CTAs
    per SM), so the solves agree bit for bit. Sizes include partial panels and
    rows that are not a multiple of 4."""
    probs, pts = instances.batched_l1(count=20, lo=3, hi=700, seed=9)
    if cost == "f32":
        probs = [pdot.OptimalTransportProblem(instances.l1_cost(*pt), p.source_distribution, p.target_distribution)
                 for p, pt in zip(probs, pts)]
    params = pdot.default_parameters(1e-4)
    kw = {} if cost == "f32" else {"points": pts}
    kw.update(panel_rows=panel_rows, ctas_per_sm=3 if panel_rows == 128 else 2)
    st, _ = pdot.optimize_batched(params, probs, cost=cost, primal_pass="staged", **kw)
    di, _ = pdot.optimize_batched(params, probs, cost=cost, primal_pass="direct", **kw)
    for x, y in zip(st, di):
        assert x.termination_reason == OPTIMAL
        assert x.iteration_count == y.iteration_count
        assert np.array_equal(x.primal_solution, y.primal_solution)
        assert np.array_equal(x.dual_source_solution, y.dual_source_solution)


@pytest.mark.parametrize("panel_rows", [256, 128])
@pytest.mark.parametrize("sizes", [[(65, 40), (3, 5), (300, 200)], [(257, 70), (700, 650), (128, 3)],
                                   [(3, 40), (300, 200)], [(65, 40), (300, 5)], [(129, 7), (127, 300), (385, 2)]])
def test_batched_small_instances_both_pass_forms(cuda, sizes, panel_rows):
    """Batches with a few rows or a few columns (fewer columns than warps, a
    single 8-row padded panel) beside larger instances, with point costs: the
    staged pass's copies and waits cover every unit (no bounded wait gives up)
    and it agrees bit for bit with the direct pass."""
    rng = np.random.default_rng(1)
    probs, pts = [], []
    for m, n in sizes:
        xs, ys = rng.uniform(0, 1, (m, 2)).astype(np.float32), rng.uniform(0, 1, (n, 2)).astype(np.float32)
        probs.append(pdot.OptimalTransportProblem(None, rng.dirichlet(np.ones(m)), rng.dirichlet(np.ones(n))))
        pts.append((xs, ys))
    params = pdot.default_parameters(1e-4, iteration_limit=3000)
    kw = dict(panel_rows=panel_rows, ctas_per_sm=3 if panel_rows == 128 else 2)
    st, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, primal_pass="staged", **kw)
    di, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, primal_pass="direct", **kw)
    for x, y in zip(st, di):
        assert x.iteration_count == y.iteration_count
        assert np.array_equal(x.primal_solution, y.primal_solution)
        assert np.array_equal(x.dual_target_solution, y.dual_target_solution)


def test_autotuner_times_every_candidate_and_picks_the_fastest(cuda):
    probs, pts = instances.batched_l1(count=12, lo=32, hi=400, seed=2)
    best, timings = pdot.tune_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, iterations=64)
    # the launch configurations with 256-row tiles at the default balance, the
    # 128-row tiles for the best of them, then the other balances for the best
    others = [c for c in pdot.api.BATCH_UNIT_COSTS if c != 0.25]
    assert len(timings) == len(pdot.api.BATCH_TUNING_CANDIDATES) + len(pdot.api.BATCH_TILE_SHAPES) + len(others)
    assert {t[0]["panel_rows"] for t in timings} == {128, 256}
    assert best == min(timings, key=lambda t: t[1])[0]
    outs, _ = pdot.optimize_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, **best)
    assert all(o.termination_reason == OPTIMAL for o in outs)


@pytest.mark.parametrize("unit_cost", [0.0, 0.125, 8.0])
def test_cost_balanced_cta_split_solves_every_instance(cuda, unit_cost):
    """The CTA ranges cut the units by cost (rows + unit_cost * 256). Every
    split must cover each unit once: the solves end optimal with objectives in
    the tolerance band of the default split's, whatever the order of the sums,
    and each split is deterministic. Sizes of 3 to 700 rows and columns give
    partial panels and short units, and a tail of few active units, where
    ranges can hold no unit."""
    tol = 1e-4
    probs, pts = instances.batched_l1(count=20, lo=3, hi=700, seed=9)
    params = pdot.default_parameters(tol)
    ref, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts)
    got, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, unit_cost=unit_cost)
    again, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts, unit_cost=unit_cost)
    for r, g, g2 in zip(ref, got, again):
        assert g.termination_reason == OPTIMAL
        assert np.array_equal(g.primal_solution, g2.primal_solution)
        ro = r.iteration_stats[-1].convergence_information[0].primal_objective
        go = g.iteration_stats[-1].convergence_information[0].primal_objective
        assert abs(go - ro) <= 2 * tol * (1 + abs(ro))


def test_batch_unit_cost_is_validated(cuda):
    probs, pts = instances.batched_l1(count=2, lo=8, hi=16, seed=1)
    with pytest.raises(pdot.api._abi.PdotError) as ei:
        pdot.optimize_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, unit_cost=9.0)
    assert ei.value.code == pdot.api._abi.PDOT_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("cost, panel_rows", [("l1", 256), ("f32", 256), ("l1", 128)])
def test_batched_persistent_chunks_match_the_graph(cuda, cost, panel_rows):
    """A regular chunk as one persistent cooperative launch runs every phase's
    body over the same virtual CTA ranges and vector blocks as the graph's
    launches (the direct pass, the same CTAs per SM), so the solves agree bit
    for bit, through compactions that drop finished instances."""
    probs, pts = instances.batched_l1(count=20, lo=3, hi=700, seed=9)
    if cost == "f32":
        probs = [pdot.OptimalTransportProblem(instances.l1_cost(*pt), p.source_distribution, p.target_distribution)
                 for p, pt in zip(probs, pts)]
    params = pdot.default_parameters(1e-4)
    kw = {} if cost == "f32" else {"points": pts}
    kw.update(panel_rows=panel_rows, ctas_per_sm=2, primal_pass="direct")
    gr, _ = pdot.optimize_batched(params, probs, cost=cost, **kw)
    pe, _ = pdot.optimize_batched(params, probs, cost=cost, persistent=True, **kw)
    iters = set()
    for x, y in zip(gr, pe):
        assert x.termination_reason == OPTIMAL
        assert x.termination_reason == y.termination_reason
        assert x.iteration_count == y.iteration_count
        assert np.array_equal(x.primal_solution, y.primal_solution)
        assert np.array_equal(x.dual_source_solution, y.dual_source_solution)
        assert np.array_equal(x.dual_target_solution, y.dual_target_solution)
        iters.add(x.iteration_count)
    assert max(iters) > 256 and len(iters) > 1  # a whole regular chunk, instances ending at different ones


def test_batched_persistent_chunks_with_warm_starts_and_races(cuda):
    """Warm starts with recovered plans and race groups through the persistent
    chunk: the same outputs as the graph, bit for bit."""
    probs, pts = instances.batched_l1(count=6, lo=40, hi=300, seed=4)
    params = pdot.default_parameters(1e-4)
    cold, _ = pdot.optimize_batched(params, probs, cost="l1", points=pts)
    rng = np.random.default_rng(0)
    warm = [(o.dual_source_solution * (1 + 0.05 * rng.standard_normal(o.dual_source_solution.size)),
             o.dual_target_solution) for o in cold]
    probs2, pts2 = probs + probs, pts + pts
    ws = [None] * len(probs) + warm
    groups = list(range(len(probs))) * 2
    kw = dict(cost="l1", points=pts2, warm_starts=ws, race_groups=groups, recover_plan=(3e-4, 20),
              primal_pass="direct", ctas_per_sm=2)
    gr, _ = pdot.optimize_batched(params, probs2, **kw)
    pe, _ = pdot.optimize_batched(params, probs2, persistent=True, **kw)
    for x, y in zip(gr, pe):
        assert x.termination_reason == y.termination_reason
        assert x.iteration_count == y.iteration_count
        assert np.array_equal(x.primal_solution, y.primal_solution)


def test_batched_persistent_chunks_need_the_direct_pass(cuda):
    probs, pts = instances.batched_l1(count=2, lo=8, hi=16, seed=1)
    with pytest.raises(pdot.api._abi.PdotError) as ei:
        pdot.optimize_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, persistent=True,
                              primal_pass="staged")
    assert ei.value.code == pdot.api._abi.PDOT_ERR_INVALID_ARGUMENT
