"""Mixed precision and warm start on the GPU (this implementation's additions).

Mixed precision keeps the plan and its average in FP32, takes the cost from
FP32 or BF16 storage or computes the squared-Euclidean cost from FP32
coordinates, and keeps duals, sums and control in FP64. Every result is judged
against the FP64 problem: the returned plan and duals are evaluated on the
host with the FP64 cost (relative KKT with the reference's definitions,
src/utils_gpu.jl:68-129 and src/termination.jl:106-134), and the objective is
compared with the FP64 drop-in solve of the same instance.

Tolerances: FP32 storage perturbs the cost by ~6e-8 relative, so the FP64
relative KKT of an FP32 solve at tolerance 1e-4 stays below 2e-4 and its
objective within the 1e-4 KKT band of the FP64 solve. BF16 storage rounds each
cost to 2^-9 relative; since the plan sums to 1, the FP64 objective of the BF16
solution is within 3 * 2^-9 * max(C) of the optimum (the cost error on the plan,
plus the optimum of the perturbed problem), plus the tolerance band.
"""
import math

import numpy as np
import pytest

import pdot
from pdot import instances

pytestmark = pytest.mark.gpu

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


def fp64_kkt(prob, X, u, v):
    """Relative L2 KKT errors of (X, u, v) on the FP64 problem."""
    C = np.asarray(prob.cost_matrix)
    a, b = prob.source_distribution, prob.target_distribution
    pres = math.sqrt(np.sum((a - X.sum(axis=1)) ** 2) + np.sum((b - X.sum(axis=0)) ** 2))
    G = C - u[:, None] - v[None, :]
    dres = float(np.linalg.norm(np.minimum(G, 0.0)))
    pobj = float(np.vdot(C, X))
    dobj = float(a @ u + b @ v)
    rel_p = pres / (1.0 + np.linalg.norm(np.concatenate([a, b])))
    rel_d = dres / (1.0 + np.linalg.norm(C))
    rel_gap = abs(pobj - dobj) / (1.0 + abs(pobj) + abs(dobj))
    return pobj, max(rel_p, rel_d, rel_gap)


def _points_problem(m, n, seed, dim=2):
    rng = np.random.default_rng(seed)
    xs = rng.uniform(0, 1, (m, dim)).astype(np.float32)
    ys = rng.uniform(0, 1, (n, dim)).astype(np.float32)
    a = rng.uniform(0.1, 1.0, m)
    b = rng.uniform(0.1, 1.0, n)
    C = instances.sqeuclid_cost(xs.astype(np.float64), ys.astype(np.float64))
    return pdot.OptimalTransportProblem(C, a / a.sum(), b / b.sum()), xs, ys


@pytest.mark.parametrize("m,n", [(300, 200), (257, 129)])
@pytest.mark.parametrize("cost", ["f32", "bf16", "sqeuclid"])
def test_mixed_precision_solves_the_fp64_problem(cuda, m, n, cost):
    tol = 1e-4
    prob, xs, ys = _points_problem(m, n, seed=m + n)
    params = pdot.default_parameters(tol)
    ref = pdot.optimize(params, prob)
    kw = {"points": (xs, ys)} if cost == "sqeuclid" else {}
    mp = pdot.optimize(params, prob if cost != "sqeuclid" else pdot.OptimalTransportProblem(
        None, prob.source_distribution, prob.target_distribution), precision="f32", cost=cost, **kw)
    assert ref.termination_reason == OPTIMAL and mp.termination_reason == OPTIMAL
    fin = mp.iteration_stats[-1].convergence_information[0]
    assert fin.relative_optimality_gap <= tol and fin.relative_l2_primal_residual <= tol
    pobj, kkt = fp64_kkt(prob, mp.primal_solution, mp.dual_source_solution, mp.dual_target_solution)
    ref_obj = ref.iteration_stats[-1].convergence_information[0].primal_objective
    if cost == "bf16":
        cmax = float(np.max(prob.cost_matrix))
        assert abs(pobj - ref_obj) <= 3 * 2.0**-9 * cmax + 2 * tol * (1 + abs(ref_obj))
    else:
        assert kkt <= 2 * tol
        assert abs(pobj - ref_obj) <= 2 * tol * (1 + abs(ref_obj))


def test_coordinate_cost_matches_stored_fp32_cost_early(cuda):
    """The on-the-fly cost equals the FP32-stored cost up to FP32 rounding, so
    the first evaluations of the two solves agree closely."""
    prob, xs, ys = _points_problem(200, 160, seed=3)
    params = pdot.default_parameters(1e-4, iteration_limit=10)
    s = pdot.optimize(params, prob, precision="f32", cost="f32")
    c = pdot.optimize(params, pdot.OptimalTransportProblem(None, prob.source_distribution,
                                                           prob.target_distribution),
                      precision="f32", cost="sqeuclid", points=(xs, ys))
    for a, b in zip(s.iteration_stats, c.iteration_stats):
        assert a.restart_used == b.restart_used
        ca, cb = a.convergence_information[0], b.convergence_information[0]
        assert ca.primal_objective == pytest.approx(cb.primal_objective, rel=1e-5, abs=1e-9)
        assert ca.l2_primal_residual == pytest.approx(cb.l2_primal_residual, rel=1e-5)


@pytest.mark.parametrize("m", [255, 256, 1001])
def test_fp32_scalar_and_vector_paths(cuda, m):
    prob, xs, ys = _points_problem(m, 97, seed=m)
    params = pdot.default_parameters(1e-4)
    out = pdot.optimize(params, prob, precision="f32", cost="f32")
    assert out.termination_reason == OPTIMAL
    _, kkt = fp64_kkt(prob, out.primal_solution, out.dual_source_solution, out.dual_target_solution)
    assert kkt <= 2e-4


def test_mixed_precision_is_deterministic(cuda):
    prob, xs, ys = _points_problem(400, 300, seed=5)
    params = pdot.default_parameters(1e-4)
    runs = [pdot.optimize(pdot.default_parameters(1e-4), pdot.OptimalTransportProblem(
        None, prob.source_distribution, prob.target_distribution), precision="f32", cost="sqeuclid",
        points=(xs, ys)) for _ in range(2)]
    assert runs[0].iteration_count == runs[1].iteration_count
    assert np.array_equal(runs[0].primal_solution, runs[1].primal_solution)
    del params


def test_warm_start_duals_are_the_starting_point(cuda):
    """A warm start sets the initial duals (and the stored gradient C - u - v);
    the plan still starts at zero, and the solve ends at the optimum."""
    prob = instances.uniform_sqeuclid(300, 250, seed=8)
    params = pdot.default_parameters(1e-4)
    cold = pdot.optimize(params, prob)
    warm = pdot.optimize(params, prob, warm_start=(cold.dual_source_solution, cold.dual_target_solution))
    assert warm.termination_reason == OPTIMAL
    obj_c = cold.iteration_stats[-1].convergence_information[0].primal_objective
    obj_w = warm.iteration_stats[-1].convergence_information[0].primal_objective
    assert abs(obj_w - obj_c) <= 2e-4 * (1 + abs(obj_c))
    # the first evaluation sees the given duals and their reduced costs
    c0 = warm.iteration_stats[0].convergence_information[0]
    assert c0.dual_objective == pytest.approx(
        float(prob.source_distribution @ cold.dual_source_solution
              + prob.target_distribution @ cold.dual_target_solution), rel=1e-12)
    G = prob.cost_matrix - cold.dual_source_solution[:, None] - cold.dual_target_solution[None, :]
    assert c0.l2_dual_residual == pytest.approx(float(np.linalg.norm(np.minimum(G, 0))), rel=1e-9, abs=1e-15)


def test_option_validation(cuda):
    prob = instances.uniform_sqeuclid(20, 20, seed=1)
    params = pdot.default_parameters(1e-4)
    with pytest.raises(pdot._abi.PdotError):
        pdot.optimize(params, prob, precision="f64", cost="bf16")
    with pytest.raises(pdot._abi.PdotError):
        pdot.optimize(params, pdot.OptimalTransportProblem(None, prob.source_distribution,
                                                           prob.target_distribution), precision="f32",
                      cost="f32")
