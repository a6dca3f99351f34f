"""The CPU oracle, pinned before it is trusted (no GPU needed).

The reference ships no tests or golden vectors, and it cannot run here (no
Julia), so the pins are: the exact LP optimum of each committed instance
(scipy HiGHS, stored in tests/golden/golden.json), analytic optima, the
reference's documented quirks, and the oracle's own committed trajectories
(a regression pin).
"""
import json
import math
import os

import numpy as np
import pytest

import oracle
import pdot
from pdot import instances

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))["cases"]
ARRAYS = np.load(os.path.join(HERE, "golden", "instances.npz"))

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


def golden_problem(case):
    k = case["key"]
    return pdot.OptimalTransportProblem(np.asfortranarray(ARRAYS[k + "_C"]), ARRAYS[k + "_a"], ARRAYS[k + "_b"])


@pytest.mark.parametrize("case", GOLDEN, ids=[c["key"] for c in GOLDEN])
def test_oracle_reaches_highs_optimum(built, case):
    tol = case["tolerance"]
    out = oracle.optimize(pdot.default_parameters(tol), golden_problem(case))
    assert out.termination_reason == OPTIMAL
    fin = out.iteration_stats[-1].convergence_information[0]
    opt = case["highs_objective"]
    # the relative KKT test bounds the gap by tol*(1 + |pobj| + |dobj|)
    assert abs(fin.primal_objective - opt) <= 4 * tol * (1 + abs(opt))
    assert fin.relative_optimality_gap <= tol
    assert fin.relative_l2_primal_residual <= tol
    assert fin.relative_l2_dual_residual <= tol


@pytest.mark.parametrize("case", GOLDEN, ids=[c["key"] for c in GOLDEN])
def test_oracle_matches_committed_trajectory(built, case):
    """Regression pin: the oracle reproduces its committed records exactly in
    structure and to 1e-12 in value (single-threaded)."""
    out = oracle.optimize(pdot.default_parameters(case["tolerance"]), golden_problem(case), num_threads=1)
    assert int(out.termination_reason) == case["termination_reason"]
    assert out.iteration_count == case["iteration_count"]
    for s, g in zip(out.iteration_stats, case["early"]):
        c = s.convergence_information[0]
        assert s.iteration_number == g["iteration_number"]
        assert int(s.restart_used) == g["restart_used"]
        assert s.cumulative_kkt_matrix_passes == g["cumulative_kkt_matrix_passes"]
        for name, val in (("step_size", s.step_size), ("primal_weight", s.primal_weight),
                          ("primal_objective", c.primal_objective), ("dual_objective", c.dual_objective),
                          ("l2_primal_residual", c.l2_primal_residual),
                          ("l2_dual_residual", c.l2_dual_residual)):
            assert val == pytest.approx(g[name], rel=1e-12, abs=1e-300), name


def test_oracle_is_independent_of_thread_count(built):
    prob = instances.uniform_sqeuclid(64, 48, seed=4)
    params = pdot.default_parameters(1e-5)
    a = oracle.optimize(params, prob, num_threads=1)
    b = oracle.optimize(params, prob, num_threads=4)
    assert a.iteration_count == b.iteration_count
    assert np.array_equal(a.primal_solution, b.primal_solution)


def test_single_source_and_single_target_are_exact(built):
    """m = 1: the only feasible plan is X = b^T; n = 1: X = a."""
    rng = np.random.default_rng(3)
    for m, n in ((1, 12), (12, 1)):
        C = np.asfortranarray(rng.uniform(0, 1, (m, n)))
        a = np.full(m, 1.0 / m)
        b = np.full(n, 1.0 / n)
        out = oracle.optimize(pdot.default_parameters(1e-8), pdot.OptimalTransportProblem(C, a, b))
        assert out.termination_reason == OPTIMAL
        expect = float(np.sum(C * (b[None, :] if m == 1 else a[:, None])))
        fin = out.iteration_stats[-1].convergence_information[0]
        assert fin.primal_objective == pytest.approx(expect, rel=1e-6)


def test_identity_permutation_has_zero_cost(built):
    k = 16
    C = np.asfortranarray(1.0 - np.eye(k))
    a = np.full(k, 1.0 / k)
    out = oracle.optimize(pdot.default_parameters(1e-8), pdot.OptimalTransportProblem(C, a, a.copy()))
    assert out.termination_reason == OPTIMAL
    assert out.iteration_stats[-1].convergence_information[0].primal_objective == pytest.approx(0.0, abs=1e-7)


def test_first_iteration_quirks(built):
    """Stored gradient starts at 0 (src/solver_gpu.jl:434): the first
    evaluation sees a zero dual residual, the first step moves only the duals
    (u = tau*omega*a) with zero interaction, so it is accepted and the step
    grows by (1 + 1/2) (src/solver_gpu.jl:359-363)."""
    prob = instances.uniform_sqeuclid(9, 6, seed=2)
    params = pdot.default_parameters(1e-4, iteration_limit=3)
    out = oracle.optimize(params, prob)
    s0, s1 = out.iteration_stats[0], out.iteration_stats[1]
    assert s0.iteration_number == 1 and s0.step_size == 1.0
    assert s0.convergence_information[0].l2_dual_residual == 0.0
    assert s0.cumulative_kkt_matrix_passes == 2.0
    assert s1.step_size == 1.5
    assert s1.cumulative_kkt_matrix_passes == 5.0  # 2 (eval) + 1 (step) + 2 (eval)
    # the dual of the first step: u = tau*omega*a; the average after one step is it
    assert s1.convergence_information[0].dual_objective == pytest.approx(
        float(prob.source_distribution @ prob.source_distribution + prob.target_distribution
              @ prob.target_distribution), rel=1e-14)
    # Q7: the reported dual-variable norm measures [u; u]
    u = prob.source_distribution
    assert s1.convergence_information[0].l2_dual_variable == pytest.approx(math.sqrt(2.0) * np.linalg.norm(u),
                                                                           rel=1e-14)


@pytest.mark.parametrize("limit,count", [(1, 0), (2, 1), (5, 4), (10, 9), (11, 11), (100, 100)])
def test_iteration_limit_is_checked_at_evaluations(built, limit, count):
    prob = instances.uniform_sqeuclid(10, 10, seed=1)
    out = oracle.optimize(pdot.default_parameters(1e-14, iteration_limit=limit), prob)
    assert out.termination_reason == pdot.TerminationReason.TERMINATION_REASON_ITERATION_LIMIT
    assert out.iteration_count == count


def test_artificial_restarts_in_warmup(built):
    """Iterations 2 and 3 satisfy restart_length >= 0.36 * iterations_completed."""
    out = oracle.optimize(pdot.default_parameters(1e-6, iteration_limit=12), instances.uniform_sqeuclid(30, 20))
    restarts = [s.restart_used for s in out.iteration_stats]
    assert restarts[0] == pdot.RestartChoice.RESTART_CHOICE_NO_RESTART
    assert restarts[1] != pdot.RestartChoice.RESTART_CHOICE_NO_RESTART
    assert restarts[2] != pdot.RestartChoice.RESTART_CHOICE_NO_RESTART


def test_constant_step_size_and_schemes_run(built):
    prob = instances.uniform_sqeuclid(20, 15, seed=5)
    for mod in ("constant", "no_restarts", "fixed", "linf"):
        params = pdot.default_parameters(1e-4, iteration_limit=3000)
        if mod == "constant":
            params.step_size_policy_params = pdot.ConstantStepsizeParams()
        elif mod == "no_restarts":
            params.restart_params.restart_scheme = pdot.NO_RESTARTS
        elif mod == "fixed":
            params.restart_params.restart_scheme = pdot.FIXED_FREQUENCY
            params.restart_params.restart_frequency_if_fixed = 64
        else:
            params.termination_criteria.optimality_norm = pdot.L_INF
        out = oracle.optimize(params, prob)
        if mod == "constant":
            assert out.iteration_stats[0].step_size == pytest.approx(0.8 / math.sqrt(35), rel=1e-15)
        assert out.termination_reason in (OPTIMAL, pdot.TerminationReason.TERMINATION_REASON_ITERATION_LIMIT)


def test_trajectory_sensitivity_to_one_ulp(built):
    """Why long GPU/oracle trajectories are compared through the KKT band: one
    input entry moved by one ulp changes the oracle's own iteration count here,
    while the final objective stays within the tolerance band."""
    tol = 1e-6
    prob = instances.uniform_sqeuclid(7, 5, seed=0)
    params = pdot.default_parameters(tol)
    base = oracle.optimize(params, prob)
    C = prob.cost_matrix.copy(order="F")
    C[2, 3] = np.nextafter(C[2, 3], 2.0)
    pert = oracle.optimize(params, pdot.OptimalTransportProblem(C, prob.source_distribution,
                                                                prob.target_distribution))
    b = base.iteration_stats[-1].convergence_information[0].primal_objective
    p = pert.iteration_stats[-1].convergence_information[0].primal_objective
    assert pert.termination_reason == OPTIMAL
    assert pert.iteration_count != base.iteration_count
    assert abs(p - b) <= 2 * tol * (1 + abs(b))


def _highs_objective(C, a, b):
    """The exact OT optimum by scipy's HiGHS (an independent known answer)."""
    from scipy.optimize import linprog

    m, n = C.shape
    A_eq = np.zeros((m + n, m * n))
    for i in range(m):
        A_eq[i, i::m] = 1.0           # column-major: entry (i, j) at i + j*m
    for j in range(n):
        A_eq[m + j, j * m:(j + 1) * m] = 1.0
    res = linprog(C.ravel(order="F"), A_eq=A_eq, b_eq=np.concatenate([a, b]), bounds=(0, None), method="highs")
    assert res.status == 0
    return res.fun


def test_zero_mass_rows_and_columns_reach_the_optimum(built):
    """Marginals with zero entries (sources or targets that carry nothing)."""
    rng = np.random.default_rng(21)
    prob = instances.uniform_sqeuclid(14, 11, seed=21)
    a = prob.source_distribution.copy()
    b = prob.target_distribution.copy()
    a[[2, 7]] = 0.0
    b[[0, 5, 10]] = 0.0
    a /= a.sum()
    b /= b.sum()
    tol = 1e-6
    out = oracle.optimize(pdot.default_parameters(tol), pdot.OptimalTransportProblem(prob.cost_matrix, a, b))
    assert out.termination_reason == OPTIMAL
    opt = _highs_objective(prob.cost_matrix, a, b)
    fin = out.iteration_stats[-1].convergence_information[0]
    assert abs(fin.primal_objective - opt) <= 4 * tol * (1 + abs(opt))
    del rng


def test_l_inf_optimality_norm_reaches_the_optimum(built):
    prob = instances.uniform_sqeuclid(12, 9, seed=5)
    params = pdot.default_parameters(1e-6)
    params.termination_criteria.optimality_norm = pdot.L_INF
    out = oracle.optimize(params, prob)
    assert out.termination_reason == OPTIMAL
    opt = _highs_objective(prob.cost_matrix, prob.source_distribution, prob.target_distribution)
    fin = out.iteration_stats[-1].convergence_information[0]
    assert abs(fin.primal_objective - opt) <= 4e-6 * (1 + abs(opt))
    assert fin.relative_l_inf_primal_residual <= 1e-6


def test_exact_warm_start_ends_at_the_first_evaluation(built):
    prob = instances.uniform_sqeuclid(20, 16, seed=6)
    params = pdot.default_parameters(1e-5)
    cold = oracle.optimize(params, prob)
    warm = oracle.optimize_warm(params, prob, cold.dual_source_solution, cold.dual_target_solution,
                                cold.primal_solution)
    assert warm.termination_reason == OPTIMAL and warm.iteration_count == 0
    # duals only: the plan starts at zero, the solve still ends at the optimum
    duals = oracle.optimize_warm(params, prob, cold.dual_source_solution, cold.dual_target_solution)
    assert duals.termination_reason == OPTIMAL
    oc = cold.iteration_stats[-1].convergence_information[0].primal_objective
    od = duals.iteration_stats[-1].convergence_information[0].primal_objective
    assert abs(od - oc) <= 4e-5 * (1 + abs(oc))
