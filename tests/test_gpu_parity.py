"""GPU parity: libpdot.so (through its C ABI) against the CPU oracle.

Tolerances: the elementwise plan/average updates are bit-exact (same operation
order, round-to-nearest, no fused multiply-add on either side). Sums are taken
in a different order on the GPU, so reduced quantities agree to 1e-12 relative
(1e-15 absolute) after one pass.

Full solves are compared in three ways:
  1. the early evaluation records agree to 1e-9 relative with identical
     restart choices;
  2. both runs stop for the same reason and the GPU run meets the relative
     KKT tolerance asked for;
  3. final objectives agree within the band the KKT test allows,
     |obj_gpu - obj_oracle| <= 2*tol*(1 + |obj|), and within 1e-6 relative
     where the two trajectories track each other (m = n = 1000).
Long trajectories are not compared record by record: the restart and
step-acceptance tests are discrete, and the oracle itself lands on a different
iteration count and objective (within the same KKT band) when one input entry
moves by one ulp (tests/test_oracle.py::test_trajectory_sensitivity_to_one_ulp).
"""
import math

import numpy as np
import pytest

import oracle
import pdot
from pdot import _abi, instances

pytestmark = pytest.mark.gpu

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


def _dev(a, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(device)


def _pass(lib, device, C, X, Xa, u, v, s, nw, aw, flags):
    import torch

    m, n = C.shape
    dC, dX, dXa, du, dv = (_dev(x, device) for x in (C, X, Xa, u, v))
    drow = torch.zeros(m, dtype=torch.float64, device=device)
    dcol = torch.zeros(n, dtype=torch.float64, device=device)
    dsq = torch.zeros(1, dtype=torch.float64, device=device)
    wsb = lib.pdot_primal_pass_workspace_bytes(m, n)
    ws = torch.empty(wsb // 8 + 1, dtype=torch.float64, device=device)
    rc = lib.pdot_primal_pass_f64(m, n, dC.data_ptr(), dX.data_ptr(), dXa.data_ptr(), du.data_ptr(),
                                  dv.data_ptr(), s, nw, aw, flags, drow.data_ptr(), dcol.data_ptr(),
                                  dsq.data_ptr(), ws.data_ptr(), wsb, None)
    _abi.check(lib, rc, "pdot_primal_pass_f64")
    torch.cuda.synchronize()
    return (dX.cpu().numpy().T, dXa.cpu().numpy().T, drow.cpu().numpy(), dcol.cpu().numpy(),
            float(dsq.item()))


@pytest.mark.parametrize("m,n", [(1, 1), (1, 37), (37, 1), (7, 5), (256, 64), (257, 33), (300, 129),
                                 (513, 1000), (1000, 1000), (2048, 3)])
@pytest.mark.parametrize("flags", [0, _abi.PDOT_PASS_ZERO_GRADIENT, _abi.PDOT_PASS_FIRST_AVERAGE])
def test_primal_pass_matches_oracle(cuda, m, n, flags):
    lib = _abi.load()
    rng = np.random.default_rng(m * 7919 + n)
    C = np.asfortranarray(rng.uniform(0, 1, (m, n)))
    X = np.asfortranarray(np.maximum(rng.uniform(-0.005, 0.01, (m, n)), 0.0))
    Xa = np.asfortranarray(rng.uniform(0, 0.01, (m, n)))
    u, v = rng.uniform(-0.5, 0.5, m), rng.uniform(-0.5, 0.5, n)
    gx, gxa, grow, gcol, gsq = _pass(lib, cuda, C, X, Xa, u, v, 0.37, 0.25, 0.8, flags)
    rrow, rcol, rsq = oracle.primal_pass(C, X, Xa, u, v, 0.37, 0.25, 0.8, flags)
    assert np.array_equal(gx, X)
    assert np.array_equal(gxa, Xa)
    np.testing.assert_allclose(grow, rrow, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(gcol, rcol, rtol=1e-12, atol=1e-15)
    assert gsq == pytest.approx(rsq, rel=1e-12, abs=1e-30)


def test_primal_pass_misaligned_buffers(cuda):
    """Odd offsets force the scalar-load path; results must not change."""
    import torch

    lib = _abi.load()
    rng = np.random.default_rng(11)
    m, n = 64, 48
    C = np.asfortranarray(rng.uniform(0, 1, (m, n)))
    X = np.asfortranarray(rng.uniform(0, 0.01, (m, n)))
    Xa = np.asfortranarray(rng.uniform(0, 0.01, (m, n)))
    u, v = rng.uniform(-0.5, 0.5, m), rng.uniform(-0.5, 0.5, n)
    big = [torch.zeros(m * n + 1, dtype=torch.float64, device=cuda) for _ in range(3)]
    for b, a in zip(big, (C, X, Xa)):
        b[1:] = torch.from_numpy(a.ravel(order="F")).to(cuda)
    du, dv = _dev(u, cuda), _dev(v, cuda)
    drow = torch.zeros(m, dtype=torch.float64, device=cuda)
    dcol = torch.zeros(n, dtype=torch.float64, device=cuda)
    dsq = torch.zeros(1, dtype=torch.float64, device=cuda)
    wsb = lib.pdot_primal_pass_workspace_bytes(m, n)
    ws = torch.empty(wsb // 8 + 1, dtype=torch.float64, device=cuda)
    ptr = [b.data_ptr() + 8 for b in big]
    rc = lib.pdot_primal_pass_f64(m, n, ptr[0], ptr[1], ptr[2], du.data_ptr(), dv.data_ptr(), 0.5, 0.3, 0.7, 0,
                                  drow.data_ptr(), dcol.data_ptr(), dsq.data_ptr(), ws.data_ptr(), wsb, None)
    _abi.check(lib, rc, "pdot_primal_pass_f64")
    torch.cuda.synchronize()
    rrow, rcol, rsq = oracle.primal_pass(C, X, Xa, u, v, 0.5, 0.3, 0.7, 0)
    assert np.array_equal(big[1][1:].cpu().numpy().reshape((m, n), order="F"), X)
    assert np.array_equal(big[2][1:].cpu().numpy().reshape((m, n), order="F"), Xa)
    np.testing.assert_allclose(drow.cpu().numpy(), rrow, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(dcol.cpu().numpy(), rcol, rtol=1e-12, atol=1e-15)


def test_primal_pass_rejects_small_workspace(cuda):
    import torch

    lib = _abi.load()
    t = torch.zeros(64, dtype=torch.float64, device=cuda)
    rc = lib.pdot_primal_pass_f64(8, 8, t.data_ptr(), t.data_ptr(), t.data_ptr() + 8, t.data_ptr(),
                                  t.data_ptr(), 1.0, 1.0, 1.0, 0, t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                  t.data_ptr(), 8, None)
    assert rc == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert "workspace" in _abi.last_error(lib)


def _final(out):
    return out.iteration_stats[-1].convergence_information[0]


def _within_kkt_band(a, b, tol):
    return abs(a - b) <= 2.0 * tol * (1.0 + abs(b))


def _assert_solve_parity(prob, params, *, early=6):
    g = pdot.optimize(params, prob)
    r = oracle.optimize(params, prob)
    assert g.termination_reason == r.termination_reason, (g.termination_string, r.termination_string)
    # the first evaluations happen before any restart decision could diverge
    for sg, sr in zip(g.iteration_stats[:early], r.iteration_stats[:early]):
        assert sg.iteration_number == sr.iteration_number
        assert sg.restart_used == sr.restart_used
        assert sg.step_size == pytest.approx(sr.step_size, rel=1e-9)
        assert sg.primal_weight == pytest.approx(sr.primal_weight, rel=1e-9)
        cg, cr = sg.convergence_information[0], sr.convergence_information[0]
        for f in ("primal_objective", "dual_objective", "l2_primal_residual", "l2_dual_residual"):
            assert getattr(cg, f) == pytest.approx(getattr(cr, f), rel=1e-9, abs=1e-14), f
    return g, r


@pytest.mark.parametrize("m,n,seed", [(7, 5, 0), (33, 17, 1), (64, 64, 2), (100, 80, 3), (257, 129, 4)])
def test_solve_matches_oracle(cuda, m, n, seed):
    prob = instances.uniform_sqeuclid(m, n, seed=seed)
    tol = 1e-6
    params = pdot.default_parameters(tol)
    g, r = _assert_solve_parity(prob, params)
    assert g.termination_reason == OPTIMAL
    cg, cr = _final(g), _final(r)
    assert _within_kkt_band(cg.primal_objective, cr.primal_objective, tol)
    assert cg.relative_l2_primal_residual <= tol
    assert cg.relative_l2_dual_residual <= tol
    assert cg.relative_optimality_gap <= tol
    # the returned plan is the average iterate, shaped like the cost matrix
    assert g.primal_solution.shape == (m, n)
    assert float(np.vdot(prob.cost_matrix, g.primal_solution)) == pytest.approx(cg.primal_objective, rel=1e-9)


def test_config1_to_tolerance(cuda):
    """m = n = 1000, sq-Euclidean on U[0,1]^2, tol 1e-4."""
    prob = instances.uniform_sqeuclid(1000, 1000, seed=0)
    params = pdot.default_parameters(1e-4)
    g, r = _assert_solve_parity(prob, params, early=12)
    assert g.termination_reason == OPTIMAL
    # the trajectories track here: same iteration count, objectives to 1e-6
    assert g.iteration_count == r.iteration_count
    assert _final(g).primal_objective == pytest.approx(_final(r).primal_objective, rel=1e-6)


def test_trajectory_first_evaluations_exact_pattern(cuda):
    """Iteration 1 is evaluated on the zero point with the stored gradient 0
    (src/solver_gpu.jl:434): dual residual 0, primal residual ||[a; b]||."""
    prob = instances.uniform_sqeuclid(40, 30, seed=5)
    params = pdot.default_parameters(1e-4)
    g = pdot.optimize(params, prob)
    s0 = g.iteration_stats[0]
    assert s0.iteration_number == 1 and s0.step_size == 1.0
    c0 = s0.convergence_information[0]
    assert c0.l2_dual_residual == 0.0 and c0.primal_objective == 0.0
    ab = np.concatenate([prob.source_distribution, prob.target_distribution])
    assert c0.l2_primal_residual == pytest.approx(np.linalg.norm(ab), rel=1e-14)
    assert g.iteration_stats[1].step_size == 1.5  # first step accepted with interaction 0


@pytest.mark.parametrize("variant", ["constant", "no_restarts", "fixed_frequency", "no_restart_to_current",
                                     "linf", "scale_invariant"])
def test_parameter_variants_match_oracle(cuda, variant):
    prob = instances.uniform_sqeuclid(50, 40, seed=7)
    params = pdot.default_parameters(1e-4, iteration_limit=600)
    rp = params.restart_params
    if variant == "constant":
        params.step_size_policy_params = pdot.ConstantStepsizeParams()
    elif variant == "no_restarts":
        rp.restart_scheme = pdot.NO_RESTARTS
    elif variant == "fixed_frequency":
        rp.restart_scheme = pdot.FIXED_FREQUENCY
        rp.restart_frequency_if_fixed = 64
    elif variant == "no_restart_to_current":
        rp.restart_to_current_metric = pdot.NO_RESTART_TO_CURRENT
    elif variant == "linf":
        params.termination_criteria.optimality_norm = pdot.L_INF
    elif variant == "scale_invariant":
        params.scale_invariant_initial_primal_weight = True
        params.primal_importance = 2.0
    g, r = _assert_solve_parity(prob, params)
    if r.termination_reason == OPTIMAL:
        assert _within_kkt_band(_final(g).primal_objective, _final(r).primal_objective, 1e-4)
    else:
        assert g.iteration_count == r.iteration_count


@pytest.mark.parametrize("limit", [1, 2, 5, 11, 129, 200])
def test_iteration_limit_semantics(cuda, limit):
    """The limit is checked at evaluations with `iteration >= limit`, so a
    limit inside the first ten iterations stops one iteration early
    (src/termination.jl:156; src/solver_gpu.jl:529-531,661)."""
    prob = instances.uniform_sqeuclid(20, 20, seed=1)
    params = pdot.default_parameters(1e-12, iteration_limit=limit)
    g = pdot.optimize(params, prob)
    r = oracle.optimize(params, prob)
    assert g.termination_reason == pdot.TerminationReason.TERMINATION_REASON_ITERATION_LIMIT
    assert g.iteration_count == r.iteration_count
    assert [s.iteration_number for s in g.iteration_stats] == [s.iteration_number for s in r.iteration_stats]


def test_kkt_pass_limit(cuda):
    prob = instances.uniform_sqeuclid(20, 20, seed=1)
    params = pdot.default_parameters(1e-12)
    params.termination_criteria.kkt_matrix_pass_limit = 300.0
    g = pdot.optimize(params, prob)
    r = oracle.optimize(params, prob)
    assert g.termination_reason == pdot.TerminationReason.TERMINATION_REASON_KKT_MATRIX_PASS_LIMIT
    assert g.iteration_count == r.iteration_count


def test_time_limit(cuda):
    prob = instances.uniform_sqeuclid(64, 64, seed=1)
    params = pdot.default_parameters(1e-14)
    params.termination_criteria.time_sec_limit = 0.05
    g = pdot.optimize(params, prob)
    assert g.termination_reason == pdot.TerminationReason.TERMINATION_REASON_TIME_LIMIT
    assert g.iteration_stats[-1].cumulative_time_sec >= 0.05


def test_record_iteration_stats_false_keeps_final_record(cuda):
    prob = instances.uniform_sqeuclid(30, 30, seed=2)
    params = pdot.default_parameters(1e-4)
    params.record_iteration_stats = False
    g = pdot.optimize(params, prob)
    assert len(g.iteration_stats) == 1
    assert g.iteration_stats[0].iteration_number == g.iteration_count + 1


def test_invalid_problem_is_reported_not_trapped(cuda):
    prob = instances.uniform_sqeuclid(16, 16, seed=1)
    C = prob.cost_matrix.copy(order="F")
    C[3, 4] = math.nan
    g = pdot.optimize(pdot.default_parameters(1e-4), pdot.OptimalTransportProblem(C, prob.source_distribution,
                                                                                  prob.target_distribution))
    assert g.termination_reason == pdot.TerminationReason.TERMINATION_REASON_INVALID_PROBLEM
    # the context stays usable
    g2 = pdot.optimize(pdot.default_parameters(1e-4), prob)
    assert g2.termination_reason == OPTIMAL


def test_bitwise_deterministic_and_graph_equivalent(cuda):
    prob = instances.uniform_sqeuclid(300, 200, seed=9)
    params = pdot.default_parameters(1e-5)
    a = pdot.optimize(params, prob)
    b = pdot.optimize(params, prob)
    c = pdot.optimize(params, prob, use_cuda_graph=False)
    for o in (b, c):
        assert o.iteration_count == a.iteration_count
        assert np.array_equal(o.primal_solution, a.primal_solution)
        assert np.array_equal(o.dual_source_solution, a.dual_source_solution)
        assert np.array_equal(o.dual_target_solution, a.dual_target_solution)


def test_analytic_identity_permutation(cuda):
    """C = 1 - I with uniform marginals: the optimum moves all mass along the
    diagonal at cost 0."""
    k = 24
    C = np.asfortranarray(1.0 - np.eye(k))
    a = np.full(k, 1.0 / k)
    g = pdot.optimize(pdot.default_parameters(1e-6), pdot.OptimalTransportProblem(C, a, a.copy()))
    assert g.termination_reason == OPTIMAL
    assert _final(g).primal_objective == pytest.approx(0.0, abs=1e-6)
    np.testing.assert_allclose(np.diag(g.primal_solution), a, atol=1e-5)


@pytest.mark.parametrize("precision,cost,m,n", [("f64", "f64", 1000, 700), ("f64", "f64", 2050, 300),
                                                ("f32", "f32", 1000, 700), ("f32", "bf16", 1024, 333),
                                                ("f32", "sqeuclid", 1000, 700)])
def test_staged_and_direct_primal_pass_agree(cuda, precision, cost, m, n):
    """The bulk-copy staged fused pass and the direct-load pass compute the same
    entries; they run different grids (shared memory limits the staged one), so
    their row sums are added in a different order: the early evaluations agree
    to 1e-9 and each variant is bitwise repeatable."""
    rng = np.random.default_rng(m + n)
    xs = rng.uniform(0, 1, (m, 2)).astype(np.float32)
    ys = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    a = rng.uniform(0.1, 1, m)
    b = rng.uniform(0.1, 1, n)
    C = instances.sqeuclid_cost(xs.astype(np.float64), ys.astype(np.float64))
    prob = pdot.OptimalTransportProblem(C if cost != "sqeuclid" else None, a / a.sum(), b / b.sum())
    params = pdot.default_parameters(1e-4, iteration_limit=300)
    kw = {"precision": precision, "cost": cost}
    if cost == "sqeuclid":
        kw["points"] = (xs, ys)
    s1 = pdot.optimize(params, prob, primal_pass="staged", **kw)
    s2 = pdot.optimize(params, prob, primal_pass="staged", **kw)
    d = pdot.optimize(params, prob, primal_pass="direct", **kw)
    assert np.array_equal(s1.primal_solution, s2.primal_solution)
    assert s1.iteration_count == d.iteration_count
    for a_, b_ in zip(s1.iteration_stats[:8], d.iteration_stats[:8]):
        assert a_.restart_used == b_.restart_used
        assert a_.step_size == pytest.approx(b_.step_size, rel=1e-9)
        ca, cb = a_.convergence_information[0], b_.convergence_information[0]
        assert ca.primal_objective == pytest.approx(cb.primal_objective, rel=1e-9, abs=1e-15)
        assert ca.l2_primal_residual == pytest.approx(cb.l2_primal_residual, rel=1e-9)


@pytest.mark.parametrize("m,n", [(1, 5), (7, 5), (300, 129), (1000, 700)])
def test_rounding_matches_oracle_and_is_feasible(cuda, m, n):
    """pdot.rounding (the GPU pass of src/utils_gpu.jl:296-318) against the
    oracle's restatement: same elementwise steps, sums in a different order, so
    entries agree to 1e-12 relative; the result meets the marginals."""
    prob = instances.uniform_sqeuclid(m, n, seed=m)
    out = pdot.optimize(pdot.default_parameters(1e-3), prob)
    Xg = out.primal_solution.copy(order="F")
    Xr = out.primal_solution.copy(order="F")
    pdot.rounding(prob, Xg)
    oracle.rounding(prob, Xr)
    np.testing.assert_allclose(Xg, Xr, rtol=1e-12, atol=1e-18)
    np.testing.assert_allclose(Xg.sum(axis=1), prob.source_distribution, rtol=1e-10, atol=1e-15)
    np.testing.assert_allclose(Xg.sum(axis=0), prob.target_distribution, rtol=1e-10, atol=1e-15)
    # non-negative up to rounding: err_c = b - colsum can round a hair below zero
    assert Xg.min() >= -1e-15


def test_device_cost_builder_matches_host_generator(cuda):
    import torch

    rng = np.random.default_rng(4)
    m, n, d = 333, 222, 3
    xs, ys = rng.uniform(0, 1, (m, d)), rng.uniform(0, 1, (n, d))
    lib = _abi.load()
    dx, dy = torch.from_numpy(xs).to(cuda), torch.from_numpy(ys).to(cuda)
    C = torch.empty((n, m), dtype=torch.float64, device=cuda)
    rc = lib.pdot_sqeuclid_cost_f64(m, n, d, dx.data_ptr(), dy.data_ptr(), 1, C.data_ptr(), None)
    _abi.check(lib, rc, "pdot_sqeuclid_cost_f64")
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy().T, instances.sqeuclid_cost(xs, ys))


def test_caller_output_arrays_receive_the_same_solution(cuda):
    """optimize(out=(X, u, v)) writes the solution into the caller's arrays,
    page-locked (one DMA) or pageable (staged copy), bit for bit what the
    default fresh arrays receive; the arrays are reused across calls."""
    import torch

    prob = instances.uniform_sqeuclid(3000, 2000, seed=4)
    params = pdot.default_parameters(1e-4, iteration_limit=40)
    ref = pdot.optimize(params, prob)
    m, n = 3000, 2000
    pinned = (torch.empty((n, m), dtype=torch.float64, pin_memory=True).numpy().T,
              torch.empty(m, dtype=torch.float64, pin_memory=True).numpy(),
              torch.empty(n, dtype=torch.float64, pin_memory=True).numpy())
    pageable = (np.full((m, n), np.nan, order="F"), np.full(m, np.nan), np.full(n, np.nan))
    for out in (pinned, pageable, pinned):
        res = pdot.optimize(params, prob, out=out)
        assert res.primal_solution is out[0]
        assert res.iteration_count == ref.iteration_count
        assert np.array_equal(out[0], ref.primal_solution)
        assert np.array_equal(out[1], ref.dual_source_solution)
        assert np.array_equal(out[2], ref.dual_target_solution)
