"""The batched solver's autotuner (pdot.tune_batched) as host logic: its three
stages, each starting from the best configuration so far, with the solver
replaced by a cost model (no GPU)."""
import pdot
from pdot import api


def _fake_solver(cost):
    calls = []

    def optimize_batched(params, problems, **kw):
        cand = {k: kw[k] for k in ("primal_pass", "ctas_per_sm", "panel_rows", "unit_cost") if k in kw}
        if kw.get("persistent"):
            cand["persistent"] = True
        calls.append((cand, params.termination_criteria.iteration_limit))
        return None, cost(cand)

    return optimize_batched, calls


def _run(monkeypatch, cost):
    fake, calls = _fake_solver(cost)
    monkeypatch.setattr(api, "optimize_batched", fake)
    best, timings = pdot.tune_batched(pdot.default_parameters(1e-4), [None], cost="l1", points=[None],
                                      iterations=64)
    return best, timings, calls


def test_three_stages_in_order(monkeypatch):
    # staged at 2 per SM is the best launch configuration, 128-row tiles lose, 8 is the best balance
    def cost(c):
        t = {"staged": 1.0, "direct": 1.5}[c["primal_pass"]] + (0.4 if c.get("persistent") else 0.0)
        t += 0.3 if c["ctas_per_sm"] == 1 else 0.0
        t += 0.2 if c["panel_rows"] == 128 else 0.0
        return t - 0.01 * c["unit_cost"]

    best, timings, calls = _run(monkeypatch, cost)
    n_launch, n_tile = len(api.BATCH_TUNING_CANDIDATES), len(api.BATCH_TILE_SHAPES)
    others = [u for u in api.BATCH_UNIT_COSTS if u != 0.25]
    assert len(timings) == n_launch + n_tile + len(others)
    assert all(limit == 64 for _, limit in calls)  # every candidate times the first iterations only
    # stage 1: every launch configuration with 256-row tiles at the default balance
    assert [t[0]["panel_rows"] for t in timings[:n_launch]] == [256] * n_launch
    assert {t[0]["unit_cost"] for t in timings[:n_launch]} == {0.25}
    assert any(t[0].get("persistent") for t in timings[:n_launch])
    # stage 2: the tiles on top of stage 1's best (staged)
    for cand, _ in timings[n_launch:n_launch + n_tile]:
        assert cand["primal_pass"] == "staged" and cand["panel_rows"] == 128
    # stage 3: the other balances on top of the best so far
    for cand, _ in timings[n_launch + n_tile:]:
        assert cand["primal_pass"] == "staged" and cand["panel_rows"] == 256 and cand["ctas_per_sm"] == 2
    assert best == {"panel_rows": 256, "primal_pass": "staged", "ctas_per_sm": 2, "unit_cost": 8.0}
    assert best == min(timings, key=lambda t: t[1])[0]


def test_later_stages_build_on_a_persistent_or_128_row_winner(monkeypatch):
    # the persistent chunk wins the launch stage and 128-row tiles at 3 per SM win the tile stage
    def cost(c):
        t = 1.0 if c.get("persistent") else 2.0
        t -= 0.5 if (c["panel_rows"], c["ctas_per_sm"]) == (128, 3) else 0.0
        return t + (0.1 if c["unit_cost"] != 0.5 else 0.0)

    best, timings, _ = _run(monkeypatch, cost)
    n_launch, n_tile = len(api.BATCH_TUNING_CANDIDATES), len(api.BATCH_TILE_SHAPES)
    for cand, _ in timings[n_launch:]:
        assert cand.get("persistent") and cand["primal_pass"] == "direct"
    for cand, _ in timings[n_launch + n_tile:]:
        assert (cand["panel_rows"], cand["ctas_per_sm"]) == (128, 3)
    assert best["persistent"] and best["panel_rows"] == 128 and best["unit_cost"] == 0.5
