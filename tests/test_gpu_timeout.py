"""The timeout path of the bounded waits, exercised without a fault.

The staged fused pass waits on an mbarrier per ring stage for its own bulk
copies. Every wait polls a bounded number of times; when the bound runs out the
kernel records `kernel_error` in the device state, waits (again bounded) for
the copies it still has in flight, and returns. The host reads the error after
the chunk and fails the call with PDOT_ERR_CUDA.

The `fail_bounded_waits` test hook makes each consumer wait report a timeout
before its first poll, so the path runs deterministically: the copies it
abandons are real ones that do arrive, and the drain must collect them before
the CTA exits. The tests check the reported error and that the context stays
usable for the next solve (no sticky CUDA error, nothing left running).
"""
import pytest

import pdot
from pdot import _abi, instances

pytestmark = pytest.mark.gpu

OPTIMAL = pdot.TerminationReason.TERMINATION_REASON_OPTIMAL


@pytest.mark.parametrize("precision,cost", [("f64", "f64"), ("f32", "f32"), ("f32", "sqeuclid")])
def test_staged_pass_timeout_is_reported_and_context_survives(cuda, precision, cost):
    import numpy as np

    m, n = 300, 200
    rng = np.random.default_rng(3)
    xs = rng.uniform(0, 1, (m, 2)).astype(np.float32)
    ys = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    prob = instances.uniform_sqeuclid(m, n, seed=3)
    kw = {"precision": precision, "cost": cost, "primal_pass": "staged"}
    if cost == "sqeuclid":
        kw["points"] = (xs, ys)
        prob = pdot.OptimalTransportProblem(None, prob.source_distribution, prob.target_distribution)
    params = pdot.default_parameters(1e-4, iteration_limit=50)
    with pytest.raises(_abi.PdotError) as ei:
        pdot.optimize(params, prob, fail_bounded_waits=True, **kw)
    assert ei.value.code == _abi.PDOT_ERR_CUDA
    assert "timed out" in str(ei.value)
    # the same solve without the hook runs normally afterwards
    ok = pdot.optimize(pdot.default_parameters(1e-4), prob, **kw)
    assert ok.termination_reason == OPTIMAL
