"""pdot_primal_pass_f64_noalloc: the fused primal pass for callers that cannot
allocate device memory (a host framework that serves its whole memory budget
from its own pool, or a loop that cannot afford cudaMalloc's device
synchronisation). Its scratch is a fixed array inside libpdot.so instead of a
caller workspace; these tests check, through the C ABI, that two calls in a row
give the same results as pdot_primal_pass_f64 with a workspace (the plan and
average bit-exact, the sums to 1e-12 relative like the other parity tests),
that a call allocates no device memory, and that oversize problems are refused.

This file is named to be collected last, so that a run stopping at the first
failure has run every other test already.
"""
import numpy as np
import pytest

from pdot import _abi

pytestmark = pytest.mark.gpu


def _inputs(m, n, seed):
    rng = np.random.default_rng(seed)
    C = rng.uniform(0, 1, (m, n))
    X = np.maximum(rng.uniform(-0.005, 0.01, (m, n)), 0.0)
    Xa = rng.uniform(0, 0.01, (m, n))
    return C, X, Xa, rng.uniform(-0.5, 0.5, m), rng.uniform(-0.5, 0.5, n)


def _dev(a, device):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a.T if a.ndim == 2 else a)).to(device)


def _run(lib, device, inputs, args, noalloc):
    import torch

    C, X, Xa, u, v = inputs
    m, n = C.shape
    dC, dX, dXa, du, dv = (_dev(x, device) for x in (C, X, Xa, u, v))
    drow = torch.zeros(m, dtype=torch.float64, device=device)
    dcol = torch.zeros(n, dtype=torch.float64, device=device)
    dsq = torch.zeros(1, dtype=torch.float64, device=device)
    ptrs = (dC.data_ptr(), dX.data_ptr(), dXa.data_ptr(), du.data_ptr(), dv.data_ptr())
    outs = (drow.data_ptr(), dcol.data_ptr(), dsq.data_ptr())
    torch.cuda.synchronize()
    if noalloc:
        free0 = torch.cuda.mem_get_info(device)[0]
        rc = lib.pdot_primal_pass_f64_noalloc(m, n, *ptrs, *args, *outs, None)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info(device)[0]
    else:
        wsb = lib.pdot_primal_pass_workspace_bytes(m, n)
        ws = torch.empty(wsb // 8 + 1, dtype=torch.float64, device=device)
        rc = lib.pdot_primal_pass_f64(m, n, *ptrs, *args, *outs, ws.data_ptr(), wsb, None)
        torch.cuda.synchronize()
        free0 = free1 = None
    _abi.check(lib, rc, "primal pass")
    return (dX.cpu().numpy().T, dXa.cpu().numpy().T, drow.cpu().numpy(), dcol.cpu().numpy(),
            float(dsq.item()), free0, free1)


def test_noalloc_matches_workspace_entry_on_two_calls(cuda):
    lib = _abi.load()
    cases = [((1000, 700, 1), (0.37, 0.25, 0.8, 0)),
             ((513, 129, 2), (0.5, 1.0, 1.0, _abi.PDOT_PASS_FIRST_AVERAGE))]
    for (m, n, seed), args in cases:  # two calls in a row, reusing the shared scratch
        inputs = _inputs(m, n, seed)
        ref = _run(lib, cuda, inputs, args, noalloc=False)
        got = _run(lib, cuda, inputs, args, noalloc=True)
        assert np.array_equal(got[0], ref[0])
        assert np.array_equal(got[1], ref[1])
        np.testing.assert_allclose(got[2], ref[2], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(got[3], ref[3], rtol=1e-12, atol=1e-15)
        assert got[4] == pytest.approx(ref[4], rel=1e-12, abs=1e-30)


def test_noalloc_call_allocates_nothing(cuda):
    lib = _abi.load()
    inputs = _inputs(300, 200, 3)
    _run(lib, cuda, inputs, (0.4, 0.2, 0.9, 0), noalloc=True)  # first call: address lookup
    for _ in range(2):
        *_, free0, free1 = _run(lib, cuda, inputs, (0.4, 0.2, 0.9, 0), noalloc=True)
        assert free0 == free1


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    """2^17 rows x 4096 columns need 512 x 4096 column partials (16 MiB) plus
    the row partials: more than the fixed scratch. Every buffer is as large as
    the request (three 4 GiB matrices), so a regression of the size check
    would run a valid pass and fail the assertion instead of reading or
    writing out of bounds."""
    import torch

    lib = _abi.load()
    m, n = 1 << 17, 4096
    mats = [torch.empty((n, m), dtype=torch.float64, device=cuda) for _ in range(3)]
    mats[1].zero_()
    mats[2].zero_()
    rows = [torch.zeros(m, dtype=torch.float64, device=cuda) for _ in range(2)]
    cols = [torch.zeros(n, dtype=torch.float64, device=cuda) for _ in range(2)]
    mats[0].fill_(1.0)
    dsq = torch.zeros(1, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    rc = lib.pdot_primal_pass_f64_noalloc(m, n, mats[0].data_ptr(), mats[1].data_ptr(), mats[2].data_ptr(),
                                          rows[0].data_ptr(), cols[0].data_ptr(), 1.0, 1.0, 1.0, 0,
                                          rows[1].data_ptr(), cols[1].data_ptr(), dsq.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == _abi.PDOT_ERR_TOO_LARGE
    assert "scratch" in _abi.last_error(lib)
    del mats
    torch.cuda.empty_cache()
