"""Argument checks of the Python API that run before any device work (no GPU
needed): shapes of warm starts and race groups, and how the options reach the
C struct."""
import ctypes as ct

import numpy as np
import pytest

import pdot
from pdot import _abi, api, instances


def _probs():
    probs, pts = instances.batched_l1(3, 8, 20, seed=1)
    return probs, pts


def test_batched_warm_start_shape_is_checked():
    probs, pts = _probs()
    m = probs[0].source_distribution.size
    bad = [(np.zeros(m + 1), np.zeros(probs[0].target_distribution.size)), None, None]
    with pytest.raises(ValueError):
        api.optimize_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, warm_starts=bad)


def test_batched_race_groups_need_one_entry_per_instance():
    probs, pts = _probs()
    with pytest.raises(ValueError):
        api.optimize_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, race_groups=[0, 0])


def test_warm_plan_shape_is_checked():
    with pytest.raises(ValueError):
        api._options(0, True, warm_start=(np.zeros(4), np.zeros(3), np.zeros((3, 4))))


def test_recovered_plan_and_warm_start_reach_the_options():
    opts, keep = api._options(0, True, warm_start=(np.ones(4), np.ones(3)), recover_plan=(3e-4, 100))
    assert opts.warm_plan_epsilon == 3e-4 and opts.warm_plan_iterations == 100
    assert bool(opts.warm_dual_source) and bool(opts.warm_dual_target) and not bool(opts.warm_primal)
    assert opts.fail_bounded_waits == 0
    u0 = np.ctypeslib.as_array(opts.warm_dual_source, shape=(4,))
    assert np.all(u0 == 1.0)
    del keep


def test_warm_plan_without_duals_is_rejected_before_device_work(built):
    """The C entry validates options before it touches a device."""
    prob = instances.uniform_sqeuclid(4, 3, seed=0)
    lib = _abi.load()
    mp = api.MarshalledProblem(prob)
    cp = api.marshal_params(pdot.default_parameters(1e-4))
    X0 = np.zeros((4, 3), order="F")
    opts = _abi.SolverOptionsC()
    opts.use_cuda_graph = 1
    opts.warm_primal = X0.ctypes.data_as(ct.POINTER(ct.c_double))
    ob = api.OutputBuffers(4, 3, 16)
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(opts), ct.byref(ob.c))
    assert rc == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert "warm" in _abi.last_error(lib)


def test_timeout_hook_is_validated_before_device_work(built):
    """fail_bounded_waits is 0 or 1; anything else is refused before device work."""
    prob = instances.uniform_sqeuclid(4, 3, seed=0)
    lib = _abi.load()
    mp = api.MarshalledProblem(prob)
    cp = api.marshal_params(pdot.default_parameters(1e-4))
    opts = _abi.SolverOptionsC()
    opts.use_cuda_graph = 1
    opts.fail_bounded_waits = 2
    ob = api.OutputBuffers(4, 3, 16)
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(opts), ct.byref(ob.c))
    assert rc == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert "fail_bounded_waits" in _abi.last_error(lib)


def test_warm_restart_flag_is_validated_before_device_work(built):
    prob = instances.uniform_sqeuclid(4, 3, seed=0)
    lib = _abi.load()
    mp = api.MarshalledProblem(prob)
    cp = api.marshal_params(pdot.default_parameters(1e-4))
    opts = _abi.SolverOptionsC()
    opts.use_cuda_graph = 1
    opts.warm_restart_at_zero = 3
    ob = api.OutputBuffers(4, 3, 16)
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(opts), ct.byref(ob.c))
    assert rc == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert "warm_restart_at_zero" in _abi.last_error(lib)
    with pytest.raises(KeyError):
        api._options(0, True, warm_restart="later")


def test_persistent_chunks_flag_is_validated_before_device_work(built):
    prob = instances.uniform_sqeuclid(4, 3, seed=0)
    lib = _abi.load()
    mp = api.MarshalledProblem(prob)
    cp = api.marshal_params(pdot.default_parameters(1e-4))
    opts = _abi.SolverOptionsC()
    opts.use_cuda_graph = 1
    opts.persistent_chunks = 2
    ob = api.OutputBuffers(4, 3, 16)
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(opts), ct.byref(ob.c))
    assert rc == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert "persistent_chunks" in _abi.last_error(lib)
    assert api._options(0, True)[0].persistent_chunks == 0
    assert api._options(0, True, persistent=True)[0].persistent_chunks == 1
    assert api._options(0, True, persistent=False)[0].persistent_chunks == -1


def test_batch_panel_rows_is_validated_before_device_work(built):
    """The batched solver's tile takes panels of 128 or 256 rows (0: 256)."""
    probs, pts = instances.batched_l1(count=2, lo=8, hi=16, seed=1)
    with pytest.raises(_abi.PdotError) as ei:
        pdot.optimize_batched(pdot.default_parameters(1e-4), probs, cost="l1", points=pts, panel_rows=192)
    assert ei.value.code == _abi.PDOT_ERR_INVALID_ARGUMENT
    assert "batch_panel_rows" in str(ei.value)


def test_caller_output_arrays_are_checked_before_device_work(built):
    prob = instances.uniform_sqeuclid(4, 3, seed=0)
    params = pdot.default_parameters(1e-4)
    good = (np.zeros((4, 3), order="F"), np.zeros(4), np.zeros(3))
    bad = [
        (np.zeros((4, 3), order="C"), good[1], good[2]),          # X row-major
        (np.zeros((3, 4), order="F"), good[1], good[2]),          # X shape
        (np.zeros((4, 3), order="F", dtype=np.float32), good[1], good[2]),
        (good[0], np.zeros(3), good[2]),                          # u size
        (good[0], good[1], np.zeros(4)),                          # v size
        good[:2],
    ]
    for out in bad:
        with pytest.raises(ValueError):
            pdot.optimize(params, prob, out=out)
    ro = np.zeros(4)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        pdot.optimize(params, prob, out=(good[0], ro, good[2]))
