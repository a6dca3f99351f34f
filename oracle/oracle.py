"""Python binding of the CPU oracle (oracle/libpdot_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, as the checker. The product (libpdot.so and the
`pdot` package) never imports this module.

It drives the oracle through the same C structs as libpdot.so (include/pdot.h),
so `optimize` here takes and returns the same Python types as `pdot.optimize`.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpdot_oracle.so")

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    from pdot import _abi

    lib = ct.CDLL(LIB_PATH)
    lib.pdot_oracle_optimize.restype = ct.c_int
    lib.pdot_oracle_optimize.argtypes = [
        ct.POINTER(_abi.ProblemC), ct.POINTER(_abi.PdhgParametersC),
        ct.POINTER(_abi.SaddlePointOutputC), ct.c_int,
    ]
    P = ct.c_void_p
    D = ct.c_double
    lib.pdot_oracle_optimize_warm.restype = ct.c_int
    lib.pdot_oracle_optimize_warm.argtypes = [
        ct.POINTER(_abi.ProblemC), ct.POINTER(_abi.PdhgParametersC), ct.c_void_p, ct.c_void_p, ct.c_void_p,
        ct.c_double, ct.c_int, ct.POINTER(_abi.SaddlePointOutputC), ct.c_int,
    ]
    lib.pdot_oracle_primal_pass.restype = None
    lib.pdot_oracle_primal_pass.argtypes = [
        ct.c_int64, ct.c_int64, P, P, P, P, P, D, D, D, ct.c_int32, P, P, P,
    ]
    lib.pdot_oracle_time_steps.restype = ct.c_int
    lib.pdot_oracle_time_steps.argtypes = [
        ct.POINTER(_abi.ProblemC), ct.POINTER(_abi.PdhgParametersC), ct.c_int, ct.c_int, ct.c_int,
        ct.c_void_p,
    ]
    lib.pdot_oracle_rounding.restype = None
    lib.pdot_oracle_rounding.argtypes = [ct.c_int64, ct.c_int64, P, P, P]
    lib.pdot_oracle_version.restype = ct.c_int
    _lib = lib
    return lib


def optimize(params, problem, num_threads: int = 0):
    """The oracle's PDOT.optimize: same inputs and outputs as pdot.optimize."""
    from pdot import api, _abi

    api.validate(params)
    lib = load()
    mp = api.MarshalledProblem(problem)
    cp = api.marshal_params(params)
    ob = api.OutputBuffers(mp.m, mp.n, api.stats_capacity_for(params))
    rc = lib.pdot_oracle_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(ob.c), int(num_threads))
    if rc != 0:
        raise _abi.PdotError(rc, f"oracle optimize failed ({rc})")
    return ob.to_output()


def optimize_warm(params, problem, u0, v0, X0=None, omega0=0.0, num_threads: int = 0,
                  restart_at_zero: bool = False):
    """The oracle's solve from a warm start (initial duals, optional plan and
    primal weight; the restart information starts at the warm point, or at
    the zero point with `restart_at_zero`)."""
    from pdot import api, _abi

    api.validate(params)
    lib = load()
    mp = api.MarshalledProblem(problem)
    cp = api.marshal_params(params)
    ob = api.OutputBuffers(mp.m, mp.n, api.stats_capacity_for(params))
    u0 = np.ascontiguousarray(u0, dtype=np.float64)
    v0 = np.ascontiguousarray(v0, dtype=np.float64)
    X0p = None
    if X0 is not None:
        X0 = np.asfortranarray(X0, dtype=np.float64)
        X0p = X0.ctypes.data
    rc = lib.pdot_oracle_optimize_warm(ct.byref(mp.c), ct.byref(cp), u0.ctypes.data, v0.ctypes.data, X0p,
                                       float(omega0), int(bool(restart_at_zero)), ct.byref(ob.c),
                                       int(num_threads))
    if rc != 0:
        raise _abi.PdotError(rc, f"oracle optimize failed ({rc})")
    return ob.to_output()


def _p(a: np.ndarray):
    return ct.c_void_p(a.ctypes.data)


def primal_pass(C, X, Xa, u, v, step_over_weight, avg_new_weight, avg_scale, flags):
    """Oracle counterpart of pdot_primal_pass_f64. X and Xa (Fortran order,
    float64) are updated in place; returns (delta_row_sum, delta_col_sum, sq)."""
    lib = load()
    m, n = C.shape
    for arr in (C, X, Xa):
        assert arr.flags.f_contiguous and arr.dtype == np.float64
    drow = np.zeros(m)
    dcol = np.zeros(n)
    dsq = np.zeros(1)
    lib.pdot_oracle_primal_pass(m, n, _p(C), _p(X), _p(Xa), _p(u), _p(v), step_over_weight,
                                avg_new_weight, avg_scale, flags, _p(drow), _p(dcol), _p(dsq))
    return drow, dcol, float(dsq[0])


def time_steps(params, problem, steps: int, num_threads: int = 0, warmup: int = 0):
    """Per-step seconds of `steps` PDHG iterations of the oracle (take_step!
    only), timed after `warmup` untimed iterations in the same state, with
    `num_threads` OpenMP threads (0 = all). Returns a numpy array."""
    from pdot import api, _abi

    lib = load()
    mp = api.MarshalledProblem(problem)
    cp = api.marshal_params(params)
    sec = np.zeros(max(int(steps), 1))
    rc = lib.pdot_oracle_time_steps(ct.byref(mp.c), ct.byref(cp), int(warmup), int(steps), int(num_threads),
                                    sec.ctypes.data)
    if rc != 0:
        raise _abi.PdotError(rc, f"oracle time_steps failed ({rc})")
    return sec[: int(steps)]


def rounding(problem, X):
    """Oracle restatement of the reference's rounding (in place on X)."""
    lib = load()
    assert X.flags.f_contiguous and X.dtype == np.float64
    a = np.ascontiguousarray(problem.source_distribution, dtype=np.float64)
    b = np.ascontiguousarray(problem.target_distribution, dtype=np.float64)
    lib.pdot_oracle_rounding(X.shape[0], X.shape[1], _p(a), _p(b), _p(X))
    return X


def warm_plan(C, a, b, u0, v0, eps: float, rounds: int):
    """The plan recovered from warm duals (csrc/pdot_warmplan.cu), in FP64:
    `rounds` of log-domain balancing from (f, g) = (u0, v0), then
    X = exp((f_i + g_j - C_ij) / eps). Returns (X, f, g)."""
    from scipy.special import logsumexp

    C = np.asarray(C, dtype=np.float64)
    f = np.asarray(u0, dtype=np.float64).copy()
    g = np.asarray(v0, dtype=np.float64).copy()
    la, lb = np.log(a), np.log(b)
    for _ in range(rounds):
        f = eps * (la - logsumexp((g[None, :] - C) / eps, axis=1))
        g = eps * (lb - logsumexp((f[:, None] - C) / eps, axis=0))
    X = np.exp((f[:, None] + g[None, :] - C) / eps)
    return X, f, g
