"""Host-side mirror of the reference's Julia API, over the C ABI of libpdot.so.

Names, argument meaning and error behaviour follow MIT-Lu-Lab/PDOT.jl:

    OptimalTransportProblem                src/io.jl:1-5
    AdaptiveStepsizeParams / Constant...   src/solver_gpu.jl:2-7
    PdhgParameters                         src/solver_gpu.jl:9-21
    TerminationCriteria, OptimalityNorm    src/termination.jl:2-69
    RestartParameters, RestartScheme, ...  src/saddle_point_gpu.jl:401-472
    ConvergenceInformation, IterationStats,
    RestartChoice, PointType,
    TerminationReason, SolveLog            src/solve_log.jl
    SaddlePointOutput                      src/saddle_point_gpu.jl:2-34
    optimize(params, problem)              src/solver_gpu.jl:413-720

`optimize` runs on the GPU through libpdot.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import enum
import math
from dataclasses import dataclass, field
from typing import Optional, Union

import numpy as np

from . import _abi

INT32_MAX = 2**31 - 1


# ---------------------------------------------------------------- enums
class OptimalityNorm(enum.IntEnum):  # src/termination.jl:2
    L_INF = 0
    L_2 = 1


class RestartScheme(enum.IntEnum):  # src/saddle_point_gpu.jl:401
    NO_RESTARTS = 0
    FIXED_FREQUENCY = 1
    ADAPTIVE_KKT = 2


class RestartToCurrentMetric(enum.IntEnum):  # src/saddle_point_gpu.jl:408
    NO_RESTART_TO_CURRENT = 0
    KKT_GREEDY = 1


class RestartChoice(enum.IntEnum):  # src/solve_log.jl:15-20
    RESTART_CHOICE_UNSPECIFIED = 0
    RESTART_CHOICE_NO_RESTART = 1
    RESTART_CHOICE_WEIGHTED_AVERAGE_RESET = 2
    RESTART_CHOICE_RESTART_TO_AVERAGE = 3


class PointType(enum.IntEnum):  # src/solve_log.jl:35-41
    POINT_TYPE_UNSPECIFIED = 0
    POINT_TYPE_CURRENT_ITERATE = 1
    POINT_TYPE_ITERATE_DIFFERENCE = 2
    POINT_TYPE_AVERAGE_ITERATE = 3
    POINT_TYPE_NONE = 4


class TerminationReason(enum.IntEnum):  # src/solve_log.jl:245-254
    TERMINATION_REASON_UNSPECIFIED = 0
    TERMINATION_REASON_OPTIMAL = 1
    TERMINATION_REASON_TIME_LIMIT = 2
    TERMINATION_REASON_ITERATION_LIMIT = 3
    TERMINATION_REASON_KKT_MATRIX_PASS_LIMIT = 4
    TERMINATION_REASON_NUMERICAL_ERROR = 5
    TERMINATION_REASON_INVALID_PROBLEM = 6
    TERMINATION_REASON_OTHER = 7


L_INF = OptimalityNorm.L_INF
L_2 = OptimalityNorm.L_2
NO_RESTARTS = RestartScheme.NO_RESTARTS
FIXED_FREQUENCY = RestartScheme.FIXED_FREQUENCY
ADAPTIVE_KKT = RestartScheme.ADAPTIVE_KKT
NO_RESTART_TO_CURRENT = RestartToCurrentMetric.NO_RESTART_TO_CURRENT
KKT_GREEDY = RestartToCurrentMetric.KKT_GREEDY


def termination_reason_to_string(reason: TerminationReason) -> str:
    """src/termination.jl:168-171: strip the TERMINATION_REASON_ prefix."""
    return TerminationReason(reason).name[len("TERMINATION_REASON_"):]


# ---------------------------------------------------------------- problem
@dataclass
class OptimalTransportProblem:
    """src/io.jl:1-5. cost_matrix is m x n (sources x targets)."""

    cost_matrix: np.ndarray
    source_distribution: np.ndarray
    target_distribution: np.ndarray


# ---------------------------------------------------------------- parameters
@dataclass
class AdaptiveStepsizeParams:  # src/solver_gpu.jl:2-5
    reduction_exponent: float
    growth_exponent: float


@dataclass
class ConstantStepsizeParams:  # src/solver_gpu.jl:7
    pass


@dataclass
class TerminationCriteria:  # src/termination.jl:5-51
    optimality_norm: OptimalityNorm
    eps_optimal_absolute: float
    eps_optimal_relative: float
    time_sec_limit: float
    iteration_limit: int
    kkt_matrix_pass_limit: float


def construct_termination_criteria(
    *,
    optimality_norm=L_2,
    eps_optimal_absolute,
    eps_optimal_relative,
    time_sec_limit=math.inf,
    iteration_limit=INT32_MAX,
    kkt_matrix_pass_limit=math.inf,
) -> TerminationCriteria:
    """src/termination.jl:53-69 (keyword-only, same defaults)."""
    return TerminationCriteria(
        OptimalityNorm(optimality_norm),
        float(eps_optimal_absolute),
        float(eps_optimal_relative),
        float(time_sec_limit),
        int(iteration_limit),
        float(kkt_matrix_pass_limit),
    )


@dataclass
class RestartParameters:  # src/saddle_point_gpu.jl:411-441
    restart_scheme: RestartScheme
    restart_to_current_metric: RestartToCurrentMetric
    restart_frequency_if_fixed: int
    artificial_restart_threshold: float
    sufficient_reduction_for_restart: float
    necessary_reduction_for_restart: float
    primal_weight_update_smoothing: float


def construct_restart_parameters(
    restart_scheme,
    restart_to_current_metric,
    restart_frequency_if_fixed: int,
    artificial_restart_threshold: float,
    sufficient_reduction_for_restart: float,
    necessary_reduction_for_restart: float,
    primal_weight_update_smoothing: float,
) -> RestartParameters:
    """src/saddle_point_gpu.jl:446-472, including its assertions."""
    assert restart_frequency_if_fixed > 1
    assert 0.0 < artificial_restart_threshold <= 1.0
    assert 0.0 < sufficient_reduction_for_restart <= necessary_reduction_for_restart <= 1.0
    assert 0.0 <= primal_weight_update_smoothing <= 1.0
    return RestartParameters(
        RestartScheme(restart_scheme),
        RestartToCurrentMetric(restart_to_current_metric),
        int(restart_frequency_if_fixed),
        float(artificial_restart_threshold),
        float(sufficient_reduction_for_restart),
        float(necessary_reduction_for_restart),
        float(primal_weight_update_smoothing),
    )


@dataclass
class PdhgParameters:  # src/solver_gpu.jl:9-21
    primal_importance: float
    scale_invariant_initial_primal_weight: bool
    verbosity: int
    record_iteration_stats: bool
    termination_evaluation_frequency: int
    termination_criteria: TerminationCriteria
    restart_params: RestartParameters
    step_size_policy_params: Union[AdaptiveStepsizeParams, ConstantStepsizeParams]


# ---------------------------------------------------------------- output
@dataclass
class ConvergenceInformation:  # src/solve_log.jl:47-151
    candidate_type: PointType = PointType.POINT_TYPE_UNSPECIFIED
    primal_objective: float = 0.0
    dual_objective: float = 0.0
    corrected_dual_objective: float = 0.0
    l_inf_primal_residual: float = 0.0
    l2_primal_residual: float = 0.0
    l_inf_dual_residual: float = 0.0
    l2_dual_residual: float = 0.0
    relative_l_inf_primal_residual: float = 0.0
    relative_l2_primal_residual: float = 0.0
    relative_l_inf_dual_residual: float = 0.0
    relative_l2_dual_residual: float = 0.0
    relative_optimality_gap: float = 0.0
    l_inf_primal_variable: float = 0.0
    l2_primal_variable: float = 0.0
    l_inf_dual_variable: float = 0.0
    l2_dual_variable: float = 0.0


@dataclass
class IterationStats:  # src/solve_log.jl:154-228
    iteration_number: int = 0
    convergence_information: list = field(default_factory=list)
    cumulative_kkt_matrix_passes: float = 0.0
    cumulative_rejected_steps: int = 0
    cumulative_time_sec: float = 0.0
    restart_used: RestartChoice = RestartChoice.RESTART_CHOICE_UNSPECIFIED
    step_size: float = 0.0
    primal_weight: float = 0.0
    method_specific_stats: dict = field(default_factory=dict)


@dataclass
class SaddlePointOutput:  # src/saddle_point_gpu.jl:2-34
    primal_solution: np.ndarray
    dual_source_solution: np.ndarray
    dual_target_solution: np.ndarray
    termination_reason: TerminationReason
    termination_string: str
    iteration_count: int
    iteration_stats: list


@dataclass
class SolveLog:  # src/solve_log.jl:256-327
    instance_name: str = ""
    command_line_invocation: str = ""
    termination_reason: TerminationReason = TerminationReason.TERMINATION_REASON_UNSPECIFIED
    termination_string: str = ""
    iteration_count: int = 0
    solve_time_sec: float = 0.0
    solution_stats: IterationStats = field(default_factory=IterationStats)
    solution_type: PointType = PointType.POINT_TYPE_UNSPECIFIED
    iteration_stats: list = field(default_factory=list)


# ---------------------------------------------------------------- marshalling
def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ct.POINTER(ct.c_double))


def marshal_params(params: PdhgParameters) -> _abi.PdhgParametersC:
    tc, rp = params.termination_criteria, params.restart_params
    c = _abi.PdhgParametersC()
    c.primal_importance = float(params.primal_importance)
    c.scale_invariant_initial_primal_weight = int(bool(params.scale_invariant_initial_primal_weight))
    c.verbosity = int(params.verbosity)
    c.record_iteration_stats = int(bool(params.record_iteration_stats))
    c.termination_evaluation_frequency = int(params.termination_evaluation_frequency)
    c.termination_criteria.optimality_norm = int(tc.optimality_norm)
    c.termination_criteria.eps_optimal_absolute = float(tc.eps_optimal_absolute)
    c.termination_criteria.eps_optimal_relative = float(tc.eps_optimal_relative)
    c.termination_criteria.time_sec_limit = float(tc.time_sec_limit)
    c.termination_criteria.iteration_limit = int(min(tc.iteration_limit, INT32_MAX))
    c.termination_criteria.kkt_matrix_pass_limit = float(tc.kkt_matrix_pass_limit)
    c.restart_params.restart_scheme = int(rp.restart_scheme)
    c.restart_params.restart_to_current_metric = int(rp.restart_to_current_metric)
    c.restart_params.restart_frequency_if_fixed = int(rp.restart_frequency_if_fixed)
    c.restart_params.artificial_restart_threshold = float(rp.artificial_restart_threshold)
    c.restart_params.sufficient_reduction_for_restart = float(rp.sufficient_reduction_for_restart)
    c.restart_params.necessary_reduction_for_restart = float(rp.necessary_reduction_for_restart)
    c.restart_params.primal_weight_update_smoothing = float(rp.primal_weight_update_smoothing)
    sp = params.step_size_policy_params
    if isinstance(sp, AdaptiveStepsizeParams):
        c.step_size_policy = 0
        c.reduction_exponent = float(sp.reduction_exponent)
        c.growth_exponent = float(sp.growth_exponent)
    elif isinstance(sp, ConstantStepsizeParams):
        c.step_size_policy = 1
    else:
        raise TypeError("step_size_policy_params must be AdaptiveStepsizeParams or ConstantStepsizeParams")
    return c


class MarshalledProblem:
    """Keeps the column-major host arrays alive for the duration of a call.
    A problem whose cost comes from coordinates may have cost_matrix None."""

    def __init__(self, problem: OptimalTransportProblem):
        self.a = np.ascontiguousarray(problem.source_distribution, dtype=np.float64).ravel()
        self.b = np.ascontiguousarray(problem.target_distribution, dtype=np.float64).ravel()
        m, n = self.a.shape[0], self.b.shape[0]
        if problem.cost_matrix is None:
            self.C = None
            cptr = None
        else:
            C = np.asarray(problem.cost_matrix, dtype=np.float64)
            if C.ndim != 2:
                raise ValueError("cost_matrix must be a matrix")
            self.C = np.asfortranarray(C)
            if self.C.shape != (m, n):
                raise ValueError("distribution lengths must match the cost matrix shape")
            cptr = _dptr(self.C)
        self.m, self.n = m, n
        self.c = _abi.ProblemC(m, n, cptr, _dptr(self.a), _dptr(self.b))


def stats_from_c(s: _abi.IterationStatsC) -> IterationStats:
    ci = ConvergenceInformation(PointType(s.convergence_information.candidate_type))
    for f in _abi.CONVERGENCE_FIELDS:
        setattr(ci, f, getattr(s.convergence_information, f))
    return IterationStats(
        iteration_number=s.iteration_number,
        convergence_information=[ci],
        cumulative_kkt_matrix_passes=s.cumulative_kkt_matrix_passes,
        cumulative_rejected_steps=s.cumulative_rejected_steps,
        cumulative_time_sec=s.cumulative_time_sec,
        restart_used=RestartChoice(s.restart_used),
        step_size=s.step_size,
        primal_weight=s.primal_weight,
        method_specific_stats={"time_spent_doing_basic_algorithm": s.time_spent_doing_basic_algorithm},
    )


def _check_out(out, m: int, n: int):
    """The caller's (X, u, v) output arrays: FP64, X m x n column-major, u of
    m and v of n entries, contiguous and writeable."""
    if len(out) != 3:
        raise ValueError("out must be (X, u, v)")
    X, u, v = out
    for name, arr, shape in (("X", X, (m, n)), ("u", u, (m,)), ("v", v, (n,))):
        if not isinstance(arr, np.ndarray) or arr.dtype != np.float64 or arr.shape != shape:
            raise ValueError(f"out {name} must be a float64 array of shape {shape}")
        if not arr.flags.writeable or not (arr.flags.f_contiguous if name == "X" else arr.flags.c_contiguous):
            raise ValueError(f"out {name} must be writeable and {'column-major' if name == 'X' else 'contiguous'}")
    return X, u, v


class OutputBuffers:
    def __init__(self, m: int, n: int, stats_capacity: int, out=None):
        if out is not None:
            self.X, self.u, self.v = _check_out(out, m, n)
        else:
            self.X = np.zeros((m, n), dtype=np.float64, order="F")
            self.u = np.zeros(m, dtype=np.float64)
            self.v = np.zeros(n, dtype=np.float64)
        self.stats = (_abi.IterationStatsC * max(stats_capacity, 1))()
        self.c = _abi.SaddlePointOutputC()
        self.c.primal_solution = _dptr(self.X)
        self.c.dual_source_solution = _dptr(self.u)
        self.c.dual_target_solution = _dptr(self.v)
        self.c.iteration_stats = ct.cast(self.stats, ct.POINTER(_abi.IterationStatsC))
        self.c.iteration_stats_capacity = stats_capacity

    def to_output(self) -> SaddlePointOutput:
        cnt = min(self.c.iteration_stats_count, self.c.iteration_stats_capacity)
        stats = [stats_from_c(self.stats[k]) for k in range(cnt)]
        if self.c.iteration_stats_count > cnt or cnt == 0:
            # Records beyond the buffer are dropped, but the final one is kept.
            stats.append(stats_from_c(self.c.final_stats))
        reason = TerminationReason(self.c.termination_reason)
        return SaddlePointOutput(
            self.X, self.u, self.v, reason, termination_reason_to_string(reason),
            int(self.c.iteration_count), stats,
        )


def stats_capacity_for(params: PdhgParameters, cap: int = 1 << 16) -> int:
    lim = params.termination_criteria.iteration_limit
    freq = max(int(params.termination_evaluation_frequency), 1)
    return int(min(cap, lim // freq + 16))


def validate(params: PdhgParameters) -> None:
    """Raise where the reference raises: src/solver_gpu.jl:420-422."""
    if params.primal_importance <= 0 or not math.isfinite(params.primal_importance):
        raise ValueError("primal_importance must be positive and finite")


# ---------------------------------------------------------------- optimize
_PRECISIONS = {"f64": _abi.PRECISION_F64, "f32": _abi.PRECISION_F32}
_COSTS = {"f64": _abi.COST_F64, "f32": _abi.COST_F32, "bf16": _abi.COST_BF16,
          "sqeuclid": _abi.COST_SQEUCLID_POINTS, "l1": _abi.COST_L1_POINTS}


def _options(device: int, use_cuda_graph: bool, time_kernels: bool = False, *, precision: str = "f64",
             cost: Optional[str] = None, points=None, cost_scale: Optional[float] = None, warm_start=None,
             device_pointers: bool = False, primal_pass: str = "auto", recover_plan=None,
             fail_bounded_waits: bool = False, warm_primal_weight: Optional[float] = None,
             warm_restart: str = "warm", persistent: Optional[bool] = None):
    """Build pdot_solver_options. Returns (options, objects to keep alive).

    precision  "f64" (the drop-in) or "f32" (mixed precision: FP32 plan)
    cost       "f64", "f32", "bf16", "sqeuclid" or "l1" (from `points`); defaults to
               "f64" for an FP64 plan and "f32" for an FP32 plan
    points     (xs, ys) coordinate arrays (m x d, n x d) for "sqeuclid"; with
               device_pointers, (xs_ptr, ys_ptr, d)
    warm_start (u0, v0) initial duals, or (u0, v0, X0) with an initial plan
               (m x n); with device_pointers, (u_ptr, v_ptr[, X_ptr])
    recover_plan  (eps, rounds): with warm duals and no plan, the plan is
               recovered from the duals by `rounds` of log-domain balancing
               of exp((u_i + v_j - C_ij) / eps)
    fail_bounded_waits  test hook: the staged pass's waits report a timeout at
               once (the call then fails with PDOT_ERR_CUDA)
    warm_primal_weight  with a warm start: the initial primal weight (None:
               primal_importance, or the scale-invariant choice)
    warm_restart  with a warm start, where the restart information starts:
               "warm" (the warm point, as the reference's starts at its initial
               point) or "zero" (the zero point, as a cold start's)
    persistent  regular chunks as one persistent cooperative launch: None
               automatic (the CUDA graph, faster on B200), True whenever
               available, False never
    """
    keep = []
    opts = _abi.SolverOptionsC()
    opts.device = device
    opts.use_cuda_graph = 1 if use_cuda_graph else 0
    opts.time_kernels = 1 if time_kernels else 0
    opts.plan_precision = _PRECISIONS[precision]
    if cost is None:
        cost = "f64" if precision == "f64" else "f32"
    opts.cost_storage = _COSTS[cost]
    opts.fail_bounded_waits = 1 if fail_bounded_waits else 0
    opts.warm_primal_weight = float(warm_primal_weight) if warm_primal_weight else 0.0
    opts.warm_restart_at_zero = {"warm": 0, "zero": 1}[warm_restart]
    opts.persistent_chunks = {None: 0, True: 1, False: -1}[persistent]
    if recover_plan is not None:
        opts.warm_plan_epsilon = float(recover_plan[0])
        opts.warm_plan_iterations = int(recover_plan[1])
    if points is None and cost in ("sqeuclid", "l1"):
        return opts, keep  # coordinates supplied per instance by the batched entry
    opts.primal_pass = {"auto": _abi.PASS_AUTO, "staged": _abi.PASS_STAGED, "direct": _abi.PASS_DIRECT}[primal_pass]
    if cost in ("sqeuclid", "l1"):
        if device_pointers:
            xs_ptr, ys_ptr, dim = points
            opts.source_points = ct.cast(ct.c_void_p(xs_ptr), ct.POINTER(ct.c_float))
            opts.target_points = ct.cast(ct.c_void_p(ys_ptr), ct.POINTER(ct.c_float))
        else:
            xs = np.ascontiguousarray(points[0], dtype=np.float32)
            ys = np.ascontiguousarray(points[1], dtype=np.float32)
            if xs.ndim == 1:
                xs, ys = xs[:, None], ys[:, None]
            dim = xs.shape[1]
            keep += [xs, ys]
            opts.source_points = xs.ctypes.data_as(ct.POINTER(ct.c_float))
            opts.target_points = ys.ctypes.data_as(ct.POINTER(ct.c_float))
        opts.point_dim = int(dim)
        opts.cost_scale = float(cost_scale) if cost_scale else 0.0
    if warm_start is not None:
        if device_pointers:
            opts.warm_dual_source = ct.cast(ct.c_void_p(warm_start[0]), ct.POINTER(ct.c_double))
            opts.warm_dual_target = ct.cast(ct.c_void_p(warm_start[1]), ct.POINTER(ct.c_double))
            if len(warm_start) > 2 and warm_start[2]:
                opts.warm_primal = ct.cast(ct.c_void_p(warm_start[2]), ct.POINTER(ct.c_double))
        else:
            u0 = np.ascontiguousarray(warm_start[0], dtype=np.float64)
            v0 = np.ascontiguousarray(warm_start[1], dtype=np.float64)
            keep += [u0, v0]
            opts.warm_dual_source = _dptr(u0)
            opts.warm_dual_target = _dptr(v0)
            if len(warm_start) > 2 and warm_start[2] is not None:
                X0 = np.asfortranarray(warm_start[2], dtype=np.float64)
                if X0.shape != (u0.shape[0], v0.shape[0]):
                    raise ValueError(f"warm-start plan shape {X0.shape} != {(u0.shape[0], v0.shape[0])}")
                keep.append(X0)
                opts.warm_primal = _dptr(X0)
    return opts, keep


def optimize(params: PdhgParameters, problem: OptimalTransportProblem, *, device: int = 0,
             use_cuda_graph: bool = True, precision: str = "f64", cost: Optional[str] = None, points=None,
             cost_scale: Optional[float] = None, warm_start=None, primal_pass: str = "auto",
             recover_plan=None, fail_bounded_waits: bool = False,
             warm_primal_weight: Optional[float] = None, warm_restart: str = "warm",
             persistent: Optional[bool] = None, out=None) -> SaddlePointOutput:
    """PDOT.optimize, src/solver_gpu.jl:413-720, run by libpdot.so on the GPU.

    The keyword options beyond `device` select this implementation's mixed
    precision (FP32 plan; FP32/BF16/coordinate cost), a warm start from
    given duals (and plan) and how regular chunks launch (`persistent`, see
    _options); the defaults are the FP64 drop-in. `out` = (X, u, v) are the
    caller's arrays for the solution (float64; X m x n column-major), as the
    C ABI's output pointers are: reused across calls they save the allocation
    and first touch of fresh arrays, and page-locked ones (a pinned torch
    tensor's numpy view) receive the plan by one DMA."""
    validate(params)
    lib = _abi.load()
    mp = MarshalledProblem(problem)
    cp = marshal_params(params)
    opts, _keep = _options(device, use_cuda_graph, precision=precision, cost=cost, points=points,
                           cost_scale=cost_scale, warm_start=warm_start, primal_pass=primal_pass,
                           recover_plan=recover_plan, fail_bounded_waits=fail_bounded_waits,
                           warm_primal_weight=warm_primal_weight, warm_restart=warm_restart,
                           persistent=persistent)
    ob = OutputBuffers(mp.m, mp.n, stats_capacity_for(params), out=out)
    rc = lib.pdot_optimize(ct.byref(mp.c), ct.byref(cp), ct.byref(opts), ct.byref(ob.c))
    _abi.check(lib, rc, "pdot_optimize")
    return ob.to_output()


class Solver:
    """A problem resident on the GPU plus the state of optimize()'s loop
    (pdot_solver in include/pdot.h). `problem` is an OptimalTransportProblem
    (copied to the device), or `device_problem` a tuple (m, n, cost_ptr,
    source_ptr, target_ptr) of device pointers read in place."""

    def __init__(self, params: PdhgParameters, problem: Optional[OptimalTransportProblem] = None, *,
                 device_problem=None, device: int = 0, use_cuda_graph: bool = True,
                 time_kernels: bool = False, precision: str = "f64", cost: Optional[str] = None,
                 points=None, cost_scale: Optional[float] = None, warm_start=None, primal_pass: str = "auto",
                 recover_plan=None, warm_primal_weight: Optional[float] = None, warm_restart: str = "warm",
                 persistent: Optional[bool] = None):
        validate(params)
        self._lib = _abi.load()
        self._params = params
        self._cp = marshal_params(params)
        opts, self._keep = _options(device, use_cuda_graph, time_kernels, precision=precision, cost=cost,
                                    points=points, cost_scale=cost_scale, warm_start=warm_start,
                                    device_pointers=device_problem is not None, primal_pass=primal_pass,
                                    recover_plan=recover_plan, warm_primal_weight=warm_primal_weight,
                                    warm_restart=warm_restart, persistent=persistent)
        handle = ct.c_void_p()
        if device_problem is not None:
            m, n, cptr, aptr, bptr = device_problem
            pc = _abi.ProblemC(m, n, ct.cast(ct.c_void_p(cptr or 0), ct.POINTER(ct.c_double)),
                               ct.cast(ct.c_void_p(aptr), ct.POINTER(ct.c_double)),
                               ct.cast(ct.c_void_p(bptr), ct.POINTER(ct.c_double)))
            rc = self._lib.pdot_solver_create_device(ct.byref(pc), ct.byref(self._cp), ct.byref(opts),
                                                     ct.byref(handle))
            self.m, self.n = m, n
        else:
            mp = MarshalledProblem(problem)
            rc = self._lib.pdot_solver_create(ct.byref(mp.c), ct.byref(self._cp), ct.byref(opts),
                                              ct.byref(handle))
            self.m, self.n = mp.m, mp.n
        _abi.check(self._lib, rc, "pdot_solver_create")
        self._h = handle

    def reset(self) -> None:
        _abi.check(self._lib, self._lib.pdot_solver_reset(self._h), "pdot_solver_reset")

    def iterate(self, iterations: int) -> dict:
        st = _abi.SolverStatusC()
        _abi.check(self._lib, self._lib.pdot_solver_iterate(self._h, int(iterations), ct.byref(st)),
                   "pdot_solver_iterate")
        return {f: getattr(st, f) for f, _ in st._fields_}

    def finish(self) -> SaddlePointOutput:
        ob = OutputBuffers(self.m, self.n, stats_capacity_for(self._params))
        _abi.check(self._lib, self._lib.pdot_solver_finish(self._h, ct.byref(ob.c)), "pdot_solver_finish")
        return ob.to_output()

    @property
    def stream(self) -> int:
        return int(self._lib.pdot_solver_stream(self._h) or 0)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.pdot_solver_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def optimize_batched(params: PdhgParameters, problems, *, cost: str = "f32", points=None, device: int = 0,
                     use_cuda_graph: bool = True, ctas_per_sm: int = 0, warm_starts=None,
                     return_primal: bool = True, recover_plan=None, race_groups=None,
                     primal_pass: str = "auto", warm_primal_weights=None, unit_cost: float = 0.25,
                     warm_restart: str = "warm", panel_rows: int = 256, persistent: bool = False):
    """Solve many independent instances at once (pdot_optimize_batched).

    problems     a list of OptimalTransportProblem (cost_matrix may be None for
                 coordinate costs)
    cost         "f32" (each FP64 matrix stored in FP32), "sqeuclid" or "l1"
                 (from `points`, a list of (xs, ys) per instance)
    warm_starts  None, or per instance None / (u0, v0) / (u0, v0, X0)
    recover_plan (eps, rounds): plans recovered from the warm duals of the
                 instances given no plan (see _options)
    race_groups  None, or a group id per instance (-1: none): once an
                 instance ends optimal, the rest of its group stop (reason OTHER)
    primal_pass  "auto" (staged for coordinate costs), "staged" or "direct"
    warm_primal_weights  None, or per instance the initial primal weight of its
                 warm start (<= 0: the parameters' choice)
    warm_restart "warm" or "zero": where warm instances start their restart
                 information (see _options)
    unit_cost    the matrix passes cut the active units into CTA ranges of
                 equal cost, a unit costing its rows + unit_cost * 256 (0..8,
                 in eighths); tune_batched picks it
    panel_rows   the matrix passes' tile: a unit is one column of a panel of
                 256 or 128 rows (128: fewer registers per thread, three
                 resident CTAs per SM, twice the units of tall instances);
                 tune_batched picks it
    persistent   True: every regular chunk of loop bodies (the evaluation,
                 the compaction and the steps up to the next evaluation) runs
                 as one persistent cooperative launch with grid barriers
                 between the phases, with the direct primal pass; the results
                 are bit-identical to the CUDA graph of launches (False)
    return_primal  False leaves every primal_solution None (no m x n copies)
    Returns (outputs, seconds): a SaddlePointOutput per instance (its
    iteration_stats holds the final evaluation record) and the device time.
    """
    validate(params)
    lib = _abi.load()
    B = len(problems)
    keep = []
    rows = (ct.c_int64 * B)()
    cols = (ct.c_int64 * B)()
    costs = (ct.c_void_p * B)()
    srcs = (ct.c_void_p * B)()
    tgts = (ct.c_void_p * B)()
    xs_p = (ct.c_void_p * B)()
    ys_p = (ct.c_void_p * B)()
    outs = (_abi.BatchOutputC * B)()
    wu = (ct.c_void_p * B)()
    wv = (ct.c_void_p * B)()
    wx = (ct.c_void_p * B)()
    results = []
    dim = 0
    for k, prob in enumerate(problems):
        a = np.ascontiguousarray(prob.source_distribution, dtype=np.float64)
        b = np.ascontiguousarray(prob.target_distribution, dtype=np.float64)
        m, n = a.shape[0], b.shape[0]
        rows[k], cols[k] = m, n
        srcs[k], tgts[k] = a.ctypes.data, b.ctypes.data
        keep += [a, b]
        if cost == "f32":
            C = np.asfortranarray(prob.cost_matrix, dtype=np.float64)
            if C.shape != (m, n):
                raise ValueError(f"instance {k}: cost matrix shape {C.shape} != {(m, n)}")
            costs[k] = C.ctypes.data
            keep.append(C)
        else:
            xs = np.ascontiguousarray(points[k][0], dtype=np.float32)
            ys = np.ascontiguousarray(points[k][1], dtype=np.float32)
            if xs.ndim == 1:
                xs, ys = xs[:, None], ys[:, None]
            dim = xs.shape[1]
            xs_p[k], ys_p[k] = xs.ctypes.data, ys.ctypes.data
            keep += [xs, ys]
        if warm_starts is not None and warm_starts[k] is not None:
            w = warm_starts[k]
            u0 = np.ascontiguousarray(w[0], dtype=np.float64)
            v0 = np.ascontiguousarray(w[1], dtype=np.float64)
            if u0.shape != (m,) or v0.shape != (n,):
                raise ValueError(f"instance {k}: warm-start dual shapes {u0.shape}, {v0.shape}")
            wu[k], wv[k] = u0.ctypes.data, v0.ctypes.data
            keep += [u0, v0]
            if len(w) > 2 and w[2] is not None:
                X0 = np.asfortranarray(w[2], dtype=np.float64)
                if X0.shape != (m, n):
                    raise ValueError(f"instance {k}: warm-start plan shape {X0.shape} != {(m, n)}")
                wx[k] = X0.ctypes.data
                keep.append(X0)
        X = np.zeros((m, n), order="F") if return_primal else None
        u = np.zeros(m)
        v = np.zeros(n)
        if X is not None:
            outs[k].primal_solution = _dptr(X)
        outs[k].dual_source_solution = _dptr(u)
        outs[k].dual_target_solution = _dptr(v)
        results.append((X, u, v))
    bp = _abi.BatchProblemC()
    bp.num_instances = B
    bp.num_rows = rows
    bp.num_cols = cols
    bp.source_distributions = srcs
    bp.target_distributions = tgts
    if cost == "f32":
        bp.cost_matrices = costs
    else:
        bp.source_points = xs_p
        bp.target_points = ys_p
    if race_groups is not None:
        rg = np.ascontiguousarray(race_groups, dtype=np.int32)
        if rg.shape != (B,):
            raise ValueError("race_groups needs one entry per instance")
        keep.append(rg)
        bp.race_groups = rg.ctypes.data_as(ct.POINTER(ct.c_int32))
    if warm_starts is not None:
        bp.warm_dual_sources = wu
        bp.warm_dual_targets = wv
        bp.warm_primals = wx
    if warm_primal_weights is not None:
        wo = np.ascontiguousarray(warm_primal_weights, dtype=np.float64)
        if wo.shape != (B,):
            raise ValueError("warm_primal_weights needs one entry per instance")
        keep.append(wo)
        bp.warm_primal_weights = _dptr(wo)
    opts, _k = _options(device, use_cuda_graph, precision="f32", cost=cost, recover_plan=recover_plan,
                        warm_restart=warm_restart)
    if cost != "f32":
        opts.point_dim = dim
    opts.ctas_per_sm = int(ctas_per_sm)
    opts.batch_unit_cost = float(unit_cost)
    opts.batch_panel_rows = int(panel_rows)
    opts.persistent_chunks = 1 if persistent else 0
    opts.primal_pass = {"auto": _abi.PASS_AUTO, "staged": _abi.PASS_STAGED, "direct": _abi.PASS_DIRECT}[primal_pass]
    cp = marshal_params(params)
    sec = ct.c_double(0.0)
    rc = lib.pdot_optimize_batched(ct.byref(bp), ct.byref(cp), ct.byref(opts), outs, ct.byref(sec))
    _abi.check(lib, rc, "pdot_optimize_batched")
    out = []
    for k, (X, u, v) in enumerate(results):
        reason = TerminationReason(outs[k].termination_reason)
        out.append(SaddlePointOutput(X, u, v, reason, termination_reason_to_string(reason),
                                     int(outs[k].iteration_count), [stats_from_c(outs[k].final_stats)]))
    return out, sec.value


BATCH_TUNING_CANDIDATES = ([{"primal_pass": pp, "ctas_per_sm": c} for pp in ("staged", "direct") for c in (2, 1)]
                           + [{"primal_pass": "direct", "ctas_per_sm": 2, "persistent": True}])
BATCH_TILE_SHAPES = ({"panel_rows": 128, "ctas_per_sm": 3}, {"panel_rows": 128, "ctas_per_sm": 2})
BATCH_UNIT_COSTS = (0.0, 0.125, 0.25, 0.5, 8.0)


def tune_batched(params: PdhgParameters, problems, *, cost: str = "f32", points=None, device: int = 0,
                 iterations: int = 256, candidates=None, tile_shapes=BATCH_TILE_SHAPES,
                 unit_costs=BATCH_UNIT_COSTS):
    """The batched solver's autotuner: times the first `iterations` iterations
    of the batch under candidate configurations and returns (best
    configuration, [(configuration, seconds)]); pass the configuration's keys
    to optimize_batched. Three stages, each starting from the best so far:
    the launch configuration (the primal pass, staged by bulk copies or
    direct, times the resident CTAs per SM of the matrix passes, and the
    persistent chunk launch with the direct pass) with 256-row tiles; the tile shape (128-row panels at three or two CTAs per
    SM); the tile balance, the per-unit overhead that the CTA split charges
    beside a unit's rows (0 cuts ranges of equal rows, 8 nearly equal unit
    counts)."""
    import copy

    p = copy.deepcopy(params)
    p.termination_criteria.iteration_limit = int(iterations)
    timings = []

    def run(cand):
        _, sec = optimize_batched(p, problems, cost=cost, points=points, device=device, return_primal=False,
                                  **cand)
        timings.append((dict(cand), sec))

    for cand in candidates or BATCH_TUNING_CANDIDATES:
        run({"panel_rows": 256, **cand, "unit_cost": 0.25})
    best = dict(min(timings, key=lambda t: t[1])[0])
    for tile in tile_shapes:
        run({**best, **tile})
    best = dict(min(timings, key=lambda t: t[1])[0])
    for uc in unit_costs:
        if uc != best["unit_cost"]:
            run({**best, "unit_cost": uc})
    best = min(timings, key=lambda t: t[1])[0]
    return best, timings
