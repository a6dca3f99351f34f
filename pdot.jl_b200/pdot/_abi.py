"""ctypes mirror of include/pdot.h and the loader of libpdot.so.

The structs here are field-for-field copies of the C declarations, which in
turn follow the reference's Julia structs (src/termination.jl:5-51,
src/saddle_point_gpu.jl:411-441, src/solver_gpu.jl:9-21, src/solve_log.jl:47-228,
src/saddle_point_gpu.jl:2-34).

There is no CPU fallback: if libpdot.so is missing, loading raises.
"""
from __future__ import annotations

import ctypes as ct
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PACKAGE_ROOT, "lib", "libpdot.so")

ABI_VERSION = 1

# error codes
PDOT_OK = 0
PDOT_ERR_INVALID_ARGUMENT = -1
PDOT_ERR_CUDA = -2
PDOT_ERR_OUT_OF_MEMORY = -3
PDOT_ERR_NO_DEVICE = -4
PDOT_ERR_TOO_LARGE = -5

NOALLOC_SCRATCH_BYTES = 16 << 20

PDOT_PASS_ZERO_GRADIENT = 1
PDOT_PASS_FIRST_AVERAGE = 2


class TerminationCriteriaC(ct.Structure):
    _fields_ = [
        ("optimality_norm", ct.c_int32),
        ("eps_optimal_absolute", ct.c_double),
        ("eps_optimal_relative", ct.c_double),
        ("time_sec_limit", ct.c_double),
        ("iteration_limit", ct.c_int32),
        ("kkt_matrix_pass_limit", ct.c_double),
    ]


class RestartParametersC(ct.Structure):
    _fields_ = [
        ("restart_scheme", ct.c_int32),
        ("restart_to_current_metric", ct.c_int32),
        ("restart_frequency_if_fixed", ct.c_int64),
        ("artificial_restart_threshold", ct.c_double),
        ("sufficient_reduction_for_restart", ct.c_double),
        ("necessary_reduction_for_restart", ct.c_double),
        ("primal_weight_update_smoothing", ct.c_double),
    ]


class PdhgParametersC(ct.Structure):
    _fields_ = [
        ("primal_importance", ct.c_double),
        ("scale_invariant_initial_primal_weight", ct.c_int32),
        ("verbosity", ct.c_int64),
        ("record_iteration_stats", ct.c_int32),
        ("termination_evaluation_frequency", ct.c_int32),
        ("termination_criteria", TerminationCriteriaC),
        ("restart_params", RestartParametersC),
        ("step_size_policy", ct.c_int32),
        ("reduction_exponent", ct.c_double),
        ("growth_exponent", ct.c_double),
    ]


PRECISION_F64 = 0
PRECISION_F32 = 1
COST_F64 = 0
COST_F32 = 1
COST_BF16 = 2
COST_SQEUCLID_POINTS = 3
COST_L1_POINTS = 4
PASS_AUTO = 0
PASS_STAGED = 1
PASS_DIRECT = 2


class SolverOptionsC(ct.Structure):
    _fields_ = [
        ("device", ct.c_int32),
        ("use_cuda_graph", ct.c_int32),
        ("time_kernels", ct.c_int32),
        ("plan_precision", ct.c_int32),
        ("cost_storage", ct.c_int32),
        ("point_dim", ct.c_int32),
        ("source_points", ct.POINTER(ct.c_float)),
        ("target_points", ct.POINTER(ct.c_float)),
        ("cost_scale", ct.c_double),
        ("warm_dual_source", ct.POINTER(ct.c_double)),
        ("warm_dual_target", ct.POINTER(ct.c_double)),
        ("primal_pass", ct.c_int32),
        ("ctas_per_sm", ct.c_int32),
        ("warm_primal", ct.POINTER(ct.c_double)),
        ("warm_plan_epsilon", ct.c_double),
        ("warm_plan_iterations", ct.c_int32),
        ("fail_bounded_waits", ct.c_int32),
        ("warm_restart_at_zero", ct.c_int32),
        ("warm_primal_weight", ct.c_double),
        ("batch_unit_cost", ct.c_double),
        ("persistent_chunks", ct.c_int32),
        ("batch_panel_rows", ct.c_int32),
    ]


class SolverStatusC(ct.Structure):
    _fields_ = [
        ("iteration", ct.c_int64),
        ("total_number_iterations", ct.c_int64),
        ("done", ct.c_int32),
        ("termination_reason", ct.c_int32),
        ("step_size", ct.c_double),
        ("primal_weight", ct.c_double),
        ("cumulative_kkt_matrix_passes", ct.c_double),
        ("iteration_stats_count", ct.c_int64),
        ("primal_passes", ct.c_int64),
        ("primal_passes_fresh_average", ct.c_int64),
        ("timed_primal_passes", ct.c_int64),
        ("primal_pass_ms", ct.c_double),
        ("dual_step_ms", ct.c_double),
        ("evaluation_ms", ct.c_double),
    ]


class BatchProblemC(ct.Structure):
    _fields_ = [
        ("num_instances", ct.c_int64),
        ("num_rows", ct.POINTER(ct.c_int64)),
        ("num_cols", ct.POINTER(ct.c_int64)),
        ("cost_matrices", ct.POINTER(ct.c_void_p)),
        ("source_distributions", ct.POINTER(ct.c_void_p)),
        ("target_distributions", ct.POINTER(ct.c_void_p)),
        ("source_points", ct.POINTER(ct.c_void_p)),
        ("target_points", ct.POINTER(ct.c_void_p)),
        ("warm_dual_sources", ct.POINTER(ct.c_void_p)),
        ("warm_dual_targets", ct.POINTER(ct.c_void_p)),
        ("warm_primals", ct.POINTER(ct.c_void_p)),
        ("race_groups", ct.POINTER(ct.c_int32)),
        ("warm_primal_weights", ct.POINTER(ct.c_double)),
    ]


class ProblemC(ct.Structure):
    _fields_ = [
        ("num_row", ct.c_int64),
        ("num_col", ct.c_int64),
        ("cost_matrix", ct.POINTER(ct.c_double)),
        ("source_distribution", ct.POINTER(ct.c_double)),
        ("target_distribution", ct.POINTER(ct.c_double)),
    ]


CONVERGENCE_FIELDS = [
    "primal_objective",
    "dual_objective",
    "corrected_dual_objective",
    "l_inf_primal_residual",
    "l2_primal_residual",
    "l_inf_dual_residual",
    "l2_dual_residual",
    "relative_l_inf_primal_residual",
    "relative_l2_primal_residual",
    "relative_l_inf_dual_residual",
    "relative_l2_dual_residual",
    "relative_optimality_gap",
    "l_inf_primal_variable",
    "l2_primal_variable",
    "l_inf_dual_variable",
    "l2_dual_variable",
]


class ConvergenceInformationC(ct.Structure):
    _fields_ = [("candidate_type", ct.c_int32)] + [(f, ct.c_double) for f in CONVERGENCE_FIELDS]


class IterationStatsC(ct.Structure):
    _fields_ = [
        ("iteration_number", ct.c_int32),
        ("convergence_information", ConvergenceInformationC),
        ("cumulative_kkt_matrix_passes", ct.c_double),
        ("cumulative_rejected_steps", ct.c_int32),
        ("cumulative_time_sec", ct.c_double),
        ("restart_used", ct.c_int32),
        ("step_size", ct.c_double),
        ("primal_weight", ct.c_double),
        ("time_spent_doing_basic_algorithm", ct.c_double),
    ]


class SaddlePointOutputC(ct.Structure):
    _fields_ = [
        ("primal_solution", ct.POINTER(ct.c_double)),
        ("dual_source_solution", ct.POINTER(ct.c_double)),
        ("dual_target_solution", ct.POINTER(ct.c_double)),
        ("iteration_stats", ct.POINTER(IterationStatsC)),
        ("iteration_stats_capacity", ct.c_int64),
        ("iteration_stats_count", ct.c_int64),
        ("termination_reason", ct.c_int32),
        ("iteration_count", ct.c_int32),
        ("solve_time_sec", ct.c_double),
        ("final_stats", IterationStatsC),
    ]


class BatchOutputC(ct.Structure):
    _fields_ = [
        ("primal_solution", ct.POINTER(ct.c_double)),
        ("dual_source_solution", ct.POINTER(ct.c_double)),
        ("dual_target_solution", ct.POINTER(ct.c_double)),
        ("termination_reason", ct.c_int32),
        ("iteration_count", ct.c_int32),
        ("final_stats", IterationStatsC),
    ]


# Every symbol include/pdot.h declares, with its ctypes signature.
_P = ct.c_void_p
_D = ct.c_double
_I64 = ct.c_int64
_I32 = ct.c_int32
SIGNATURES = {
    "pdot_version": (ct.c_int, []),
    "pdot_last_error": (ct.c_char_p, []),
    "pdot_optimize": (
        ct.c_int,
        [ct.POINTER(ProblemC), ct.POINTER(PdhgParametersC), ct.POINTER(SolverOptionsC),
         ct.POINTER(SaddlePointOutputC)],
    ),
    "pdot_default_parameters": (None, [_D, ct.POINTER(PdhgParametersC)]),
    "pdot_solver_create": (
        ct.c_int,
        [ct.POINTER(ProblemC), ct.POINTER(PdhgParametersC), ct.POINTER(SolverOptionsC), ct.POINTER(_P)],
    ),
    "pdot_solver_create_device": (
        ct.c_int,
        [ct.POINTER(ProblemC), ct.POINTER(PdhgParametersC), ct.POINTER(SolverOptionsC), ct.POINTER(_P)],
    ),
    "pdot_solver_reset": (ct.c_int, [_P]),
    "pdot_solver_iterate": (ct.c_int, [_P, _I64, ct.POINTER(SolverStatusC)]),
    "pdot_solver_finish": (ct.c_int, [_P, ct.POINTER(SaddlePointOutputC)]),
    "pdot_solver_stream": (_P, [_P]),
    "pdot_solver_destroy": (None, [_P]),
    "pdot_optimize_batched": (
        ct.c_int,
        [ct.POINTER(BatchProblemC), ct.POINTER(PdhgParametersC), ct.POINTER(SolverOptionsC),
         ct.POINTER(BatchOutputC), ct.POINTER(ct.c_double)],
    ),
    "pdot_rounding_f64": (ct.c_int, [_I64, _I64, _P, _P, _P, _P]),
    "pdot_rounding_host": (ct.c_int, [_I64, _I64, _P, _P, _P, _I32]),
    "pdot_sqeuclid_cost_f64": (ct.c_int, [_I64, _I64, _I32, _P, _P, _I32, _P, _P]),
    "pdot_points_max_sqdist": (ct.c_int, [_I64, _I64, _I32, _P, _P, _P, _P]),
    "pdot_points_c_transform": (ct.c_int, [_I64, _I64, _I32, _P, _P, _P, _D, _P, _P]),
    "pdot_primal_pass_workspace_bytes": (_I64, [_I64, _I64]),
    "pdot_primal_pass_f64_noalloc": (
        ct.c_int,
        [_I64, _I64, _P, _P, _P, _P, _P, _D, _D, _D, _I32, _P, _P, _P, _P],
    ),
    "pdot_primal_pass_f64": (
        ct.c_int,
        [_I64, _I64, _P, _P, _P, _P, _P, _D, _D, _D, _I32, _P, _P, _P, _P, _I64, _P],
    ),
    "pdot_mlp_create": (ct.c_int, [_I32, _I64, _I64, _I64, _I64, ct.c_uint64, ct.POINTER(_P)]),
    "pdot_mlp_destroy": (ct.c_int, [_P]),
    "pdot_mlp_num_parameters": (_I64, [_P]),
    "pdot_mlp_stream": (_P, [_P]),
    "pdot_mlp_get_parameters": (ct.c_int, [_P, _P, _I64]),
    "pdot_mlp_set_parameters": (ct.c_int, [_P, _P, _I64]),
    "pdot_mlp_get_gradients": (ct.c_int, [_P, _P, _I64]),
    "pdot_mlp_set_input": (ct.c_int, [_P, _I64, _P, _D, _D]),
    "pdot_mlp_forward": (ct.c_int, [_P, _P]),
    "pdot_mlp_backward": (ct.c_int, [_P, _P, ct.POINTER(_D)]),
    "pdot_mlp_adamw": (ct.c_int, [_P, ct.c_float, ct.c_float, ct.c_float, ct.c_float, ct.c_float]),
    "pdot_mlp_train_step": (ct.c_int, [_P, _P, ct.c_float, ct.c_float, ct.POINTER(_D)]),
}

_lib = None


def bind(lib: ct.CDLL, signatures=SIGNATURES) -> ct.CDLL:
    for name, (res, args) in signatures.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def load(path: str | None = None) -> ct.CDLL:
    """Load libpdot.so (built in-tree by __graft_entry__.build()). Raises if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"libpdot.so not found at {p}; build it with `python -c 'import __graft_entry__ as g; g.build()'`"
        )
    lib = bind(ct.CDLL(p))
    if lib.pdot_version() != ABI_VERSION:
        raise RuntimeError("libpdot.so ABI version mismatch")
    if path is None:
        _lib = lib
    return lib


def last_error(lib: ct.CDLL) -> str:
    msg = lib.pdot_last_error()
    return msg.decode() if msg else ""


def check(lib: ct.CDLL, rc: int, what: str) -> None:
    if rc != PDOT_OK:
        raise PdotError(rc, f"{what} failed ({rc}): {last_error(lib)}")


class PdotError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code
