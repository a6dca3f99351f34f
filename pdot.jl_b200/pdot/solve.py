"""Mirror of scripts/solve.jl: `solve_instance_and_output`, `warm_up`,
`write_vector_to_file`, plus `rounding` (src/utils_gpu.jl:296-318).

Compatibility fixes to the script as shipped (it does not run as written):
`output_dir` is the `output_directory` argument (scripts/solve.jl:54,101,...),
`time_sec_limit` is +inf (:72), the warm-up uses the caller's tolerance and its
own termination criteria (:25-26, :39), `rounding` is the package's (:117),
and the dual file holds [dual_source; dual_target] (:120, the struct has no
`dual_solution` field, src/saddle_point_gpu.jl:11-12).
"""
from __future__ import annotations

import gzip
import json
import math
import os
import sys
from decimal import Decimal
from dataclasses import asdict

import numpy as np

from . import api


def julia_float_str(x: float) -> str:
    """Float64 text as Julia writes it (`println`, and JSON3 through the same
    `Base.Ryu.writeshortest`): the shortest round-trip digits, in fixed
    notation when 1e-4 <= |x| < 1e6 (decimal point position pt with
    -4 < pt <= 6) and as d.ddde±x otherwise (0.25, 100000.0, 1.0e6, 1.0e-5,
    1.234567e8); `Inf`, `-Inf`, `NaN`. Python's repr gives the same digits."""
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Inf" if x > 0 else "-Inf"
    if x == 0.0:
        return "-0.0" if math.copysign(1.0, x) < 0 else "0.0"
    sign, digits, exponent = Decimal(repr(x)).normalize().as_tuple()
    ds = "".join(str(d) for d in digits)
    pt = len(ds) + exponent  # digits before the decimal point
    neg = "-" if sign else ""
    if -4 < pt <= 6:
        if pt <= 0:
            return f"{neg}0.{'0' * (-pt)}{ds}"
        if pt >= len(ds):
            return f"{neg}{ds}{'0' * (pt - len(ds))}.0"
        return f"{neg}{ds[:pt]}.{ds[pt:]}"
    return f"{neg}{ds[0]}.{ds[1:] or '0'}e{pt - 1}"


def write_vector_to_file(filename: str, vector) -> None:
    """scripts/solve.jl:5-11: one value per line, matrices in column-major order."""
    arr = np.asarray(vector)
    flat = arr.ravel(order="F")
    with open(filename, "w") as io:
        for x in flat:
            io.write(julia_float_str(x) + "\n")


def rounding(problem: api.OptimalTransportProblem, primal_solution: np.ndarray, *, device: int = 0) -> np.ndarray:
    """src/utils_gpu.jl:296-318, run on the GPU (pdot_rounding_host): scale the
    rows, then the columns, onto the marginals and add the rank-one correction.
    Like the reference it modifies `primal_solution` in place and returns it."""
    from . import _abi

    X = primal_solution
    if not (isinstance(X, np.ndarray) and X.dtype == np.float64 and X.flags.f_contiguous):
        raise TypeError("primal_solution must be a Fortran-ordered float64 matrix (updated in place)")
    a = np.ascontiguousarray(problem.source_distribution, dtype=np.float64)
    b = np.ascontiguousarray(problem.target_distribution, dtype=np.float64)
    m, n = X.shape
    lib = _abi.load()
    rc = lib.pdot_rounding_host(m, n, a.ctypes.data, b.ctypes.data, X.ctypes.data, device)
    _abi.check(lib, rc, "pdot_rounding_host")
    return X


def default_parameters(tolerance: float = 1.0e-4, *, verbosity: int = 2,
                       iteration_limit: int = api.INT32_MAX) -> api.PdhgParameters:
    """The parameters scripts/solve.jl:58-86 builds."""
    restart_params = api.construct_restart_parameters(
        api.ADAPTIVE_KKT, api.KKT_GREEDY, 1000, 0.36, 0.1, 0.9, 0.5
    )
    termination_params = api.construct_termination_criteria(
        optimality_norm=api.L_2,
        eps_optimal_absolute=tolerance,
        eps_optimal_relative=tolerance,
        time_sec_limit=math.inf,
        iteration_limit=iteration_limit,
        kkt_matrix_pass_limit=math.inf,
    )
    return api.PdhgParameters(
        1.0, False, verbosity, True, 128, termination_params, restart_params,
        api.AdaptiveStepsizeParams(2, 1),
    )


def warm_up(ot: api.OptimalTransportProblem, tolerance: float = 1.0e-4) -> None:
    """scripts/solve.jl:13-45: a 100-iteration solve, verbosity 0."""
    params = default_parameters(tolerance, verbosity=0, iteration_limit=100)
    api.optimize(params, ot)


def _json3(obj) -> str:
    """JSON text as JSON3.write(x; allow_inf = true) writes it: compact, fields
    in declaration order, enums by name, floats in Julia's shortest form."""
    if isinstance(obj, dict):
        return "{" + ",".join(f"{json.dumps(k, ensure_ascii=False)}:{_json3(v)}" for k, v in obj.items()) + "}"
    if isinstance(obj, (list, tuple)):
        return "[" + ",".join(_json3(v) for v in obj) + "]"
    if isinstance(obj, bool):
        return "true" if obj else "false"
    if hasattr(obj, "name") and hasattr(obj, "value") and isinstance(obj, int):
        return json.dumps(obj.name)  # enums serialise as their names (StructTypes' StringType)
    if isinstance(obj, (int, np.integer)):
        return str(int(obj))
    if isinstance(obj, (float, np.floating)):
        return julia_float_str(float(obj))
    if isinstance(obj, str):
        return json.dumps(obj, ensure_ascii=False)
    if obj is None:
        return "null"
    raise TypeError(f"cannot write {type(obj).__name__} as JSON")


def solve_log_json(log: api.SolveLog) -> str:
    """src/solve_log.jl:256-327 serialised as scripts/solve.jl:100-112 writes it."""
    return _json3(asdict(log))


def solve_instance_and_output(output_directory: str, instance_name: str,
                              instance: api.OptimalTransportProblem, *, tolerance: float = 1.0e-4):
    """scripts/solve.jl:48-131 (README.md:26-31 signature)."""
    os.makedirs(output_directory, exist_ok=True)
    parameters = default_parameters(tolerance)
    warm_up(instance, tolerance)
    output = api.optimize(parameters, instance)

    log = api.SolveLog()
    log.instance_name = instance_name
    log.command_line_invocation = " ".join(sys.argv)
    log.termination_reason = output.termination_reason
    log.termination_string = output.termination_string
    log.iteration_count = output.iteration_count
    log.solve_time_sec = output.iteration_stats[-1].cumulative_time_sec
    log.solution_stats = output.iteration_stats[-1]
    log.solution_type = api.PointType.POINT_TYPE_AVERAGE_ITERATE

    with open(os.path.join(output_directory, instance_name + "_summary.json"), "w") as io:
        io.write(solve_log_json(log))
    log.iteration_stats = output.iteration_stats
    with gzip.open(os.path.join(output_directory, instance_name + "_full_log.json.gz"), "wt") as io:
        io.write(solve_log_json(log))
    write_vector_to_file(os.path.join(output_directory, instance_name + "_primal.txt"),
                         output.primal_solution)
    write_vector_to_file(os.path.join(output_directory, instance_name + "_primal_rounded.txt"),
                         rounding(instance, output.primal_solution.copy(order="F")))
    write_vector_to_file(os.path.join(output_directory, instance_name + "_dual.txt"),
                         np.concatenate([output.dual_source_solution, output.dual_target_solution]))
    return output
