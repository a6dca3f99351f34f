"""pdot — B200-native restarted adaptive PDHG for discrete optimal transport.

Drop-in for MIT-Lu-Lab/PDOT.jl's API: the names below mirror the reference's
Julia module, and `optimize` runs the hand-written sm_100a kernels of
libpdot.so through its C ABI (include/pdot.h).
"""
from .api import (  # noqa: F401
    ADAPTIVE_KKT,
    FIXED_FREQUENCY,
    KKT_GREEDY,
    L_2,
    L_INF,
    NO_RESTART_TO_CURRENT,
    NO_RESTARTS,
    AdaptiveStepsizeParams,
    ConstantStepsizeParams,
    ConvergenceInformation,
    IterationStats,
    OptimalityNorm,
    OptimalTransportProblem,
    PdhgParameters,
    PointType,
    RestartChoice,
    RestartParameters,
    RestartScheme,
    RestartToCurrentMetric,
    SaddlePointOutput,
    SolveLog,
    Solver,
    TerminationCriteria,
    TerminationReason,
    construct_restart_parameters,
    construct_termination_criteria,
    optimize,
    optimize_batched,
    termination_reason_to_string,
    tune_batched,
)
from .solve import default_parameters, rounding, solve_instance_and_output, warm_up, write_vector_to_file  # noqa: F401
