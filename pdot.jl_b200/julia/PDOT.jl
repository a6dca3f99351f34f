"""
    PDOT

Drop-in for MIT-Lu-Lab/PDOT.jl's API backed by libpdot.so, the B200 (sm_100a)
implementation of restarted adaptive PDHG for discrete optimal transport.

The user-facing types and functions keep the reference's names, fields and
argument order (src/io.jl, src/solver_gpu.jl, src/saddle_point_gpu.jl,
src/termination.jl, src/solve_log.jl). `optimize` marshals them into the C
structs of include/pdot.h and `ccall`s `pdot_optimize`; the solve runs on the
GPU with no Julia-side device code and no CPU fallback.
"""
module PDOT

import LinearAlgebra
import Printf
import StructTypes

const libpdot = get(ENV, "PDOT_LIBRARY", normpath(joinpath(@__DIR__, "..", "lib", "libpdot.so")))

# ---------------------------------------------------------------- problem
mutable struct OptimalTransportProblem          # src/io.jl:1-5
    cost_matrix::Matrix{Float64}
    source_distribution::Vector{Float64}
    target_distribution::Vector{Float64}
end

# ---------------------------------------------------------------- enums
@enum OptimalityNorm L_INF L_2                                              # src/termination.jl:2
@enum RestartScheme NO_RESTARTS FIXED_FREQUENCY ADAPTIVE_KKT                # src/saddle_point_gpu.jl:401
@enum RestartToCurrentMetric NO_RESTART_TO_CURRENT KKT_GREEDY              # src/saddle_point_gpu.jl:408
@enum RestartChoice begin                                                   # src/solve_log.jl:15-20
    RESTART_CHOICE_UNSPECIFIED
    RESTART_CHOICE_NO_RESTART
    RESTART_CHOICE_WEIGHTED_AVERAGE_RESET
    RESTART_CHOICE_RESTART_TO_AVERAGE
end
@enum PointType begin                                                       # src/solve_log.jl:35-41
    POINT_TYPE_UNSPECIFIED
    POINT_TYPE_CURRENT_ITERATE
    POINT_TYPE_ITERATE_DIFFERENCE
    POINT_TYPE_AVERAGE_ITERATE
    POINT_TYPE_NONE
end
@enum TerminationReason begin                                               # src/solve_log.jl:245-254
    TERMINATION_REASON_UNSPECIFIED
    TERMINATION_REASON_OPTIMAL
    TERMINATION_REASON_TIME_LIMIT
    TERMINATION_REASON_ITERATION_LIMIT
    TERMINATION_REASON_KKT_MATRIX_PASS_LIMIT
    TERMINATION_REASON_NUMERICAL_ERROR
    TERMINATION_REASON_INVALID_PROBLEM
    TERMINATION_REASON_OTHER
end

# ---------------------------------------------------------------- parameters
struct AdaptiveStepsizeParams                  # src/solver_gpu.jl:2-5
    reduction_exponent::Float64
    growth_exponent::Float64
end
struct ConstantStepsizeParams end              # src/solver_gpu.jl:7

mutable struct TerminationCriteria             # src/termination.jl:5-51
    optimality_norm::OptimalityNorm
    eps_optimal_absolute::Float64
    eps_optimal_relative::Float64
    time_sec_limit::Float64
    iteration_limit::Int32
    kkt_matrix_pass_limit::Float64
end

function construct_termination_criteria(;      # src/termination.jl:53-69
    optimality_norm = L_2,
    eps_optimal_absolute,
    eps_optimal_relative,
    time_sec_limit = Inf,
    iteration_limit = typemax(Int32),
    kkt_matrix_pass_limit = Inf,
)
    return TerminationCriteria(optimality_norm, eps_optimal_absolute, eps_optimal_relative,
                               time_sec_limit, iteration_limit, kkt_matrix_pass_limit)
end

mutable struct RestartParameters               # src/saddle_point_gpu.jl:411-441
    restart_scheme::RestartScheme
    restart_to_current_metric::RestartToCurrentMetric
    restart_frequency_if_fixed::Int64
    artificial_restart_threshold::Float64
    sufficient_reduction_for_restart::Float64
    necessary_reduction_for_restart::Float64
    primal_weight_update_smoothing::Float64
end

function construct_restart_parameters(         # src/saddle_point_gpu.jl:446-472
    restart_scheme::RestartScheme,
    restart_to_current_metric::RestartToCurrentMetric,
    restart_frequency_if_fixed::Int64,
    artificial_restart_threshold::Float64,
    sufficient_reduction_for_restart::Float64,
    necessary_reduction_for_restart::Float64,
    primal_weight_update_smoothing::Float64,
)
    @assert restart_frequency_if_fixed > 1
    @assert 0.0 < artificial_restart_threshold <= 1.0
    @assert 0.0 < sufficient_reduction_for_restart <= necessary_reduction_for_restart <= 1.0
    @assert 0.0 <= primal_weight_update_smoothing <= 1.0
    return RestartParameters(restart_scheme, restart_to_current_metric, restart_frequency_if_fixed,
                             artificial_restart_threshold, sufficient_reduction_for_restart,
                             necessary_reduction_for_restart, primal_weight_update_smoothing)
end

struct PdhgParameters                          # src/solver_gpu.jl:9-21
    primal_importance::Float64
    scale_invariant_initial_primal_weight::Bool
    verbosity::Int64
    record_iteration_stats::Bool
    termination_evaluation_frequency::Int32
    termination_criteria::TerminationCriteria
    restart_params::RestartParameters
    step_size_policy_params::Union{AdaptiveStepsizeParams,ConstantStepsizeParams}
end

# ---------------------------------------------------------------- logs and output
mutable struct ConvergenceInformation          # src/solve_log.jl:47-147
    candidate_type::PointType
    primal_objective::Float64
    dual_objective::Float64
    corrected_dual_objective::Float64
    l_inf_primal_residual::Float64
    l2_primal_residual::Float64
    l_inf_dual_residual::Float64
    l2_dual_residual::Float64
    relative_l_inf_primal_residual::Float64
    relative_l2_primal_residual::Float64
    relative_l_inf_dual_residual::Float64
    relative_l2_dual_residual::Float64
    relative_optimality_gap::Float64
    l_inf_primal_variable::Float64
    l2_primal_variable::Float64
    l_inf_dual_variable::Float64
    l2_dual_variable::Float64
end
ConvergenceInformation() = ConvergenceInformation(POINT_TYPE_UNSPECIFIED, zeros(16)...)

mutable struct IterationStats                  # src/solve_log.jl:154-228
    iteration_number::Int32
    convergence_information::Vector{ConvergenceInformation}
    cumulative_kkt_matrix_passes::Float64
    cumulative_rejected_steps::Int32
    cumulative_time_sec::Float64
    restart_used::RestartChoice
    step_size::Float64
    primal_weight::Float64
    method_specific_stats::Dict{String,Float64}
end
IterationStats() = IterationStats(0, ConvergenceInformation[], 0.0, Int32(0), 0.0,
                                  RESTART_CHOICE_UNSPECIFIED, 0.0, 0.0, Dict{String,Float64}())

mutable struct SolveLog                        # src/solve_log.jl:256-327
    instance_name::String
    command_line_invocation::String
    termination_reason::TerminationReason
    termination_string::String
    iteration_count::Int32
    solve_time_sec::Float64
    solution_stats::IterationStats
    solution_type::PointType
    iteration_stats::Vector{IterationStats}
end
SolveLog() = SolveLog("", "", TERMINATION_REASON_UNSPECIFIED, "", Int32(0), 0.0, IterationStats(),
                      POINT_TYPE_UNSPECIFIED, IterationStats[])

StructTypes.StructType(::Type{ConvergenceInformation}) = StructTypes.Mutable()
StructTypes.StructType(::Type{IterationStats}) = StructTypes.Mutable()
StructTypes.StructType(::Type{SolveLog}) = StructTypes.Mutable()

struct SaddlePointOutput                       # src/saddle_point_gpu.jl:2-34
    primal_solution::Matrix{Float64}
    dual_source_solution::Vector{Float64}
    dual_target_solution::Vector{Float64}
    termination_reason::TerminationReason
    termination_string::String
    iteration_count::Int32
    iteration_stats::Vector{IterationStats}
end

termination_reason_to_string(r::TerminationReason) = string(r)[20:end]   # src/termination.jl:168-171

# ---------------------------------------------------------------- C mirrors (include/pdot.h)
struct CProblem
    num_row::Int64
    num_col::Int64
    cost_matrix::Ptr{Float64}
    source_distribution::Ptr{Float64}
    target_distribution::Ptr{Float64}
end

struct CTerminationCriteria
    optimality_norm::Int32
    eps_optimal_absolute::Float64
    eps_optimal_relative::Float64
    time_sec_limit::Float64
    iteration_limit::Int32
    kkt_matrix_pass_limit::Float64
end

struct CRestartParameters
    restart_scheme::Int32
    restart_to_current_metric::Int32
    restart_frequency_if_fixed::Int64
    artificial_restart_threshold::Float64
    sufficient_reduction_for_restart::Float64
    necessary_reduction_for_restart::Float64
    primal_weight_update_smoothing::Float64
end

struct CPdhgParameters
    primal_importance::Float64
    scale_invariant_initial_primal_weight::Int32
    verbosity::Int64
    record_iteration_stats::Int32
    termination_evaluation_frequency::Int32
    termination_criteria::CTerminationCriteria
    restart_params::CRestartParameters
    step_size_policy::Int32
    reduction_exponent::Float64
    growth_exponent::Float64
end

struct CConvergenceInformation
    candidate_type::Int32
    values::NTuple{16,Float64}   # the 16 Float64 fields of ConvergenceInformation, in order
end

struct CIterationStats
    iteration_number::Int32
    convergence_information::CConvergenceInformation
    cumulative_kkt_matrix_passes::Float64
    cumulative_rejected_steps::Int32
    cumulative_time_sec::Float64
    restart_used::Int32
    step_size::Float64
    primal_weight::Float64
    time_spent_doing_basic_algorithm::Float64
end

mutable struct COutput
    primal_solution::Ptr{Float64}
    dual_source_solution::Ptr{Float64}
    dual_target_solution::Ptr{Float64}
    iteration_stats::Ptr{CIterationStats}
    iteration_stats_capacity::Int64
    iteration_stats_count::Int64
    termination_reason::Int32
    iteration_count::Int32
    solve_time_sec::Float64
    final_stats::CIterationStats
    COutput() = new()
end

function to_c(tc::TerminationCriteria)
    return CTerminationCriteria(Int32(tc.optimality_norm), tc.eps_optimal_absolute, tc.eps_optimal_relative,
                                tc.time_sec_limit, tc.iteration_limit, tc.kkt_matrix_pass_limit)
end
function to_c(rp::RestartParameters)
    return CRestartParameters(Int32(rp.restart_scheme), Int32(rp.restart_to_current_metric),
                              rp.restart_frequency_if_fixed, rp.artificial_restart_threshold,
                              rp.sufficient_reduction_for_restart, rp.necessary_reduction_for_restart,
                              rp.primal_weight_update_smoothing)
end
function to_c(p::PdhgParameters)
    sp = p.step_size_policy_params
    adaptive = sp isa AdaptiveStepsizeParams
    return CPdhgParameters(p.primal_importance, Int32(p.scale_invariant_initial_primal_weight), p.verbosity,
                           Int32(p.record_iteration_stats), p.termination_evaluation_frequency,
                           to_c(p.termination_criteria), to_c(p.restart_params), adaptive ? Int32(0) : Int32(1),
                           adaptive ? sp.reduction_exponent : 0.0, adaptive ? sp.growth_exponent : 0.0)
end

function from_c(s::CIterationStats)
    v = s.convergence_information.values
    ci = ConvergenceInformation(PointType(s.convergence_information.candidate_type), v...)
    return IterationStats(s.iteration_number, [ci], s.cumulative_kkt_matrix_passes, s.cumulative_rejected_steps,
                          s.cumulative_time_sec, RestartChoice(s.restart_used), s.step_size, s.primal_weight,
                          Dict{String,Float64}("time_spent_doing_basic_algorithm" =>
                                                   s.time_spent_doing_basic_algorithm))
end

last_error() = unsafe_string(ccall((:pdot_last_error, libpdot), Cstring, ()))

"""
    optimize(params::PdhgParameters, original_problem::OptimalTransportProblem) -> SaddlePointOutput

src/solver_gpu.jl:413-720, run by libpdot.so on the GPU. Raises where the
reference raises (`primal_importance`, src/solver_gpu.jl:420-422).
"""
function optimize(params::PdhgParameters, original_problem::OptimalTransportProblem)
    if params.primal_importance <= 0 || !isfinite(params.primal_importance)
        error("primal_importance must be positive and finite")
    end
    C = original_problem.cost_matrix
    a = original_problem.source_distribution
    b = original_problem.target_distribution
    nrow, ncol = size(C)
    primal = zeros(nrow, ncol)
    dual_source = zeros(nrow)
    dual_target = zeros(ncol)
    limit = Int64(params.termination_criteria.iteration_limit)
    capacity = min(1 << 16, limit ÷ max(Int64(params.termination_evaluation_frequency), 1) + 16)
    stats = Vector{CIterationStats}(undef, capacity)
    out = COutput()
    cparams = to_c(params)
    GC.@preserve C a b primal dual_source dual_target stats begin
        cprob = CProblem(nrow, ncol, pointer(C), pointer(a), pointer(b))
        out.primal_solution = pointer(primal)
        out.dual_source_solution = pointer(dual_source)
        out.dual_target_solution = pointer(dual_target)
        out.iteration_stats = pointer(stats)
        out.iteration_stats_capacity = capacity
        rc = ccall((:pdot_optimize, libpdot), Cint,
                   (Ref{CProblem}, Ref{CPdhgParameters}, Ptr{Cvoid}, Ref{COutput}),
                   cprob, cparams, C_NULL, out)
        rc == 0 || error("pdot_optimize failed ($rc): ", last_error())
    end
    n = min(out.iteration_stats_count, capacity)
    iteration_stats = IterationStats[from_c(stats[k]) for k in 1:n]
    if out.iteration_stats_count > n || n == 0
        push!(iteration_stats, from_c(out.final_stats))
    end
    reason = TerminationReason(out.termination_reason)
    return SaddlePointOutput(primal, dual_source, dual_target, reason, termination_reason_to_string(reason),
                             out.iteration_count, iteration_stats)
end

"""
    rounding(problem, primal_solution)

src/utils_gpu.jl:296-318: scale rows, then columns, onto the marginals and add
the rank-one correction, making the plan feasible.
"""
function rounding(problem::OptimalTransportProblem, primal_solution::Matrix{Float64})
    feas_solution = primal_solution
    tmp = map(x -> isnan(x) ? 0.0 : x, problem.source_distribution ./ vec(sum(feas_solution, dims = 2)))
    feas_solution .= LinearAlgebra.Diagonal(vec(min.(tmp, 1.0))) * feas_solution
    tmp = map(x -> isnan(x) ? 0.0 : x, problem.target_distribution ./ vec(sum(feas_solution, dims = 1)))
    feas_solution .= feas_solution * LinearAlgebra.Diagonal(vec(min.(tmp, 1.0)))
    err_r = problem.source_distribution .- vec(sum(feas_solution, dims = 2))
    if LinearAlgebra.norm(err_r, 1) != 0.0
        err_r ./= LinearAlgebra.norm(err_r, 1)
    end
    err_c = problem.target_distribution .- vec(sum(feas_solution, dims = 1))
    feas_solution .+= err_r * err_c'
    return feas_solution
end

end # module PDOT
