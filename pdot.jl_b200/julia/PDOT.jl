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

struct CSolverOptions                           # pdot_solver_options
    device::Int32
    use_cuda_graph::Int32
    time_kernels::Int32
    plan_precision::Int32
    cost_storage::Int32
    point_dim::Int32
    source_points::Ptr{Float32}
    target_points::Ptr{Float32}
    cost_scale::Float64
    warm_dual_source::Ptr{Float64}
    warm_dual_target::Ptr{Float64}
    primal_pass::Int32
    ctas_per_sm::Int32
    warm_primal::Ptr{Float64}
    warm_plan_epsilon::Float64
    warm_plan_iterations::Int32
    fail_bounded_waits::Int32
    warm_restart_at_zero::Int32
    warm_primal_weight::Float64
    batch_unit_cost::Float64
    persistent_chunks::Int32
    batch_panel_rows::Int32
end

struct CBatchProblem                            # pdot_batch_problem
    num_instances::Int64
    num_rows::Ptr{Int64}
    num_cols::Ptr{Int64}
    cost_matrices::Ptr{Ptr{Float64}}
    source_distributions::Ptr{Ptr{Float64}}
    target_distributions::Ptr{Ptr{Float64}}
    source_points::Ptr{Ptr{Float32}}
    target_points::Ptr{Ptr{Float32}}
    warm_dual_sources::Ptr{Ptr{Float64}}
    warm_dual_targets::Ptr{Ptr{Float64}}
    warm_primals::Ptr{Ptr{Float64}}
    race_groups::Ptr{Int32}
    warm_primal_weights::Ptr{Float64}
end

struct CBatchOutput                             # pdot_batch_output
    primal_solution::Ptr{Float64}
    dual_source_solution::Ptr{Float64}
    dual_target_solution::Ptr{Float64}
    termination_reason::Int32
    iteration_count::Int32
    final_stats::CIterationStats
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

# Options of this implementation beyond the reference (include/pdot.h):
# precision :f64 (the drop-in) or :f32 (FP32 plan); cost :f64, :f32, :bf16,
# :sqeuclid or :l1 (the last two from `points`, a tuple of Float32 matrices
# m x dim and n x dim, one point per row); warm_start (u0, v0) or (u0, v0, X0);
# recover_plan (eps, rounds) recovers X0 from (u0, v0).
const PRECISIONS = Dict(:f64 => Int32(0), :f32 => Int32(1))
const COSTS = Dict(:f64 => Int32(0), :f32 => Int32(1), :bf16 => Int32(2), :sqeuclid => Int32(3), :l1 => Int32(4))

function solver_options(; device::Integer = 0, precision::Symbol = :f64, cost::Union{Symbol,Nothing} = nothing,
                        point_dim::Integer = 0, source_points::Ptr{Float32} = Ptr{Float32}(0),
                        target_points::Ptr{Float32} = Ptr{Float32}(0), u0::Ptr{Float64} = Ptr{Float64}(0),
                        v0::Ptr{Float64} = Ptr{Float64}(0), X0::Ptr{Float64} = Ptr{Float64}(0),
                        recover_plan = nothing, primal_pass::Integer = 0, ctas_per_sm::Integer = 0,
                        warm_primal_weight::Real = 0.0, warm_restart_at_zero::Bool = false)
    c = cost === nothing ? (precision == :f64 ? :f64 : :f32) : cost
    eps, rounds = recover_plan === nothing ? (0.0, 0) : (Float64(recover_plan[1]), Int(recover_plan[2]))
    return CSolverOptions(Int32(device), Int32(1), Int32(0), PRECISIONS[precision], COSTS[c], Int32(point_dim),
                          source_points, target_points, 0.0, u0, v0, Int32(primal_pass), Int32(ctas_per_sm), X0,
                          eps, Int32(rounds), Int32(0), Int32(warm_restart_at_zero), Float64(warm_primal_weight), 0.0,
                          Int32(0), Int32(0))
end

# points are given one per row (m x dim); the C ABI reads them row-major
row_major(P::AbstractMatrix) = Matrix{Float32}(permutedims(P))

"""
    optimize(params::PdhgParameters, original_problem::OptimalTransportProblem; kwargs...) -> SaddlePointOutput

src/solver_gpu.jl:413-720, run by libpdot.so on the GPU. Raises where the
reference raises (`primal_importance`, src/solver_gpu.jl:420-422). Without
keywords this is the FP64 drop-in; the keywords (`precision`, `cost`,
`points`, `warm_start`, `recover_plan`, `device`) select this implementation's
mixed precision and warm starts.
"""
function optimize(params::PdhgParameters, original_problem::OptimalTransportProblem;
                  precision::Symbol = :f64, cost::Union{Symbol,Nothing} = nothing, points = nothing,
                  warm_start = nothing, recover_plan = nothing, device::Integer = 0)
    if params.primal_importance <= 0 || !isfinite(params.primal_importance)
        error("primal_importance must be positive and finite")
    end
    C = original_problem.cost_matrix
    a = original_problem.source_distribution
    b = original_problem.target_distribution
    nrow, ncol = length(a), length(b)
    plain = precision == :f64 && cost === nothing && points === nothing && warm_start === nothing &&
            recover_plan === nothing && device == 0
    xs = points === nothing ? Float32[] : row_major(points[1])
    ys = points === nothing ? Float32[] : row_major(points[2])
    dim = points === nothing ? 0 : size(points[1], 2)
    u0 = warm_start === nothing ? Float64[] : Vector{Float64}(warm_start[1])
    v0 = warm_start === nothing ? Float64[] : Vector{Float64}(warm_start[2])
    X0 = (warm_start === nothing || length(warm_start) < 3) ? Float64[] : Matrix{Float64}(warm_start[3])
    primal = zeros(nrow, ncol)
    dual_source = zeros(nrow)
    dual_target = zeros(ncol)
    limit = Int64(params.termination_criteria.iteration_limit)
    capacity = min(1 << 16, limit ÷ max(Int64(params.termination_evaluation_frequency), 1) + 16)
    stats = Vector{CIterationStats}(undef, capacity)
    out = COutput()
    cparams = to_c(params)
    GC.@preserve C a b primal dual_source dual_target stats xs ys u0 v0 X0 begin
        cprob = CProblem(nrow, ncol, isempty(C) ? Ptr{Float64}(0) : pointer(C), pointer(a), pointer(b))
        out.primal_solution = pointer(primal)
        out.dual_source_solution = pointer(dual_source)
        out.dual_target_solution = pointer(dual_target)
        out.iteration_stats = pointer(stats)
        out.iteration_stats_capacity = capacity
        if plain
            rc = ccall((:pdot_optimize, libpdot), Cint,
                       (Ref{CProblem}, Ref{CPdhgParameters}, Ptr{Cvoid}, Ref{COutput}),
                       cprob, cparams, C_NULL, out)
        else
            opts = solver_options(device = device, precision = precision, cost = cost, point_dim = dim,
                                  source_points = isempty(xs) ? Ptr{Float32}(0) : pointer(xs),
                                  target_points = isempty(ys) ? Ptr{Float32}(0) : pointer(ys),
                                  u0 = isempty(u0) ? Ptr{Float64}(0) : pointer(u0),
                                  v0 = isempty(v0) ? Ptr{Float64}(0) : pointer(v0),
                                  X0 = isempty(X0) ? Ptr{Float64}(0) : pointer(X0), recover_plan = recover_plan)
            rc = ccall((:pdot_optimize, libpdot), Cint,
                       (Ref{CProblem}, Ref{CPdhgParameters}, Ref{CSolverOptions}, Ref{COutput}),
                       cprob, cparams, opts, out)
        end
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
the rank-one correction, making the plan feasible. Runs on the GPU
(`pdot_rounding_host`), in place on `primal_solution`, which it returns, as the
reference's `feas_solution` aliases it.
"""
function rounding(problem::OptimalTransportProblem, primal_solution::Matrix{Float64}; device::Integer = 0)
    a, b = problem.source_distribution, problem.target_distribution
    m, n = size(primal_solution)
    GC.@preserve a b primal_solution begin
        rc = ccall((:pdot_rounding_host, libpdot), Cint,
                   (Int64, Int64, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Int32),
                   m, n, pointer(a), pointer(b), pointer(primal_solution), Int32(device))
        rc == 0 || error("pdot_rounding_host failed ($rc): ", last_error())
    end
    return primal_solution
end

"""
    optimize_batched(params, problems; cost = :f32, points = nothing, warm_starts = nothing,
                     race_groups = nothing, recover_plan = nothing, device = 0)
        -> (Vector{SaddlePointOutput}, seconds)

Many independent instances of uneven sizes in one lockstep solve on the GPU
(`pdot_optimize_batched`), each with its own step size, restarts and
termination. `cost = :f32` stores each instance's cost matrix in FP32;
`:sqeuclid` and `:l1` compute it from `points[k] = (xs, ys)` (one point per row).
`warm_starts[k]` is `nothing`, `(u0, v0)` or `(u0, v0, X0)`; instances with the
same `race_groups` id stop once one of them ends optimal. Each output's
`iteration_stats` holds its final evaluation.
"""
function optimize_batched(params::PdhgParameters, problems::Vector{OptimalTransportProblem};
                          cost::Symbol = :f32, points = nothing, warm_starts = nothing, race_groups = nothing,
                          recover_plan = nothing, device::Integer = 0)
    B = length(problems)
    rows = Int64[length(p.source_distribution) for p in problems]
    cols = Int64[length(p.target_distribution) for p in problems]
    keep = Any[]
    null64, null32 = Ptr{Float64}(0), Ptr{Float32}(0)
    ptr(x) = (push!(keep, x); isempty(x) ? (eltype(x) == Float32 ? null32 : null64) : pointer(x))
    costs = Ptr{Float64}[cost == :f32 ? ptr(p.cost_matrix) : null64 for p in problems]
    srcs = Ptr{Float64}[ptr(p.source_distribution) for p in problems]
    tgts = Ptr{Float64}[ptr(p.target_distribution) for p in problems]
    xs = Ptr{Float32}[points === nothing ? null32 : ptr(row_major(points[k][1])) for k in 1:B]
    ys = Ptr{Float32}[points === nothing ? null32 : ptr(row_major(points[k][2])) for k in 1:B]
    dim = points === nothing ? 0 : size(points[1][1], 2)
    wu = Ptr{Float64}[warm_starts === nothing || warm_starts[k] === nothing ? null64 :
                      ptr(Vector{Float64}(warm_starts[k][1])) for k in 1:B]
    wv = Ptr{Float64}[warm_starts === nothing || warm_starts[k] === nothing ? null64 :
                      ptr(Vector{Float64}(warm_starts[k][2])) for k in 1:B]
    wx = Ptr{Float64}[warm_starts === nothing || warm_starts[k] === nothing || length(warm_starts[k]) < 3 ?
                      null64 : ptr(Matrix{Float64}(warm_starts[k][3])) for k in 1:B]
    groups = race_groups === nothing ? Int32[] : Int32.(race_groups)
    primals = [zeros(rows[k], cols[k]) for k in 1:B]
    us = [zeros(rows[k]) for k in 1:B]
    vs = [zeros(cols[k]) for k in 1:B]
    outs = CBatchOutput[CBatchOutput(pointer(primals[k]), pointer(us[k]), pointer(vs[k]), Int32(0), Int32(0),
                                     CIterationStats(Int32(0), CConvergenceInformation(Int32(0), ntuple(_ -> 0.0, 16)),
                                                     0.0, Int32(0), 0.0, Int32(0), 0.0, 0.0, 0.0)) for k in 1:B]
    seconds = Ref{Float64}(0.0)
    opts = solver_options(device = device, precision = :f32, cost = cost, point_dim = dim,
                          recover_plan = recover_plan)
    GC.@preserve keep rows cols costs srcs tgts xs ys wu wv wx groups primals us vs outs begin
        bp = CBatchProblem(B, pointer(rows), pointer(cols), cost == :f32 ? pointer(costs) : Ptr{Ptr{Float64}}(0),
                           pointer(srcs), pointer(tgts),
                           points === nothing ? Ptr{Ptr{Float32}}(0) : pointer(xs),
                           points === nothing ? Ptr{Ptr{Float32}}(0) : pointer(ys),
                           warm_starts === nothing ? Ptr{Ptr{Float64}}(0) : pointer(wu),
                           warm_starts === nothing ? Ptr{Ptr{Float64}}(0) : pointer(wv),
                           warm_starts === nothing ? Ptr{Ptr{Float64}}(0) : pointer(wx),
                           isempty(groups) ? Ptr{Int32}(0) : pointer(groups), Ptr{Float64}(0))
        rc = ccall((:pdot_optimize_batched, libpdot), Cint,
                   (Ref{CBatchProblem}, Ref{CPdhgParameters}, Ref{CSolverOptions}, Ptr{CBatchOutput}, Ref{Float64}),
                   bp, to_c(params), opts, outs, seconds)
        rc == 0 || error("pdot_optimize_batched failed ($rc): ", last_error())
    end
    results = SaddlePointOutput[]
    for k in 1:B
        reason = TerminationReason(outs[k].termination_reason)
        push!(results, SaddlePointOutput(primals[k], us[k], vs[k], reason, termination_reason_to_string(reason),
                                         outs[k].iteration_count, [from_c(outs[k].final_stats)]))
    end
    return results, seconds[]
end

end # module PDOT
