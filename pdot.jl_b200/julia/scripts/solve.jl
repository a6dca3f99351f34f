# scripts/solve.jl of the reference, over the libpdot.so-backed PDOT module.
#
# The signature of solve_instance_and_output is the reference's
# (scripts/solve.jl:48-53, README.md:26-31). The names the shipped script
# leaves undefined are bound here: `output_dir` is the `output_directory`
# argument, `time_sec_limit` is Inf, the warm-up uses the caller's tolerance
# and its own termination criteria, `rounding` is PDOT.rounding and the dual
# file holds [dual_source_solution; dual_target_solution].
import GZip
import JSON3

include(joinpath(@__DIR__, "..", "PDOT.jl"))
using .PDOT

function write_vector_to_file(filename, vector)
    open(filename, "w") do io
        for x in vector
            println(io, x)
        end
    end
end

function default_parameters(tolerance; verbosity = 2, iteration_limit = typemax(Int32))
    restart_params = PDOT.construct_restart_parameters(
        PDOT.ADAPTIVE_KKT,      # NO_RESTARTS FIXED_FREQUENCY ADAPTIVE_KKT
        PDOT.KKT_GREEDY,        # NO_RESTART_TO_CURRENT KKT_GREEDY
        1000,                   # restart_frequency_if_fixed
        0.36,                   # artificial_restart_threshold
        0.1,                    # sufficient_reduction_for_restart
        0.9,                    # necessary_reduction_for_restart
        0.5,                    # primal_weight_update_smoothing
    )
    termination_params = PDOT.construct_termination_criteria(
        optimality_norm = PDOT.L_2,
        eps_optimal_absolute = tolerance,
        eps_optimal_relative = tolerance,
        time_sec_limit = Inf,
        iteration_limit = iteration_limit,
        kkt_matrix_pass_limit = Inf,
    )
    return PDOT.PdhgParameters(1.0, false, verbosity, true, 128, termination_params, restart_params,
                               PDOT.AdaptiveStepsizeParams(2, 1))
end

function warm_up(ot::PDOT.OptimalTransportProblem; tolerance = 1.0e-4)
    PDOT.optimize(default_parameters(tolerance; verbosity = 0, iteration_limit = 100), ot)
end

function solve_instance_and_output(
    output_directory::String,
    instance_name::String,
    instance::PDOT.OptimalTransportProblem;
    tolerance = 1.0e-4,
)
    if !isdir(output_directory)
        mkpath(output_directory)
    end
    parameters = default_parameters(tolerance)
    warm_up(instance; tolerance = tolerance)

    output::PDOT.SaddlePointOutput = PDOT.optimize(parameters, instance)
    log = PDOT.SolveLog()
    log.instance_name = instance_name
    log.command_line_invocation = join([PROGRAM_FILE; ARGS...], " ")
    log.termination_reason = output.termination_reason
    log.termination_string = output.termination_string
    log.iteration_count = output.iteration_count
    log.solve_time_sec = output.iteration_stats[end].cumulative_time_sec
    log.solution_stats = output.iteration_stats[end]
    log.solution_type = PDOT.POINT_TYPE_AVERAGE_ITERATE

    open(joinpath(output_directory, instance_name * "_summary.json"), "w") do io
        write(io, JSON3.write(log, allow_inf = true))
    end
    log.iteration_stats = output.iteration_stats
    GZip.open(joinpath(output_directory, instance_name * "_full_log.json.gz"), "w") do io
        write(io, JSON3.write(log, allow_inf = true))
    end
    write_vector_to_file(joinpath(output_directory, instance_name * "_primal.txt"), output.primal_solution)
    write_vector_to_file(joinpath(output_directory, instance_name * "_primal_rounded.txt"),
                         PDOT.rounding(instance, copy(output.primal_solution)))
    write_vector_to_file(joinpath(output_directory, instance_name * "_dual.txt"),
                         [output.dual_source_solution; output.dual_target_solution])
    return
end
