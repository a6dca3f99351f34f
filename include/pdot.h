/*
 * pdot.h — C ABI of libpdot.so, a B200 (sm_100a) implementation of PDOT's
 * restarted, adaptive-step PDHG solver for discrete optimal transport.
 *
 * The ABI mirrors the reference's Julia API (MIT-Lu-Lab/PDOT.jl) so that a
 * thin Julia module can `ccall` into it and keep the reference's types:
 *
 *   optimize(params::PdhgParameters, problem::OptimalTransportProblem)
 *       -> SaddlePointOutput                         src/solver_gpu.jl:413-720
 *
 * Conventions
 *   - Matrices are column-major with leading dimension num_row, exactly as a
 *     Julia Matrix{Float64} is laid out: entry (i, j) sits at i + j*num_row.
 *     i indexes sources (rows), j indexes targets (columns).
 *   - Every enum value is the 0-based position of the matching member of the
 *     reference's `@enum` declaration.
 *   - Functions return 0 on success and a negative PDOT_ERR_* code on failure;
 *     pdot_last_error() then returns a thread-local message. Solver outcomes
 *     (optimal, iteration limit, numerical error, ...) are not errors: they are
 *     reported in pdot_saddle_point_output.termination_reason.
 *   - No C++ exception crosses this boundary. Calls are blocking.
 */
#ifndef PDOT_H
#define PDOT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PDOT_ABI_VERSION 1

/* ---- error codes ------------------------------------------------------- */
enum {
  PDOT_OK = 0,
  PDOT_ERR_INVALID_ARGUMENT = -1, /* bad sizes, null pointers, parameter asserts */
  PDOT_ERR_CUDA = -2,             /* a CUDA runtime call failed */
  PDOT_ERR_OUT_OF_MEMORY = -3,    /* device allocation failed */
  PDOT_ERR_NO_DEVICE = -4,        /* no CUDA device, or not an sm_100 device */
  PDOT_ERR_TOO_LARGE = -5         /* a size exceeds a documented maximum */
};

/* ---- enums (values = 0-based order of the reference's @enum) ----------- */
/* OptimalityNorm, src/termination.jl:2 */
enum { PDOT_L_INF = 0, PDOT_L_2 = 1 };
/* RestartScheme, src/saddle_point_gpu.jl:401 */
enum { PDOT_NO_RESTARTS = 0, PDOT_FIXED_FREQUENCY = 1, PDOT_ADAPTIVE_KKT = 2 };
/* RestartToCurrentMetric, src/saddle_point_gpu.jl:408 */
enum { PDOT_NO_RESTART_TO_CURRENT = 0, PDOT_KKT_GREEDY = 1 };
/* RestartChoice, src/solve_log.jl:15-20 */
enum {
  PDOT_RESTART_CHOICE_UNSPECIFIED = 0,
  PDOT_RESTART_CHOICE_NO_RESTART = 1,
  PDOT_RESTART_CHOICE_WEIGHTED_AVERAGE_RESET = 2,
  PDOT_RESTART_CHOICE_RESTART_TO_AVERAGE = 3
};
/* PointType, src/solve_log.jl:35-41 */
enum {
  PDOT_POINT_TYPE_UNSPECIFIED = 0,
  PDOT_POINT_TYPE_CURRENT_ITERATE = 1,
  PDOT_POINT_TYPE_ITERATE_DIFFERENCE = 2,
  PDOT_POINT_TYPE_AVERAGE_ITERATE = 3,
  PDOT_POINT_TYPE_NONE = 4
};
/* TerminationReason, src/solve_log.jl:245-254 */
enum {
  PDOT_TERMINATION_REASON_UNSPECIFIED = 0,
  PDOT_TERMINATION_REASON_OPTIMAL = 1,
  PDOT_TERMINATION_REASON_TIME_LIMIT = 2,
  PDOT_TERMINATION_REASON_ITERATION_LIMIT = 3,
  PDOT_TERMINATION_REASON_KKT_MATRIX_PASS_LIMIT = 4,
  PDOT_TERMINATION_REASON_NUMERICAL_ERROR = 5,
  PDOT_TERMINATION_REASON_INVALID_PROBLEM = 6,
  PDOT_TERMINATION_REASON_OTHER = 7
};
/* Union{AdaptiveStepsizeParams, ConstantStepsizeParams}, src/solver_gpu.jl:2-7,17-20 */
enum { PDOT_STEP_SIZE_ADAPTIVE = 0, PDOT_STEP_SIZE_CONSTANT = 1 };

/* ---- problem: OptimalTransportProblem, src/io.jl:1-5 -------------------- */
typedef struct pdot_problem {
  int64_t num_row;                    /* m, number of sources */
  int64_t num_col;                    /* n, number of targets */
  const double* cost_matrix;          /* m*n, column-major, ld = m (host memory);
                                       * NULL with PDOT_COST_SQEUCLID_POINTS */
  const double* source_distribution;  /* m (host memory) */
  const double* target_distribution;  /* n (host memory) */
} pdot_problem;

/* ---- parameters --------------------------------------------------------- */
/* TerminationCriteria, src/termination.jl:5-51 (same field order) */
typedef struct pdot_termination_criteria {
  int32_t optimality_norm;            /* PDOT_L_INF or PDOT_L_2 */
  double eps_optimal_absolute;
  double eps_optimal_relative;
  double time_sec_limit;              /* +inf for none */
  int32_t iteration_limit;            /* INT32_MAX for none */
  double kkt_matrix_pass_limit;       /* +inf for none */
} pdot_termination_criteria;

/* RestartParameters, src/saddle_point_gpu.jl:411-441 (same field order) */
typedef struct pdot_restart_parameters {
  int32_t restart_scheme;             /* PDOT_NO_RESTARTS / FIXED_FREQUENCY / ADAPTIVE_KKT */
  int32_t restart_to_current_metric;  /* PDOT_NO_RESTART_TO_CURRENT / PDOT_KKT_GREEDY */
  int64_t restart_frequency_if_fixed;
  double artificial_restart_threshold;
  double sufficient_reduction_for_restart;
  double necessary_reduction_for_restart;
  double primal_weight_update_smoothing;
} pdot_restart_parameters;

/* PdhgParameters, src/solver_gpu.jl:9-21 (same field order; the
 * Union{AdaptiveStepsizeParams, ConstantStepsizeParams} is a tag plus the
 * AdaptiveStepsizeParams fields, src/solver_gpu.jl:2-7) */
typedef struct pdot_pdhg_parameters {
  double primal_importance;
  int32_t scale_invariant_initial_primal_weight;  /* Bool */
  int64_t verbosity;                              /* printing is left to the host language */
  int32_t record_iteration_stats;                 /* Bool */
  int32_t termination_evaluation_frequency;
  pdot_termination_criteria termination_criteria;
  pdot_restart_parameters restart_params;
  int32_t step_size_policy;                       /* PDOT_STEP_SIZE_ADAPTIVE / _CONSTANT */
  double reduction_exponent;                      /* AdaptiveStepsizeParams */
  double growth_exponent;                         /* AdaptiveStepsizeParams */
} pdot_pdhg_parameters;

/* Options of this implementation that have no counterpart in the reference.
 * Pass NULL for the defaults: device 0, the FP64 drop-in, CUDA graphs on. */
enum { PDOT_PRECISION_F64 = 0, PDOT_PRECISION_F32 = 1 };
enum {
  PDOT_COST_F64 = 0,              /* the problem's FP64 cost matrix, as given */
  PDOT_COST_F32 = 1,              /* stored in FP32 (converted on the device) */
  PDOT_COST_BF16 = 2,             /* stored in BF16 (converted on the device) */
  PDOT_COST_SQEUCLID_POINTS = 3,  /* C_ij = scale*||x_i - y_j||^2 computed on the fly
                                   * from FP32 coordinates; cost_matrix may be NULL */
  PDOT_COST_L1_POINTS = 4         /* C_ij = scale*||x_i - y_j||_1, likewise */
};
/* How the fused primal pass reads its operands: with direct 16-byte vector
 * loads, or staged through shared memory by bulk copies with an mbarrier per
 * stage (where the buffers are 16-byte aligned). PDOT_PASS_AUTO picks the one
 * measured faster on B200: staged for BF16 and coordinate costs, direct for
 * FP64 and FP32 costs. */
enum { PDOT_PASS_AUTO = 0, PDOT_PASS_STAGED = 1, PDOT_PASS_DIRECT = 2 };
typedef struct pdot_solver_options {
  int32_t device;                     /* CUDA device ordinal */
  int32_t use_cuda_graph;             /* 1: replay captured iteration chunks */
  int32_t time_kernels;               /* 1: CUDA events around every launch (direct launches) */
  int32_t plan_precision;             /* PDOT_PRECISION_F64 (drop-in) or _F32 (mixed precision) */
  int32_t cost_storage;               /* PDOT_COST_*; anything but F64 needs plan_precision F32 */
  int32_t point_dim;                  /* 1..4, for the coordinate costs */
  const float* source_points;         /* m x point_dim, row-major (same memory kind as the problem) */
  const float* target_points;         /* n x point_dim, row-major */
  double cost_scale;                  /* > 0: the scale; <= 0: 1 / max_ij of the distance */
  const double* warm_dual_source;     /* m initial source duals, or NULL (zero start) */
  const double* warm_dual_target;     /* n initial target duals, or NULL */
  int32_t primal_pass;                /* PDOT_PASS_AUTO, _STAGED or _DIRECT */
  int32_t ctas_per_sm;                /* batched solver: CTAs per SM of its matrix passes (0 = most) */
  const double* warm_primal;          /* m x n column-major initial plan (needs the warm duals), or NULL */
  /* > 0 with warm duals and no warm plan: the plan is recovered from the duals
   * by warm_plan_iterations rounds of log-domain row/column balancing of
   * exp((u_i + v_j - C_ij) / eps) (0 rounds: that kernel as it is) */
  double warm_plan_epsilon;
  int32_t warm_plan_iterations;
  /* Test hook, 0 in normal use. 1: each consumer wait of the staged fused pass
   * reports a timeout without polling; the kernel still waits (bounded) for the
   * copies it has in flight, sets its error word and returns, and the call
   * fails with PDOT_ERR_CUDA. It exercises the timeout path without a fault. */
  int32_t fail_bounded_waits;
  /* With a warm start: 0 (default) starts the restart information (the last
   * restart point of the adaptive restart test and of the primal-weight
   * update) at the warm point, as the reference starts it at its initial
   * point; 1 starts it at the zero point, as a cold start's. */
  int32_t warm_restart_at_zero;
  /* > 0 with warm-start duals: the initial primal weight, in place of
   * primal_importance (or the scale-invariant choice); <= 0: that choice. */
  double warm_primal_weight;
  /* Batched solver: its matrix passes cut the units (one column of one
   * 256-row panel) of all active instances into CTA ranges of equal cost, a
   * unit costing its rows plus batch_unit_cost * 256 (the per-unit overhead,
   * 0..8, in eighths). 0 balances the rows alone. */
  double batch_unit_cost;
  /* Regular chunks of loop bodies (the evaluation and the steps up to the next
   * one) as one persistent cooperative launch with grid barriers between the
   * phases, instead of a CUDA graph of separate launches; the results are
   * bit-identical. 0: automatic (the CUDA graph, which measured faster on
   * B200), 1: whenever the direct 16-byte pass runs, -1: never. The batched
   * solver takes it too: 1 runs its regular chunks (evaluation, compaction,
   * steps) as one persistent launch with the direct pass throughout (the
   * staged pass is then refused). */
  int32_t persistent_chunks;
  /* Batched solver: the rows of one panel of its matrix passes' tiles (a unit
   * is one column of one panel): 256 or 128, 0 = 256. A 128-row tile holds
   * half the registers per thread, so three CTAs per SM are resident where a
   * 256-row tile allows two, at twice the units of tall instances;
   * pdot.tune_batched picks the tile. */
  int32_t batch_panel_rows;
} pdot_solver_options;

/* ---- output -------------------------------------------------------------- */
/* ConvergenceInformation, src/solve_log.jl:47-147 (same field order) */
typedef struct pdot_convergence_information {
  int32_t candidate_type;             /* PointType */
  double primal_objective;
  double dual_objective;
  double corrected_dual_objective;
  double l_inf_primal_residual;
  double l2_primal_residual;
  double l_inf_dual_residual;
  double l2_dual_residual;
  double relative_l_inf_primal_residual;
  double relative_l2_primal_residual;
  double relative_l_inf_dual_residual;
  double relative_l2_dual_residual;
  double relative_optimality_gap;
  double l_inf_primal_variable;
  double l2_primal_variable;
  double l_inf_dual_variable;
  double l2_dual_variable;
} pdot_convergence_information;

/* IterationStats, src/solve_log.jl:154-228 (same field order; the single
 * ConvergenceInformation the reference stores is inlined and the one
 * method-specific stat the reference records, src/solver_gpu.jl:579-581, is a
 * field) */
typedef struct pdot_iteration_stats {
  int32_t iteration_number;
  pdot_convergence_information convergence_information;
  double cumulative_kkt_matrix_passes;
  int32_t cumulative_rejected_steps;
  double cumulative_time_sec;
  int32_t restart_used;               /* RestartChoice */
  double step_size;
  double primal_weight;
  double time_spent_doing_basic_algorithm;
} pdot_iteration_stats;

/* SaddlePointOutput, src/saddle_point_gpu.jl:2-34. The caller owns every
 * array. A NULL solution pointer skips that copy. */
typedef struct pdot_saddle_point_output {
  double* primal_solution;            /* m*n column-major, or NULL */
  double* dual_source_solution;       /* m, or NULL */
  double* dual_target_solution;       /* n, or NULL */
  pdot_iteration_stats* iteration_stats; /* capacity records, or NULL */
  int64_t iteration_stats_capacity;
  int64_t iteration_stats_count;      /* out: records produced (can exceed capacity) */
  int32_t termination_reason;         /* out: TerminationReason */
  int32_t iteration_count;            /* out: iterations, src/solver_gpu.jl:661 */
  double solve_time_sec;              /* out: cumulative_time_sec of the last record */
  pdot_iteration_stats final_stats;   /* out: the record that ended the solve */
} pdot_saddle_point_output;

/* ---- solver entry points ------------------------------------------------- */

/* Library identity. Returns PDOT_ABI_VERSION. */
int pdot_version(void);

/* Thread-local description of the last error on this thread ("" if none). */
const char* pdot_last_error(void);

/* Replaces PDOT.optimize(params, problem), src/solver_gpu.jl:413-720, with
 * the host->device copy of src/io.jl:18-36 and the device->host copy of
 * src/io.jl:41-53 inside. Parameter validation follows
 * src/solver_gpu.jl:420-422 and src/saddle_point_gpu.jl:455-461 and returns
 * PDOT_ERR_INVALID_ARGUMENT where the reference raises. `options` may be NULL. */
int pdot_optimize(const pdot_problem* problem,
                  const pdot_pdhg_parameters* params,
                  const pdot_solver_options* options,
                  pdot_saddle_point_output* output);

/* Fills `params` with the values scripts/solve.jl:58-86 uses
 * (ADAPTIVE_KKT, KKT_GREEDY, 1000, 0.36, 0.1, 0.9, 0.5; L_2; eps = tolerance;
 * primal_importance 1.0; record stats; evaluation every 128 iterations;
 * AdaptiveStepsizeParams(2, 1)). */
void pdot_default_parameters(double tolerance, pdot_pdhg_parameters* params);

/* ---- solver objects ------------------------------------------------------
 * A solver holds one problem on the device and the state of optimize()'s
 * loop, so that a caller can reuse the device copy (the warm-up solve of
 * scripts/solve.jl:123-126 followed by the real solve) and advance the loop in
 * pieces. pdot_optimize is create + finish + destroy. */
typedef struct pdot_solver pdot_solver;

typedef struct pdot_solver_status {
  int64_t iteration;                  /* number of the next loop body (1 at the start) */
  int64_t total_number_iterations;    /* solver_state.total_number_iterations */
  int32_t done;                       /* 1 once a termination reason is set */
  int32_t termination_reason;
  double step_size;
  double primal_weight;
  double cumulative_kkt_matrix_passes;
  int64_t iteration_stats_count;      /* records produced so far */
  int64_t primal_passes;              /* fused primal passes run (accepted steps) */
  int64_t primal_passes_fresh_average;/* of those, passes that started a new average */
  /* device time per kernel family, accumulated while options->time_kernels */
  int64_t timed_primal_passes;
  double primal_pass_ms;
  double dual_step_ms;
  double evaluation_ms;
} pdot_solver_status;

/* Copies the host problem to `options->device` and prepares the loop. */
int pdot_solver_create(const pdot_problem* problem, const pdot_pdhg_parameters* params,
                       const pdot_solver_options* options, pdot_solver** solver);
/* Same, but the problem's three arrays are device pointers on
 * options->device, read in place (they must outlive the solver). */
int pdot_solver_create_device(const pdot_problem* device_problem, const pdot_pdhg_parameters* params,
                              const pdot_solver_options* options, pdot_solver** solver);
/* Back to the state optimize() starts from (iteration 1, zero iterates). */
int pdot_solver_reset(pdot_solver* solver);
/* Runs up to `max_iterations` more loop bodies of optimize() (fewer if it
 * terminates) and waits for them; `status` may be NULL. */
int pdot_solver_iterate(pdot_solver* solver, int64_t max_iterations, pdot_solver_status* status);
/* Runs to termination and fills `output` like pdot_optimize. */
int pdot_solver_finish(pdot_solver* solver, pdot_saddle_point_output* output);
/* The CUDA stream (cudaStream_t) all of the solver's work is issued on. */
void* pdot_solver_stream(pdot_solver* solver);
void pdot_solver_destroy(pdot_solver* solver);

/* ---- device-level entry points of the hot path --------------------------- */
/* These act on device memory (pointers from cudaMalloc or torch) and on the
 * given CUDA stream (NULL = legacy default stream); they are the per-iteration
 * building blocks that pdot_optimize chains. */

/* One fused primal pass, replacing compute_next_primal_solution_kernel! plus
 * the two `sum(delta_primal; dims)` reductions (src/solver_gpu.jl:125-174),
 * `current_primal_solution .+= delta_primal` (src/solver_gpu.jl:242), the
 * gradient refresh (src/solver_gpu.jl:249-250, recomputed on the fly from
 * C, u, v instead of stored) and the primal weighted average
 * (src/saddle_point_gpu.jl:115-135). For every entry:
 *     g    = (C - u[i]) - v[j]                (g = 0 if flags & PDOT_PASS_ZERO_GRADIENT)
 *     p    = max(X - step_over_weight*g, 0)
 *     d    = p - X;   X <- X + d
 *     Xavg <- (Xavg + X*avg_new_weight)*avg_scale   (Xavg <- X if flags & PDOT_PASS_FIRST_AVERAGE)
 * and it returns delta_row_sum[i] = sum_j d, delta_col_sum[j] = sum_i d and
 * delta_sq_norm[0] = sum d^2. Reductions are deterministic (fixed order).
 * `workspace` must hold pdot_primal_pass_workspace_bytes(m, n) bytes. */
enum { PDOT_PASS_ZERO_GRADIENT = 1, PDOT_PASS_FIRST_AVERAGE = 2 };
int64_t pdot_primal_pass_workspace_bytes(int64_t m, int64_t n);
int pdot_primal_pass_f64(int64_t m, int64_t n,
                         const double* cost, double* primal, double* primal_avg,
                         const double* dual_source, const double* dual_target,
                         double step_over_weight, double avg_new_weight, double avg_scale,
                         int32_t flags,
                         double* delta_row_sum, double* delta_col_sum, double* delta_sq_norm,
                         void* workspace, int64_t workspace_bytes, void* stream);

/* ---- batched solver -------------------------------------------------------
 * Many independent instances of uneven sizes in one solve: each runs
 * optimize()'s loop with its own step size, primal weight, restarts and
 * termination (the instances advance in lockstep, one loop body each per
 * global iteration, and finished ones drop out). Plans are FP32 and the
 * cost is stored FP32 (options->cost_storage = PDOT_COST_F32, converted from
 * the FP64 matrices) or computed from FP32 coordinates (PDOT_COST_SQEUCLID_POINTS
 * or PDOT_COST_L1_POINTS, point_dim 1..3, each instance normalised by its own
 * maximum). options->plan_precision must be PDOT_PRECISION_F32. */
typedef struct pdot_batch_problem {
  int64_t num_instances;
  const int64_t* num_rows;                  /* m of each instance */
  const int64_t* num_cols;                  /* n of each instance */
  const double* const* cost_matrices;       /* column-major host matrices, or NULL for coordinates */
  const double* const* source_distributions;
  const double* const* target_distributions;
  const float* const* source_points;        /* m x point_dim, row-major, or NULL */
  const float* const* target_points;        /* n x point_dim */
  /* Warm starts (NULL arrays, or NULL entries, start that instance at zero):
   * initial duals and, optionally, an initial plan (column-major, m x n). */
  const double* const* warm_dual_sources;
  const double* const* warm_dual_targets;
  const double* const* warm_primals;
  /* Racing (NULL: none): race_groups[k] in 0..num_instances-1, or -1. Once an
   * instance ends optimal, the other members of its group stop with
   * PDOT_TERMINATION_REASON_OTHER at the same evaluation; a warm start and a
   * cold start of one problem raced this way finish as soon as the faster one. */
  const int32_t* race_groups;
  /* Initial primal weights of warm instances (NULL, or entries <= 0: the
   * parameters' choice), like pdot_solver_options.warm_primal_weight. */
  const double* warm_primal_weights;
} pdot_batch_problem;

typedef struct pdot_batch_output {          /* one per instance; arrays may be NULL */
  double* primal_solution;                  /* m*n column-major (the returned average, widened) */
  double* dual_source_solution;             /* m */
  double* dual_target_solution;             /* n */
  int32_t termination_reason;
  int32_t iteration_count;
  pdot_iteration_stats final_stats;         /* the evaluation that ended this instance */
} pdot_batch_output;

/* `solve_seconds` (may be NULL) receives the device time of the solve. */
int pdot_optimize_batched(const pdot_batch_problem* problem, const pdot_pdhg_parameters* params,
                          const pdot_solver_options* options, pdot_batch_output* outputs,
                          double* solve_seconds);

/* ---- passes around a solve ------------------------------------------------ */

/* The feasibility rounding of a plan, src/utils_gpu.jl:296-318 (the reference
 * runs it on the CPU after the solve; scripts/solve.jl:116-117 writes its
 * result): rows scaled by min(1, a/rowsum), columns by min(1, b/colsum), then
 * X += err_r err_c^T with err_r = (a - rowsum)/||a - rowsum||_1. In place, on
 * device arrays and the given stream. */
int pdot_rounding_f64(int64_t m, int64_t n, const double* source, const double* target, double* plan,
                      void* stream);
/* The same on host arrays (copied to `device` and back). */
int pdot_rounding_host(int64_t m, int64_t n, const double* source, const double* target, double* plan,
                       int32_t device);

/* C_ij = ||x_i - y_j||^2 (divided by its maximum if `normalise`) into a device
 * cost matrix (column-major, ld = m) from device FP64 coordinates (m x dim and
 * n x dim, row-major): builds the problem where it is solved instead of
 * copying m*n doubles to the device. */
int pdot_sqeuclid_cost_f64(int64_t m, int64_t n, int32_t dim, const double* source_points,
                           const double* target_points, int32_t normalise, double* cost, void* stream);

/* ---- the coarse-to-fine warm start for point clouds -----------------------
 * Device passes of pdot/multiscale.py (no counterpart in the reference, which
 * always starts at zero, src/solver_gpu.jl:428-441). Points are FP32, row-major
 * (one point per row, dim 1..3), in device memory; work is ordered on `stream`. */
/* out[0] = max_ij ||x_i - y_j||^2 (FP64), the normaliser of the squared-Euclidean
 * cost (`out` is device memory). */
int pdot_points_max_sqdist(int64_t m, int64_t n, int32_t dim, const float* source_points,
                           const float* target_points, double* out, void* stream);
/* The semi-discrete c-transform out_i = min_J (scale * ||p_i - c_J||^2 - dual_J):
 * duals known on num_centres points (FP64 centres, num_centres x dim, row-major)
 * extended to every point p_i. */
int pdot_points_c_transform(int64_t num_points, int64_t num_centres, int32_t dim, const float* points,
                            const double* centres, const double* duals, double scale, double* out,
                            void* stream);

/* The same fused primal pass for callers that cannot allocate device memory
 * (a host framework that hands out its whole memory budget from its own pool,
 * or a latency-critical loop that cannot afford cudaMalloc's implicit device
 * synchronisation). It has no counterpart in the reference. Its scratch is a
 * fixed PDOT_NOALLOC_SCRATCH_BYTES array inside the library (held by every GPU
 * that loads it until exit), so the call allocates nothing; sizes whose
 * scratch would exceed it return PDOT_ERR_TOO_LARGE. Every call looks up the
 * array's device address on the current device; the first call on a device
 * loads the library's module there: make it before any stream capture. Calls
 * share the array: calls that overlap on the GPU race. */
#define PDOT_NOALLOC_SCRATCH_BYTES (16u << 20)
int pdot_primal_pass_f64_noalloc(int64_t m, int64_t n,
                                 const double* cost, double* primal, double* primal_avg,
                                 const double* dual_source, const double* dual_target,
                                 double step_over_weight, double avg_new_weight, double avg_scale,
                                 int32_t flags,
                                 double* delta_row_sum, double* delta_col_sum, double* delta_sq_norm,
                                 void* stream);

/* ---- the learned warm start ---------------------------------------------
 * A small MLP predicts optimal dual potentials from the marginals; its warm
 * start is finished by plain PDHG (pdot_solver_options.warm_dual_*). It has no
 * counterpart in the reference. Layers input -> hidden -> hidden -> output
 * with GELU; BF16 weights and activations, FP32 master weights, AdamW moments
 * and accumulation; every product on the tensor cores (tcgen05). Widths are
 * multiples of 128. Parameters are laid out W1 [hidden x input] (row-major),
 * b1, W2 [hidden x hidden], b2, W3 [output x hidden], b3. Device pointers are
 * on the network's device; calls are ordered on pdot_mlp_stream. */
typedef struct pdot_mlp pdot_mlp;
int pdot_mlp_create(int32_t device, int64_t input_dim, int64_t hidden_dim, int64_t output_dim,
                    int64_t max_batch, uint64_t seed, pdot_mlp** out);
int pdot_mlp_destroy(pdot_mlp* net);
int64_t pdot_mlp_num_parameters(const pdot_mlp* net);
void* pdot_mlp_stream(pdot_mlp* net);
int pdot_mlp_get_parameters(pdot_mlp* net, float* host, int64_t count);
int pdot_mlp_set_parameters(pdot_mlp* net, const float* host, int64_t count);  /* resets AdamW */
int pdot_mlp_get_gradients(pdot_mlp* net, float* host, int64_t count);
/* The input rows: x = bf16((log(max(h, 1e-30)) + shift) * scale) of the
 * device array histograms [batch x input_dim] (row-major, FP64). */
int pdot_mlp_set_input(pdot_mlp* net, int64_t batch, const double* histograms, double shift, double scale);
/* Y = the network's output for the input rows; copied to `out` (device,
 * batch x output_dim) when not NULL. */
int pdot_mlp_forward(pdot_mlp* net, float* out);
/* After pdot_mlp_forward: the gradients of the mean squared error against the
 * device array target [batch x output_dim]; the loss to *loss when not NULL. */
int pdot_mlp_backward(pdot_mlp* net, const float* target, double* loss);
int pdot_mlp_adamw(pdot_mlp* net, float lr, float beta1, float beta2, float eps, float weight_decay);
/* forward + backward + AdamW(beta1 0.9, beta2 0.999, eps 1e-8) */
int pdot_mlp_train_step(pdot_mlp* net, const float* target, float lr, float weight_decay, double* loss);

#ifdef __cplusplus
}
#endif

#endif /* PDOT_H */
