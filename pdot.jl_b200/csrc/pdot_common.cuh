// pdot_common.cuh — shared declarations of the sm_100a PDHG-for-OT solver.
//
// Data layout in HBM (one solve):
//   C          m x n, column-major (entry (i,j) at i + j*m), read-only; FP64
//              in the drop-in, FP32 or BF16 in mixed precision, or absent when
//              the squared-Euclidean cost is computed from FP32 coordinates
//   X[2]       two m x n plans (FP64 drop-in, FP32 mixed precision): X[buf] is
//              the current iterate, X[1-buf] the running weighted average. A
//              restart to the average flips `buf`, so restarts copy nothing.
//   u[2] v[2]  source/target duals (current / average), FP64
//   r[2] c[2]  row / column sums of the plan (current / average), FP64
//   partials   per-CTA and per-(panel, column) partial sums; reductions are
//              two-stage with a fixed order, so results are bitwise repeatable.
//
// Work decomposition of the matrix passes: the rows are cut into panels of
// kPanelRows; a "unit" is one column of one panel (kPanelRows contiguous
// doubles). Units are numbered panel-major (q = p*n + j) and CTA c owns the
// contiguous range [c*U/G, (c+1)*U/G): every CTA streams the same number of
// bytes. A warp handles a whole unit, so a column's partial sum is a warp
// shuffle; row sums accumulate per lane across the units of a panel and are
// combined across warps in shared memory when the panel ends.
#pragma once

#include <cstdint>
#include <functional>
#include <cuda_runtime.h>

#include "pdot.h"

namespace pdot {

constexpr int kThreads = 256;              // CTA size of the matrix passes
constexpr int kWarps = kThreads / 32;
constexpr int kPanelRows = 256;            // rows per panel (one unit = 256 doubles)
constexpr int kVecThreads = 256;           // CTA size of the vector passes
constexpr int kEvalSums = 10;              // per-CTA partials of the eval matrix pass
constexpr int kVecSums = 10;               // per-CTA partials of the eval vector pass
constexpr int kStepSums = 2;               // per-CTA partials of the dual step
constexpr int kNormSums = 2;               // per-CTA partials of the cost-norm pass

struct Geometry {
  int64_t m, n;
  int64_t panels;      // P = ceil(m / kPanelRows)
  int64_t units;       // U = P * n
  int32_t grid;        // CTAs of the matrix passes (<= U)
  int32_t vec;         // rows per lane load: 16 B / sizeof(plan element), or 1
  int32_t row_blocks;  // CTAs of the vector passes covering m
  int32_t col_blocks;  // CTAs of the vector passes covering n
  int32_t plan_f32;    // 1: FP32 plan and average, 0: FP64
  int32_t cost_kind;   // PDOT_COST_F64 / _F32 / _BF16, or a coordinate kind (internal_cost_kind)
  int32_t tma;         // 1: the fused pass stages its operands with bulk copies
  int32_t tma_smem;    // dynamic shared memory of the staged pass (bytes)
  int32_t fail_waits;  // test hook: the staged pass's consumer waits report a timeout at once
  // CTAs of the dual step covering the rows: row_blocks (a thread per row) or,
  // when a panel's row partials lie in many CTA slots (small problems, kDualWarpSlots
  // or more), ceil(m / kWarps) (a warp per row)
  int32_t dual_row_blocks;
  // CTAs of the persistent chunk kernel (all co-resident; each runs the CTA
  // ranges grid / chunk_ctas of the matrix passes in turn), 0: not available
  int32_t chunk_ctas;
};
constexpr int kDualWarpSlots = 16;

// Where the cost entries come from.
struct CostSource {
  const void* C;       // PDOT_COST_F64 / F32 / BF16 storage
  const float* xs;     // PDOT_COST_SQEUCLID_POINTS: m x dim source points
  const float* ys;     // n x dim target points
  int dim;             // 1..kMaxPointDim
};
constexpr int kMaxPointDim = 4;
// Internal cost kinds: the stored PDOT_COST_* values, kCostSqBase + dim for the
// squared-Euclidean coordinate cost and kCostL1Base + dim for the L1 one (the
// point dimension is a compile-time constant of the kernels).
constexpr int kCostSqBase = 10;
constexpr int kCostL1Base = 20;
__host__ __device__ constexpr bool is_sq_cost(int kind) {
  return kind > kCostSqBase && kind <= kCostSqBase + kMaxPointDim;
}
__host__ __device__ constexpr bool is_l1_cost(int kind) {
  return kind > kCostL1Base && kind <= kCostL1Base + kMaxPointDim;
}
__host__ __device__ constexpr bool is_point_cost(int kind) { return is_sq_cost(kind) || is_l1_cost(kind); }
// The internal kind of a public PDOT_COST_* with points of dimension `dim`.
__host__ __device__ constexpr int internal_cost_kind(int pub, int dim) {
  return pub == PDOT_COST_SQEUCLID_POINTS ? kCostSqBase + dim : (pub == PDOT_COST_L1_POINTS ? kCostL1Base + dim : pub);
}

__host__ __device__ __forceinline__ int64_t unit_begin(const Geometry& g, int64_t cta) {
  return cta * g.units / g.grid;
}
// The CTA whose unit range holds unit q (the largest c with unit_begin(c) <= q).
__host__ __device__ __forceinline__ int64_t cta_of_unit(const Geometry& g, int64_t q) {
  return ((q + 1) * (int64_t)g.grid - 1) / g.units;
}
// Row partials of CTA c for panel p live in slot c + p: along the unit line,
// both c and p are non-decreasing and one of them grows at every boundary, so
// the slot is unique. There are at most grid + panels slots.
__host__ __device__ __forceinline__ int64_t row_slot(int64_t cta, int64_t panel) { return cta + panel; }

// Solver state in device memory. Every per-iteration decision is taken on the
// device, so the host only reads this record between replayed chunks.
struct DevState {
  double step_size;          // solver_state.step_size (tau)
  double primal_weight;      // solver_state.primal_weight (omega)
  double kkt_passes;         // solver_state.cumulative_kkt_passes
  double sum_weights;        // sum of averaging weights (all averages share it)
  long long avg_count;       // primal_solutions_count
  long long total_iters;     // solver_state.total_number_iterations
  long long iteration;       // number of the next loop body of optimize()
  // last restart point (saddle_point_gpu.jl:332-366 reduced to scalars)
  double last_rp;            // its l2 primal residual
  double last_rd;            // its l2 dual residual
  double last_gap;           // |primal obj - dual obj|
  double last_xnorm;         // ||X_last||_2
  double last_ynorm;         // ||[u_last; v_last]||_2
  double ratio_last_trial;   // kkt_reduction_ratio_last_trial
  long long last_restart_length;
  double pdist, ddist;       // distances moved in the last restart period
  // cached_ot_info, termination.jl:87-92
  double linf_obj, linf_rhs, l2_obj, l2_rhs;
  double cost_scale;         // PDOT_COST_SQEUCLID_POINTS: C = scale * ||x - y||^2
  // timing (globaltimer ns)
  unsigned long long t_start_ns;
  unsigned long long eval_t0_ns;
  double eval_time_sec;      // device time spent in evaluations
  long long num_stats;       // iteration-stats records written
  long long primal_passes;   // fused primal passes that ran
  long long fresh_passes;    // of those, passes that started a new average
  long long xsums_iter;      // loop body whose primal pass left the next evaluation's plan sums (-1: none)
  int numerical_error;
  int g_is_zero;             // the stored gradient is still its initial 0
  int done;
  int termination_reason;
  int buf;                   // which half of each pair is the current iterate
  int out_current;           // at termination: 1 = return current, 0 = average
  int last_restart_choice;
  int kernel_error;          // non-zero: a bounded wait in a kernel timed out
  unsigned int ticket_step;  // last-CTA tickets
  unsigned int ticket_eval;
  unsigned int ticket_init;
  unsigned int bar_count;    // grid barrier of the persistent chunk kernel: arrivals
  unsigned int bar_gen;      // and generation
  int pad_[1];
};

// Parameters of one solve, passed by value to the control kernels.
struct SolveConfig {
  int adaptive;
  double reduction_exponent, growth_exponent;
  int restart_scheme, restart_to_current_metric;
  long long restart_frequency_if_fixed;
  double artificial_restart_threshold;
  double sufficient_reduction_for_restart;
  double necessary_reduction_for_restart;
  double primal_weight_update_smoothing;
  int optimality_norm;
  double eps_abs, eps_rel, time_sec_limit;
  long long iteration_limit;
  double kkt_matrix_pass_limit;
  int record_iteration_stats;
  int scale_invariant_initial_primal_weight;
  double primal_importance;
  double cost_scale;         // given scale (> 0) or 0: normalise by the max
  int warm_start;            // duals were given: the stored gradient is C - u - v
  double warm_primal_weight; // > 0 with a warm start: the initial primal weight
};

struct Buffers {
  CostSource cost;
  const double* a;
  const double* b;
  void* X[2];        // double (FP64 plan) or float (FP32 plan)
  double* u[2];
  double* v[2];
  double* r[2];
  double* c[2];
  double* rowpart;   // (grid + panels) * kPanelRows
  double* colpart;   // panels * n
  double* sqpart;    // grid
  double* steppart;  // (row_blocks + col_blocks) * kStepSums
  double* evpart;    // grid * kEvalSums
  double* vecpart;   // (row_blocks + col_blocks) * kVecSums
  pdot_iteration_stats* ring;
  int ring_cap;
  DevState* st;
};

// ---- launchers (pdot_kernels.cu) ----------------------------------------
// vec_ok: the cost and plan buffers are 16-byte aligned (vector and staged
// paths allowed); staged_ok: the fused pass may use the bulk-copy staging.
Geometry make_geometry(int64_t m, int64_t n, int vec_ok, int device, int plan_f32 = 0,
                       int cost_kind = PDOT_COST_F64, int staged_ok = 0);
size_t workspace_doubles(const Geometry& g);
// Scratch of the stand-alone primal pass (launch_primal_pass): its row
// partials, column partials and per-CTA sums of squares, in that order.
inline size_t pass_scratch_doubles(const Geometry& g) {
  return ((size_t)g.grid + g.panels) * kPanelRows + (size_t)g.panels * g.n + (size_t)g.grid;
}

cudaError_t launch_init(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s);
// xsums = 1: the next loop body evaluates; the direct pass also leaves that
// evaluation's plan sums (k1_primal_xs), so the evaluation reads only the cost
// (the staged pass ignores it and the evaluation reads the plans).
cudaError_t launch_primal(const Buffers& B, const Geometry& g, cudaStream_t s, int xsums = 0);
cudaError_t launch_dual(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s);
cudaError_t launch_step(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s,
                        int xsums = 0);
// One regular chunk (evaluation, then `steps` steps, the last with xsums) as
// one persistent cooperative launch (needs g.chunk_ctas > 0); bit-identical to
// launch_eval followed by the steps.
cudaError_t launch_chunk(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s, int steps);
// start_only = 1: a warm start's initial point becomes the last restart
// point; nothing else of the evaluation block runs.
cudaError_t launch_eval(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s,
                        int start_only = 0);

// Conversions used by the host: FP64 cost to its stored precision, and an
// FP32 plan widened to FP64 for the caller.
cudaError_t launch_convert_cost(const double* src, void* dst, int cost_kind, size_t count, cudaStream_t s);
cudaError_t launch_widen(const float* src, double* dst, size_t count, cudaStream_t s);

// Passes around a solve (pdot_aux.cu).
size_t plan_sums_workspace_doubles(int64_t m, int64_t n);
// r = X 1 and c = X^T 1 of an m x n column-major plan (FP32 when plan_f32)
cudaError_t launch_plan_sums(int64_t m, int64_t n, const void* X, int plan_f32, double* r, double* c, double* work,
                             cudaStream_t s);
size_t rounding_workspace_doubles(int64_t m, int64_t n);
cudaError_t launch_rounding(int64_t m, int64_t n, const double* a, const double* b, double* X, double* work,
                            cudaStream_t s);
size_t sqeuclid_workspace_doubles();
cudaError_t launch_sqeuclid_cost(int64_t m, int64_t n, int dim, const double* xs, const double* ys, int normalise,
                                 double* C, double* work, cudaStream_t s);

// A warm-start plan recovered from warm duals (pdot_warmplan.cu), for one
// instance or the concatenated instances of the batched solver.
struct PlanInstance {
  int64_t m, n, ld;  // rows, columns, leading dimension of the plan (and stored cost)
  int64_t x_off;     // offset of the plan and of the stored cost (elements)
  int64_t row_off;   // offset of the row vectors and source points (rows)
  int64_t col_off;   // offset of the column vectors and target points (columns)
  int active;        // 1: recover this instance's plan
  int pad_;
};
struct WarmPlanArgs {
  const PlanInstance* inst;     // num (device)
  int num;
  const long long* row_prefix;  // num + 1: instance k owns global rows [row_prefix[k], row_prefix[k+1])
  const long long* col_prefix;  // num + 1
  long long total_rows, total_cols;
  int kind;                     // internal cost kind
  int dim;                      // point dimension of the coordinate costs
  const void* C;
  const float* xs;
  const float* ys;
  const DevState* st;           // per instance: cost_scale
  const double *a, *b, *u0, *v0;
  double *f, *g;                // balanced potentials (work, total rows / columns)
  void* X;                      // the plans (FP32 when plan_f32)
  int plan_f32;
  double *r, *c;                // their row and column sums
  double eps;
};
cudaError_t launch_warm_plan(const WarmPlanArgs& A, int iterations, cudaStream_t s);

// Large host <-> device copies (pdot_transfer.cu): one DMA for page-locked host
// memory, a two-buffer pinned staging pipeline with parallel host copies for
// pageable memory. copy_to_host returns after the copy has completed;
// copy_to_device may return with a copy from page-locked memory still queued
// on `s` (the source must stay valid until `s` is synchronised).
constexpr size_t kTransferChunk = size_t(8) << 20;  // doubles per staged chunk (64 MiB)
bool host_is_pinned(const void* p);
cudaError_t copy_to_device(void* dst, const void* src, size_t bytes, cudaStream_t s);
// The device data of `count` doubles from element `off` of the array being
// copied out: the device address, after enqueueing on `s` whatever makes it
// ready (at most kTransferChunk doubles; `slot` alternates 0 / 1 between
// consecutive chunks, so a producer can double-buffer its own scratch).
using ChunkSource = std::function<const double*(size_t off, size_t count, int slot, cudaStream_t s)>;
cudaError_t copy_to_host(double* dst, size_t count, const ChunkSource& source, cudaStream_t s);

// Sets the thread-local text pdot_last_error() returns (pdot_host.cu).
void set_last_error(const char* msg);

// Stand-alone primal pass on caller buffers (pdot_primal_pass_f64).
cudaError_t launch_primal_pass(const Geometry& g, const double* C, double* X, double* Xa,
                               const double* u, const double* v, double step_over_weight,
                               double avg_new_weight, double avg_scale, int flags,
                               double* drow, double* dcol, double* dsq, double* work,
                               cudaStream_t s);

}  // namespace pdot
