// pdot_host.cu — C ABI of libpdot.so and the host orchestration of a solve.
//
// pdot_optimize replaces PDOT.optimize (src/solver_gpu.jl:413-720). The host
// copies the problem to the device once (src/io.jl:18-36), launches the init
// kernel, then enqueues the loop of optimize() as device work: per iteration
// an optional evaluation (k3 + k4) and a step (k1 + k2). Iterations are
// grouped in chunks of termination_evaluation_frequency iterations; the
// regular chunk [eval, step x freq] is captured once as a CUDA graph and
// replayed. Two chunks are kept in flight; after each one the host reads the
// device state record (a 200-byte copy) and the new iteration-stats records,
// and stops once the device has set `done`. All decisions (step size, restart,
// primal weight, termination) are taken on the device.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "pdot_common.cuh"

namespace {

thread_local std::string g_last_error;

struct Failure {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Failure{code, buf};
}

void check_cuda(cudaError_t e, const char* what, int line) {
  if (e != cudaSuccess) {
    const int code = (e == cudaErrorMemoryAllocation) ? PDOT_ERR_OUT_OF_MEMORY : PDOT_ERR_CUDA;
    cudaGetLastError();  // clear a sticky-free error
    fail(code, "%s failed: %s (pdot_host.cu:%d)", what, cudaGetErrorString(e), line);
  }
}
#define CK(x) check_cuda((x), #x, __LINE__)

template <typename F>
int guarded(F&& f) {
  try {
    g_last_error.clear();
    f();
    return PDOT_OK;
  } catch (const Failure& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return PDOT_ERR_OUT_OF_MEMORY;
  } catch (...) {
    g_last_error = "unexpected C++ exception";
    return PDOT_ERR_CUDA;
  }
}

void require_sm100(int device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
    cudaGetLastError();
    fail(PDOT_ERR_NO_DEVICE, "no CUDA device is visible");
  }
  if (device < 0 || device >= count) fail(PDOT_ERR_INVALID_ARGUMENT, "device %d out of range (%d visible)", device, count);
  int major = 0, minor = 0;
  CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  CK(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
  if (major != 10 || minor != 0)
    fail(PDOT_ERR_NO_DEVICE, "libpdot.so is built for sm_100a (B200); device %d is sm_%d%d", device, major, minor);
}

// src/solver_gpu.jl:420-422 and src/saddle_point_gpu.jl:455-461
void validate(const pdot_problem* P, const pdot_pdhg_parameters* prm) {
  if (!P || !prm) fail(PDOT_ERR_INVALID_ARGUMENT, "null problem or parameters");
  if (P->num_row < 1 || P->num_col < 1) fail(PDOT_ERR_INVALID_ARGUMENT, "empty problem (%lld x %lld)",
                                             (long long)P->num_row, (long long)P->num_col);
  if (!P->cost_matrix || !P->source_distribution || !P->target_distribution)
    fail(PDOT_ERR_INVALID_ARGUMENT, "null problem array");
  if (!(prm->primal_importance > 0) || !std::isfinite(prm->primal_importance))
    fail(PDOT_ERR_INVALID_ARGUMENT, "primal_importance must be positive and finite");
  const pdot_restart_parameters& rp = prm->restart_params;
  if (!(rp.restart_frequency_if_fixed > 1)) fail(PDOT_ERR_INVALID_ARGUMENT, "restart_frequency_if_fixed > 1 failed");
  if (!(0.0 < rp.artificial_restart_threshold && rp.artificial_restart_threshold <= 1.0))
    fail(PDOT_ERR_INVALID_ARGUMENT, "0.0 < artificial_restart_threshold <= 1.0 failed");
  if (!(0.0 < rp.sufficient_reduction_for_restart &&
        rp.sufficient_reduction_for_restart <= rp.necessary_reduction_for_restart &&
        rp.necessary_reduction_for_restart <= 1.0))
    fail(PDOT_ERR_INVALID_ARGUMENT,
         "0.0 < sufficient_reduction_for_restart <= necessary_reduction_for_restart <= 1.0 failed");
  if (!(0.0 <= rp.primal_weight_update_smoothing && rp.primal_weight_update_smoothing <= 1.0))
    fail(PDOT_ERR_INVALID_ARGUMENT, "0.0 <= primal_weight_update_smoothing <= 1.0 failed");
  if (prm->termination_evaluation_frequency < 1)
    fail(PDOT_ERR_INVALID_ARGUMENT, "termination_evaluation_frequency must be positive");
  if (prm->step_size_policy != PDOT_STEP_SIZE_ADAPTIVE && prm->step_size_policy != PDOT_STEP_SIZE_CONSTANT)
    fail(PDOT_ERR_INVALID_ARGUMENT, "unknown step_size_policy %d", prm->step_size_policy);
}

pdot::SolveConfig make_config(const pdot_pdhg_parameters& p) {
  pdot::SolveConfig c;
  memset(&c, 0, sizeof(c));
  c.adaptive = p.step_size_policy == PDOT_STEP_SIZE_ADAPTIVE;
  c.reduction_exponent = p.reduction_exponent;
  c.growth_exponent = p.growth_exponent;
  c.restart_scheme = p.restart_params.restart_scheme;
  c.restart_to_current_metric = p.restart_params.restart_to_current_metric;
  c.restart_frequency_if_fixed = p.restart_params.restart_frequency_if_fixed;
  c.artificial_restart_threshold = p.restart_params.artificial_restart_threshold;
  c.sufficient_reduction_for_restart = p.restart_params.sufficient_reduction_for_restart;
  c.necessary_reduction_for_restart = p.restart_params.necessary_reduction_for_restart;
  c.primal_weight_update_smoothing = p.restart_params.primal_weight_update_smoothing;
  c.optimality_norm = p.termination_criteria.optimality_norm;
  c.eps_abs = p.termination_criteria.eps_optimal_absolute;
  c.eps_rel = p.termination_criteria.eps_optimal_relative;
  c.time_sec_limit = p.termination_criteria.time_sec_limit;
  c.iteration_limit = p.termination_criteria.iteration_limit;
  c.kkt_matrix_pass_limit = p.termination_criteria.kkt_matrix_pass_limit;
  c.record_iteration_stats = p.record_iteration_stats != 0;
  c.scale_invariant_initial_primal_weight = p.scale_invariant_initial_primal_weight != 0;
  c.primal_importance = p.primal_importance;
  return c;
}

constexpr int kRingCap = 4096;
constexpr int kInFlight = 2;

// Device memory and launch state of one solve.
class Solve {
 public:
  Solve(int device, int64_t m, int64_t n) : device_(device) {
    CK(cudaSetDevice(device));
    g_ = pdot::make_geometry(m, n, 1, device);
    const size_t N = (size_t)m * (size_t)n;
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    alloc(&C_, N);
    alloc(&X_[0], N);
    alloc(&X_[1], N);
    alloc(&a_, m);
    alloc(&b_, n);
    for (int k = 0; k < 2; ++k) {
      alloc(&u_[k], m);
      alloc(&r_[k], m);
      alloc(&v_[k], n);
      alloc(&c_[k], n);
    }
    alloc(&work_, pdot::workspace_doubles(g_));
    void* p = nullptr;
    CK(cudaMalloc(&p, sizeof(pdot::DevState)));
    allocs_.push_back(p);
    st_ = static_cast<pdot::DevState*>(p);
    CK(cudaMalloc(&p, sizeof(pdot_iteration_stats) * kRingCap));
    allocs_.push_back(p);
    ring_ = static_cast<pdot_iteration_stats*>(p);
    CK(cudaMallocHost(&p, sizeof(pdot::DevState) * kInFlight));
    host_status_ = static_cast<pdot::DevState*>(p);
    for (int k = 0; k < kInFlight; ++k) CK(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming));

    B_.C = C_;
    B_.a = a_;
    B_.b = b_;
    for (int k = 0; k < 2; ++k) {
      B_.X[k] = X_[k];
      B_.u[k] = u_[k];
      B_.v[k] = v_[k];
      B_.r[k] = r_[k];
      B_.c[k] = c_[k];
    }
    const pdot::Geometry& g = g_;
    const size_t vb = (size_t)g.row_blocks + g.col_blocks;
    double* w = work_;
    B_.rowpart = w;
    w += ((size_t)g.grid + g.panels) * pdot::kPanelRows;
    B_.colpart = w;
    w += (size_t)g.panels * g.n;
    B_.sqpart = w;
    w += g.grid;
    B_.steppart = w;
    w += vb * pdot::kStepSums;
    B_.evpart = w;
    w += (size_t)g.grid * pdot::kEvalSums;
    B_.vecpart = w;
    B_.ring = ring_;
    B_.ring_cap = kRingCap;
    B_.st = st_;
  }

  ~Solve() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (stream_) cudaStreamSynchronize(stream_);
    for (int k = 0; k < kInFlight; ++k)
      if (ev_[k]) cudaEventDestroy(ev_[k]);
    if (host_status_) cudaFreeHost(host_status_);
    for (void* p : allocs_) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
  }

  void upload(const pdot_problem& P) {
    const size_t N = (size_t)g_.m * (size_t)g_.n;
    CK(cudaMemcpyAsync(C_, P.cost_matrix, N * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(a_, P.source_distribution, g_.m * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(b_, P.target_distribution, g_.n * sizeof(double), cudaMemcpyHostToDevice, stream_));
    // CuPdhgSolverState starts at zero (src/solver_gpu.jl:428-441); the
    // average halves need no clearing: the first accepted step overwrites them.
    CK(cudaMemsetAsync(X_[0], 0, N * sizeof(double), stream_));
    CK(cudaMemsetAsync(u_[0], 0, g_.m * sizeof(double), stream_));
    CK(cudaMemsetAsync(r_[0], 0, g_.m * sizeof(double), stream_));
    CK(cudaMemsetAsync(v_[0], 0, g_.n * sizeof(double), stream_));
    CK(cudaMemsetAsync(c_[0], 0, g_.n * sizeof(double), stream_));
    CK(cudaMemsetAsync(st_, 0, sizeof(pdot::DevState), stream_));
  }

  void run(const pdot_pdhg_parameters& prm, bool use_graph, pdot_saddle_point_output* out) {
    cfg_ = make_config(prm);
    freq_ = prm.termination_evaluation_frequency;
    limit_ = prm.termination_criteria.iteration_limit;
    CK(pdot::launch_init(B_, g_, cfg_, stream_));
    if (use_graph) capture_regular_chunk();

    long long host_it = 1;
    long long drained = 0;
    int issued = 0, completed = 0;
    std::vector<pdot_iteration_stats> records;
    pdot::DevState s{};
    // keep kInFlight chunks queued; stop when the device reports `done`
    for (;;) {
      while (issued - completed < kInFlight) {
        enqueue_chunk(host_it, use_graph);
        CK(cudaMemcpyAsync(&host_status_[issued % kInFlight], st_, sizeof(pdot::DevState),
                           cudaMemcpyDeviceToHost, stream_));
        CK(cudaEventRecord(ev_[issued % kInFlight], stream_));
        ++issued;
      }
      CK(cudaEventSynchronize(ev_[completed % kInFlight]));
      s = host_status_[completed % kInFlight];
      ++completed;
      drain(s, drained, records);
      if (s.done) break;
      if (s.numerical_error) {
        // The step kernels stop once a numerical error is flagged; the next
        // evaluation terminates (src/solver_gpu.jl:529-533,594-596).
        CK(cudaStreamSynchronize(stream_));
        CK(cudaMemcpy(&s, st_, sizeof(s), cudaMemcpyDeviceToHost));
        if (!s.done) {
          CK(pdot::launch_eval(B_, g_, cfg_, stream_));
          CK(cudaStreamSynchronize(stream_));
          CK(cudaMemcpy(&s, st_, sizeof(s), cudaMemcpyDeviceToHost));
        }
        drain(s, drained, records);
        break;
      }
    }
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&s, st_, sizeof(s), cudaMemcpyDeviceToHost));
    drain(s, drained, records);
    if (!s.done) fail(PDOT_ERR_CUDA, "solver stopped without a termination reason");

    // gpu_to_cpu!, src/io.jl:41-53 (average, or current if no average exists)
    const int xb = s.out_current ? s.buf : (s.buf ^ 1);
    const size_t N = (size_t)g_.m * (size_t)g_.n;
    if (out->primal_solution)
      CK(cudaMemcpy(out->primal_solution, X_[xb], N * sizeof(double), cudaMemcpyDeviceToHost));
    if (out->dual_source_solution)
      CK(cudaMemcpy(out->dual_source_solution, u_[xb], g_.m * sizeof(double), cudaMemcpyDeviceToHost));
    if (out->dual_target_solution)
      CK(cudaMemcpy(out->dual_target_solution, v_[xb], g_.n * sizeof(double), cudaMemcpyDeviceToHost));
    out->termination_reason = s.termination_reason;
    out->iteration_count = (int32_t)(s.iteration - 1);
    out->iteration_stats_count = (int64_t)records.size();
    if (out->iteration_stats) {
      const int64_t k = std::min<int64_t>((int64_t)records.size(), out->iteration_stats_capacity);
      for (int64_t i = 0; i < k; ++i) out->iteration_stats[i] = records[i];
    }
    memset(&out->final_stats, 0, sizeof(out->final_stats));
    if (!records.empty()) {
      out->final_stats = records.back();
      out->solve_time_sec = records.back().cumulative_time_sec;
    } else {
      out->solve_time_sec = 0.0;  // invalid problem: no evaluation ran
    }
  }

 private:
  template <typename T>
  void alloc(T** p, size_t count) {
    void* q = nullptr;
    CK(cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T)));
    allocs_.push_back(q);
    *p = static_cast<T*>(q);
  }

  bool is_eval(long long it) const { return (it - 1) % freq_ == 0 || it == limit_ + 1 || it <= 10; }

  // A chunk starting here may be the captured graph: evaluation at its first
  // iteration only, and no forced evaluation (iteration_limit + 1) inside.
  bool regular_start(long long it) const {
    if (it <= 10 || (it - 1) % freq_ != 0) return false;
    for (long long k = it + 1; k < it + freq_; ++k)
      if (is_eval(k)) return false;
    return true;
  }

  void enqueue_iteration(long long it) {
    if (is_eval(it)) CK(pdot::launch_eval(B_, g_, cfg_, stream_));
    CK(pdot::launch_step(B_, g_, cfg_, stream_));
  }

  void enqueue_chunk(long long& it, bool use_graph) {
    if (use_graph && graph_exec_ && regular_start(it)) {
      CK(cudaGraphLaunch(graph_exec_, stream_));
      it += freq_;
      return;
    }
    // direct launches up to the next regular chunk (at most freq iterations)
    long long k = 0;
    do {
      enqueue_iteration(it);
      ++it;
      ++k;
    } while (k < freq_ && !(use_graph && graph_exec_ && regular_start(it)));
  }

  void capture_regular_chunk() {
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = pdot::launch_eval(B_, g_, cfg_, stream_);
    for (long long k = 0; k < freq_ && e == cudaSuccess; ++k) e = pdot::launch_step(B_, g_, cfg_, stream_);
    cudaError_t e2 = cudaStreamEndCapture(stream_, &graph);
    CK(e);
    CK(e2);
    cudaError_t e3 = cudaGraphInstantiate(&graph_exec_, graph, 0);
    cudaGraphDestroy(graph);
    CK(e3);
  }

  void drain(const pdot::DevState& s, long long& drained, std::vector<pdot_iteration_stats>& recs) {
    const long long total = s.num_stats;
    if (total <= drained) return;
    if (total - drained > kRingCap) fail(PDOT_ERR_CUDA, "iteration-stats ring overflow");
    std::vector<pdot_iteration_stats> tmp((size_t)(total - drained));
    for (long long k = drained; k < total; ++k) {
      CK(cudaMemcpy(&tmp[(size_t)(k - drained)], ring_ + (k % kRingCap), sizeof(pdot_iteration_stats),
                    cudaMemcpyDeviceToHost));
    }
    recs.insert(recs.end(), tmp.begin(), tmp.end());
    drained = total;
  }

  int device_;
  pdot::Geometry g_{};
  pdot::SolveConfig cfg_{};
  long long freq_ = 128, limit_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[kInFlight] = {};
  cudaGraphExec_t graph_exec_ = nullptr;
  std::vector<void*> allocs_;
  double* C_ = nullptr;
  double* X_[2] = {};
  double *a_ = nullptr, *b_ = nullptr;
  double* u_[2] = {};
  double* v_[2] = {};
  double* r_[2] = {};
  double* c_[2] = {};
  double* work_ = nullptr;
  pdot::DevState* st_ = nullptr;
  pdot_iteration_stats* ring_ = nullptr;
  pdot::DevState* host_status_ = nullptr;
  pdot::Buffers B_{};
};

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int64_t pass_workspace_bytes(const pdot::Geometry& g) {
  return (int64_t)((((size_t)g.grid + g.panels) * pdot::kPanelRows + (size_t)g.panels * g.n + g.grid) *
                   sizeof(double));
}

}  // namespace

extern "C" {

int pdot_version(void) { return PDOT_ABI_VERSION; }

const char* pdot_last_error(void) { return g_last_error.c_str(); }

void pdot_default_parameters(double tolerance, pdot_pdhg_parameters* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->primal_importance = 1.0;
  p->scale_invariant_initial_primal_weight = 0;
  p->verbosity = 2;
  p->record_iteration_stats = 1;
  p->termination_evaluation_frequency = 128;
  p->termination_criteria.optimality_norm = PDOT_L_2;
  p->termination_criteria.eps_optimal_absolute = tolerance;
  p->termination_criteria.eps_optimal_relative = tolerance;
  p->termination_criteria.time_sec_limit = INFINITY;
  p->termination_criteria.iteration_limit = 2147483647;
  p->termination_criteria.kkt_matrix_pass_limit = INFINITY;
  p->restart_params.restart_scheme = PDOT_ADAPTIVE_KKT;
  p->restart_params.restart_to_current_metric = PDOT_KKT_GREEDY;
  p->restart_params.restart_frequency_if_fixed = 1000;
  p->restart_params.artificial_restart_threshold = 0.36;
  p->restart_params.sufficient_reduction_for_restart = 0.1;
  p->restart_params.necessary_reduction_for_restart = 0.9;
  p->restart_params.primal_weight_update_smoothing = 0.5;
  p->step_size_policy = PDOT_STEP_SIZE_ADAPTIVE;
  p->reduction_exponent = 2.0;
  p->growth_exponent = 1.0;
}

int pdot_optimize(const pdot_problem* problem, const pdot_pdhg_parameters* params,
                  const pdot_solver_options* options, pdot_saddle_point_output* output) {
  return guarded([&] {
    validate(problem, params);
    if (!output) fail(PDOT_ERR_INVALID_ARGUMENT, "null output");
    const int device = options ? options->device : 0;
    const bool use_graph = options ? options->use_cuda_graph != 0 : true;
    require_sm100(device);
    Solve solve(device, problem->num_row, problem->num_col);
    solve.upload(*problem);
    solve.run(*params, use_graph, output);
  });
}

int64_t pdot_primal_pass_workspace_bytes(int64_t m, int64_t n) {
  if (m < 1 || n < 1) return 0;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  // the grid depends on the load width the buffers allow: cover both
  const int64_t a = pass_workspace_bytes(pdot::make_geometry(m, n, 1, device));
  const int64_t b = pass_workspace_bytes(pdot::make_geometry(m, n, 0, device));
  return a > b ? a : b;
}

int pdot_primal_pass_f64(int64_t m, int64_t n, const double* cost, double* primal, double* primal_avg,
                         const double* dual_source, const double* dual_target, double step_over_weight,
                         double avg_new_weight, double avg_scale, int32_t flags, double* delta_row_sum,
                         double* delta_col_sum, double* delta_sq_norm, void* workspace, int64_t workspace_bytes,
                         void* stream) {
  return guarded([&] {
    if (m < 1 || n < 1) fail(PDOT_ERR_INVALID_ARGUMENT, "empty matrix");
    if (!cost || !primal || !primal_avg || !dual_source || !dual_target || !delta_row_sum || !delta_col_sum ||
        !delta_sq_norm || !workspace)
      fail(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
    if (primal == primal_avg) fail(PDOT_ERR_INVALID_ARGUMENT, "primal and primal_avg must not alias");
    int device = 0;
    CK(cudaGetDevice(&device));
    const int vec_ok = aligned16(cost) && aligned16(primal) && aligned16(primal_avg);
    const pdot::Geometry g = pdot::make_geometry(m, n, vec_ok, device);
    const int64_t need = pass_workspace_bytes(g);
    if (workspace_bytes < need)
      fail(PDOT_ERR_INVALID_ARGUMENT, "workspace of %lld bytes, %lld needed", (long long)workspace_bytes,
           (long long)need);
    CK(pdot::launch_primal_pass(g, cost, primal, primal_avg, dual_source, dual_target, step_over_weight,
                                avg_new_weight, avg_scale, flags, delta_row_sum, delta_col_sum, delta_sq_norm,
                                static_cast<double*>(workspace), static_cast<cudaStream_t>(stream)));
  });
}

}  // extern "C"
