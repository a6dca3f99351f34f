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
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
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

}  // namespace

namespace pdot {
void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
}  // namespace pdot

namespace {

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
  if (!P->source_distribution || !P->target_distribution) fail(PDOT_ERR_INVALID_ARGUMENT, "null problem array");
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

// Options of this implementation (include/pdot.h: pdot_solver_options).
struct Variant {
  int device = 0;
  bool use_graph = true, time_kernels = false;
  int plan_f32 = 0;
  int cost_kind = PDOT_COST_F64;
  int point_dim = 0;
  const float* xs = nullptr;
  const float* ys = nullptr;
  double cost_scale = 0.0;
  const double* warm_u = nullptr;
  const double* warm_v = nullptr;
  const double* warm_x = nullptr;
  double plan_eps = 0.0;  // > 0: recover the warm plan from the warm duals
  int plan_iters = 0;
  int staged = 2;  // 0 direct, 1 staged, 2 automatic
  int fail_waits = 0;  // test hook: the staged pass's waits report timeouts
  double warm_omega = 0.0;  // > 0: initial primal weight of a warm start
  bool warm_zero = false;   // a warm start's restart information starts at the zero point
  int persistent = 0;       // persistent chunk kernel: 0 automatic, 1 on, -1 off
};

Variant read_options(const pdot_problem& P, const pdot_solver_options* o) {
  Variant v;
  if (!o) {
    if (!P.cost_matrix) fail(PDOT_ERR_INVALID_ARGUMENT, "null cost matrix");
    return v;
  }
  v.device = o->device;
  v.use_graph = o->use_cuda_graph != 0;
  v.time_kernels = o->time_kernels != 0;
  if (o->plan_precision != PDOT_PRECISION_F64 && o->plan_precision != PDOT_PRECISION_F32)
    fail(PDOT_ERR_INVALID_ARGUMENT, "unknown plan_precision %d", o->plan_precision);
  v.plan_f32 = o->plan_precision == PDOT_PRECISION_F32;
  v.cost_kind = o->cost_storage;
  if (v.cost_kind < PDOT_COST_F64 || v.cost_kind > PDOT_COST_L1_POINTS)
    fail(PDOT_ERR_INVALID_ARGUMENT, "unknown cost_storage %d", v.cost_kind);
  if (v.plan_f32 == (v.cost_kind == PDOT_COST_F64))
    fail(PDOT_ERR_INVALID_ARGUMENT,
         "the FP64 plan runs with the FP64 cost; an FP32 plan runs with FP32, BF16 or coordinate costs");
  if (v.cost_kind == PDOT_COST_SQEUCLID_POINTS || v.cost_kind == PDOT_COST_L1_POINTS) {
    if (o->point_dim < 1 || o->point_dim > pdot::kMaxPointDim)
      fail(PDOT_ERR_INVALID_ARGUMENT, "point_dim must be 1..%d", pdot::kMaxPointDim);
    if (!o->source_points || !o->target_points) fail(PDOT_ERR_INVALID_ARGUMENT, "null point coordinates");
    v.point_dim = o->point_dim;
    v.xs = o->source_points;
    v.ys = o->target_points;
    v.cost_scale = o->cost_scale > 0.0 ? o->cost_scale : 0.0;
  } else if (!P.cost_matrix) {
    fail(PDOT_ERR_INVALID_ARGUMENT, "null cost matrix");
  }
  if ((o->warm_dual_source == nullptr) != (o->warm_dual_target == nullptr))
    fail(PDOT_ERR_INVALID_ARGUMENT, "give both warm-start dual vectors or neither");
  v.warm_u = o->warm_dual_source;
  v.warm_v = o->warm_dual_target;
  if (o->warm_primal && !o->warm_dual_source)
    fail(PDOT_ERR_INVALID_ARGUMENT, "a warm-start plan needs the warm-start dual vectors");
  v.warm_x = o->warm_primal;
  if (!(o->warm_plan_epsilon >= 0.0) || !std::isfinite(o->warm_plan_epsilon))
    fail(PDOT_ERR_INVALID_ARGUMENT, "warm_plan_epsilon must be finite and >= 0");
  if (o->warm_plan_iterations < 0 || o->warm_plan_iterations > 100000)
    fail(PDOT_ERR_INVALID_ARGUMENT, "warm_plan_iterations must be 0..100000");
  if (o->warm_plan_epsilon > 0.0) {
    if (!o->warm_dual_source) fail(PDOT_ERR_INVALID_ARGUMENT, "a recovered warm plan needs the warm-start duals");
    if (o->warm_primal) fail(PDOT_ERR_INVALID_ARGUMENT, "give a warm plan or warm_plan_epsilon, not both");
    v.plan_eps = o->warm_plan_epsilon;
    v.plan_iters = o->warm_plan_iterations;
  }
  if (o->primal_pass != PDOT_PASS_AUTO && o->primal_pass != PDOT_PASS_STAGED && o->primal_pass != PDOT_PASS_DIRECT)
    fail(PDOT_ERR_INVALID_ARGUMENT, "unknown primal_pass %d", o->primal_pass);
  v.staged = o->primal_pass == PDOT_PASS_STAGED ? 1 : (o->primal_pass == PDOT_PASS_DIRECT ? 0 : 2);
  if (o->fail_bounded_waits != 0 && o->fail_bounded_waits != 1)
    fail(PDOT_ERR_INVALID_ARGUMENT, "fail_bounded_waits must be 0 or 1");
  v.fail_waits = o->fail_bounded_waits;
  if (!std::isfinite(o->warm_primal_weight)) fail(PDOT_ERR_INVALID_ARGUMENT, "warm_primal_weight must be finite");
  if (o->warm_primal_weight > 0.0 && !o->warm_dual_source)
    fail(PDOT_ERR_INVALID_ARGUMENT, "warm_primal_weight needs the warm-start duals");
  v.warm_omega = o->warm_primal_weight > 0.0 ? o->warm_primal_weight : 0.0;
  if (o->warm_restart_at_zero != 0 && o->warm_restart_at_zero != 1)
    fail(PDOT_ERR_INVALID_ARGUMENT, "warm_restart_at_zero must be 0 or 1");
  v.warm_zero = o->warm_restart_at_zero == 1;
  if (o->persistent_chunks < -1 || o->persistent_chunks > 1)
    fail(PDOT_ERR_INVALID_ARGUMENT, "persistent_chunks must be -1, 0 or 1");
  v.persistent = o->persistent_chunks;
  return v;
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

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// A temporary device buffer freed when it goes out of scope, also when a CK
// check throws on the way (cudaFree waits for the work that still uses it).
struct DeviceTemp {
  void* p = nullptr;
  DeviceTemp() = default;
  DeviceTemp(const DeviceTemp&) = delete;
  DeviceTemp& operator=(const DeviceTemp&) = delete;
  ~DeviceTemp() {
    if (p) cudaFree(p);
  }
  template <typename T>
  T* get() const {
    return static_cast<T*>(p);
  }
};

int64_t pass_workspace_bytes(const pdot::Geometry& g) {
  return (int64_t)(pdot::pass_scratch_doubles(g) * sizeof(double));
}

constexpr int kRingCap = 4096;
constexpr int kInFlight = 2;


enum TimedKind { kTimedPrimal = 0, kTimedDual = 1, kTimedEval = 2 };

struct TimedLaunch {
  cudaEvent_t start, stop;
  int kind;
};

// Device memory and launch state of one problem and its optimize() loop.
class Solver {
 public:
  Solver(const pdot_problem& P, bool device_inputs, const pdot_pdhg_parameters& prm,
         const pdot_solver_options* opt)
      : params_(prm) {
    const Variant var = read_options(P, opt);
    device_ = var.device;
    use_graph_ = var.use_graph;
    time_kernels_ = var.time_kernels;
    CK(cudaSetDevice(device_));
    const int64_t m = P.num_row, n = P.num_col;
    const size_t N = (size_t)m * (size_t)n;
    const size_t xbytes = var.plan_f32 ? sizeof(float) : sizeof(double);
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));

    // the cost: as given (FP64), converted to FP32 / BF16 on the device, or
    // coordinates for the on-the-fly squared-Euclidean cost
    bool cost_aligned = true;
    if (var.cost_kind == PDOT_COST_SQEUCLID_POINTS || var.cost_kind == PDOT_COST_L1_POINTS) {
      const size_t d = (size_t)var.point_dim;
      if (device_inputs) {
        cost_.xs = var.xs;
        cost_.ys = var.ys;
      } else {
        float *xs = nullptr, *ys = nullptr;
        alloc(&xs, (size_t)m * d);
        alloc(&ys, (size_t)n * d);
        CK(cudaMemcpyAsync(xs, var.xs, (size_t)m * d * sizeof(float), cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(ys, var.ys, (size_t)n * d * sizeof(float), cudaMemcpyHostToDevice, stream_));
        cost_.xs = xs;
        cost_.ys = ys;
      }
      cost_.dim = var.point_dim;
      cost_.C = nullptr;
    } else if (var.cost_kind == PDOT_COST_F64) {
      if (device_inputs) {
        cost_.C = P.cost_matrix;
        cost_aligned = aligned16(P.cost_matrix);
      } else {
        double* C = nullptr;
        alloc(&C, N);
        CK(pdot::copy_to_device(C, P.cost_matrix, N * sizeof(double), stream_));
        cost_.C = C;
      }
    } else {
      const size_t cbytes = var.cost_kind == PDOT_COST_F32 ? 4 : 2;
      void* Cs = nullptr;
      CK(cudaMalloc(&Cs, std::max<size_t>(N, 1) * cbytes));
      allocs_.push_back(Cs);
      const double* src = P.cost_matrix;
      DeviceTemp tmp;
      if (!device_inputs) {
        CK(cudaMalloc(&tmp.p, N * sizeof(double)));
        CK(pdot::copy_to_device(tmp.p, P.cost_matrix, N * sizeof(double), stream_));
        src = tmp.get<const double>();
      }
      CK(pdot::launch_convert_cost(src, Cs, var.cost_kind, N, stream_));
      CK(cudaStreamSynchronize(stream_));
      cost_.C = Cs;
    }
    const int kind = pdot::internal_cost_kind(var.cost_kind, var.point_dim);
    g_ = pdot::make_geometry(m, n, cost_aligned ? 1 : 0, device_, var.plan_f32, kind, var.staged);
    g_.fail_waits = var.fail_waits;
    if (device_inputs) {
      a_ = P.source_distribution;
      b_ = P.target_distribution;
    } else {
      double *a = nullptr, *b = nullptr;
      alloc(&a, m);
      alloc(&b, n);
      CK(cudaMemcpyAsync(a, P.source_distribution, m * sizeof(double), cudaMemcpyHostToDevice, stream_));
      CK(cudaMemcpyAsync(b, P.target_distribution, n * sizeof(double), cudaMemcpyHostToDevice, stream_));
      a_ = a;
      b_ = b;
    }
    if (var.warm_u) {
      alloc(&warm_u_, m);
      alloc(&warm_v_, n);
      const cudaMemcpyKind kind = device_inputs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
      CK(cudaMemcpyAsync(warm_u_, var.warm_u, m * sizeof(double), kind, stream_));
      CK(cudaMemcpyAsync(warm_v_, var.warm_v, n * sizeof(double), kind, stream_));
    }
    if (var.plan_eps > 0.0) {
      // recovery of the warm plan from the warm duals (run by reset())
      plan_eps_ = var.plan_eps;
      plan_iters_ = var.plan_iters;
      pdot::PlanInstance pi{};
      pi.m = m;
      pi.n = n;
      pi.ld = m;
      pi.active = 1;
      const long long pre[4] = {0, (long long)m, 0, (long long)n};
      void* p = nullptr;
      CK(cudaMalloc(&p, sizeof(pi) + sizeof(pre)));
      allocs_.push_back(p);
      CK(cudaMemcpy(p, &pi, sizeof(pi), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(static_cast<char*>(p) + sizeof(pi), pre, sizeof(pre), cudaMemcpyHostToDevice));
      double *f = nullptr, *gg = nullptr;
      alloc(&f, m);
      alloc(&gg, n);
      wp_.inst = static_cast<const pdot::PlanInstance*>(p);
      wp_.num = 1;
      wp_.row_prefix = reinterpret_cast<const long long*>(static_cast<char*>(p) + sizeof(pi));
      wp_.col_prefix = wp_.row_prefix + 2;
      wp_.total_rows = m;
      wp_.total_cols = n;
      wp_.f = f;
      wp_.g = gg;
      wp_.eps = plan_eps_;
      wp_.plan_f32 = var.plan_f32;
    }
    if (var.warm_x) {
      // the warm plan in plan precision, and its row and column sums
      void* wx = nullptr;
      CK(cudaMalloc(&wx, std::max<size_t>(N, 1) * xbytes));
      allocs_.push_back(wx);
      warm_x_ = wx;
      alloc(&warm_r_, m);
      alloc(&warm_c_, n);
      const double* src = var.warm_x;
      DeviceTemp tmp, work;
      if (!device_inputs) {
        CK(cudaMalloc(&tmp.p, std::max<size_t>(N, 1) * sizeof(double)));
        CK(pdot::copy_to_device(tmp.p, var.warm_x, N * sizeof(double), stream_));
        src = tmp.get<const double>();
      }
      if (var.plan_f32)
        CK(pdot::launch_convert_cost(src, wx, PDOT_COST_F32, N, stream_));
      else
        CK(cudaMemcpyAsync(wx, src, N * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      CK(cudaMalloc(&work.p, std::max<size_t>(pdot::plan_sums_workspace_doubles(m, n), 1) * sizeof(double)));
      CK(pdot::launch_plan_sums(m, n, wx, var.plan_f32, warm_r_, warm_c_, work.get<double>(), stream_));
      CK(cudaStreamSynchronize(stream_));
    }
    void* xp = nullptr;
    for (int k = 0; k < 2; ++k) {
      CK(cudaMalloc(&xp, std::max<size_t>(N, 1) * xbytes));
      allocs_.push_back(xp);
      X_[k] = xp;
    }
    xbytes_ = xbytes;
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

    B_.cost = cost_;
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
    const size_t db = (size_t)g.dual_row_blocks + g.col_blocks;
    double* w = work_;
    B_.rowpart = w;
    w += ((size_t)g.grid + g.panels) * pdot::kPanelRows;
    B_.colpart = w;
    w += (size_t)g.panels * g.n;
    B_.sqpart = w;
    w += g.grid;
    B_.steppart = w;
    w += db * pdot::kStepSums;
    B_.evpart = w;
    w += (size_t)g.grid * pdot::kEvalSums;
    B_.vecpart = w;
    B_.ring = ring_;
    B_.ring_cap = kRingCap;
    B_.st = st_;
    if (plan_eps_ > 0.0) {
      wp_.kind = pdot::internal_cost_kind(var.cost_kind, var.point_dim);
      wp_.dim = cost_.dim;
      wp_.C = cost_.C;
      wp_.xs = cost_.xs;
      wp_.ys = cost_.ys;
      wp_.st = st_;
      wp_.a = a_;
      wp_.b = b_;
      wp_.u0 = warm_u_;
      wp_.v0 = warm_v_;
    }

    cfg_ = make_config(prm);
    cfg_.cost_scale = var.cost_scale;
    cfg_.warm_start = warm_u_ != nullptr;
    cfg_.warm_primal_weight = var.warm_omega;
    warm_zero_ = var.warm_zero;
    freq_ = prm.termination_evaluation_frequency;
    limit_ = prm.termination_criteria.iteration_limit;
    // automatic = the CUDA graph: on B200 the persistent chunk measured slower
    // at every size tried (31 against 16 us per iteration at 1000 x 1000, 1071
    // against 718 at 10000 x 10000)
    persistent_ = g_.chunk_ctas > 0 && !time_kernels_ && var.persistent == 1;
    if (use_graph_ && !time_kernels_ && !persistent_) capture_regular_chunk();
    reset();
  }

  ~Solver() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    for (int k = 0; k < kInFlight; ++k) {
      if (ev_[k]) cudaEventDestroy(ev_[k]);
      for (TimedLaunch& t : timed_[k]) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
      }
    }
    for (TimedLaunch& t : spare_) {
      cudaEventDestroy(t.start);
      cudaEventDestroy(t.stop);
    }
    if (host_status_) cudaFreeHost(host_status_);
    for (void* p : allocs_) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
  }

  cudaStream_t stream() const { return stream_; }

  // CuPdhgSolverState starts at zero (src/solver_gpu.jl:428-441), or at the
  // warm start (duals, and the plan with its row and column sums); the average
  // halves need no clearing: the first accepted step overwrites them.
  void reset() {
    CK(cudaSetDevice(device_));
    CK(cudaStreamSynchronize(stream_));
    const size_t N = (size_t)g_.m * (size_t)g_.n;
    if (warm_x_)
      CK(cudaMemcpyAsync(X_[0], warm_x_, N * xbytes_, cudaMemcpyDeviceToDevice, stream_));
    else
      CK(cudaMemsetAsync(X_[0], 0, N * xbytes_, stream_));
    if (warm_u_) {
      CK(cudaMemcpyAsync(u_[0], warm_u_, g_.m * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      CK(cudaMemcpyAsync(v_[0], warm_v_, g_.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    } else {
      CK(cudaMemsetAsync(u_[0], 0, g_.m * sizeof(double), stream_));
      CK(cudaMemsetAsync(v_[0], 0, g_.n * sizeof(double), stream_));
    }
    if (warm_x_) {
      CK(cudaMemcpyAsync(r_[0], warm_r_, g_.m * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      CK(cudaMemcpyAsync(c_[0], warm_c_, g_.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    } else {
      CK(cudaMemsetAsync(r_[0], 0, g_.m * sizeof(double), stream_));
      CK(cudaMemsetAsync(c_[0], 0, g_.n * sizeof(double), stream_));
    }
    CK(cudaMemsetAsync(st_, 0, sizeof(pdot::DevState), stream_));
    CK(pdot::launch_init(B_, g_, cfg_, stream_));
    if (plan_eps_ > 0.0) {
      wp_.X = X_[0];
      wp_.r = r_[0];
      wp_.c = c_[0];
      CK(pdot::launch_warm_plan(wp_, plan_iters_, stream_));
    }
    // a warm start's restart information starts at the warm point, as the
    // reference's starts at its initial point (unless asked to start at zero,
    // k0_init's record)
    if (cfg_.warm_start && !warm_zero_) CK(pdot::launch_eval(B_, g_, cfg_, stream_, 1));
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&status_, st_, sizeof(status_), cudaMemcpyDeviceToHost));
    host_it_ = 1;
    drained_ = 0;
    records_.clear();
    primal_ms_ = dual_ms_ = eval_ms_ = 0.0;
    timed_primal_ = 0;
  }

  void iterate(int64_t max_iterations) {
    CK(cudaSetDevice(device_));
    int64_t remaining = max_iterations;
    int issued = 0, completed = 0;
    while (!status_.done && (remaining > 0 || issued > completed)) {
      while (issued - completed < kInFlight && remaining > 0 && !status_.done) {
        const int slot = issued % kInFlight;
        remaining -= enqueue_chunk(remaining, slot);
        CK(cudaMemcpyAsync(&host_status_[slot], st_, sizeof(pdot::DevState), cudaMemcpyDeviceToHost, stream_));
        CK(cudaEventRecord(ev_[slot], stream_));
        ++issued;
      }
      const int slot = completed % kInFlight;
      CK(cudaEventSynchronize(ev_[slot]));
      status_ = host_status_[slot];
      collect_timings(slot);
      ++completed;
      drain();
      if (status_.kernel_error) {
        sync_all(issued, completed);
        fail(PDOT_ERR_CUDA,
             "a bounded wait timed out (staged primal pass or persistent chunk barrier; kernel_error %d)",
             status_.kernel_error);
      }
      if (status_.done) break;
      if (status_.numerical_error) {
        // The step kernels stop once a numerical error is flagged; the next
        // evaluation terminates (src/solver_gpu.jl:529-533,594-596).
        sync_all(issued, completed);
        if (!status_.done) {
          CK(pdot::launch_eval(B_, g_, cfg_, stream_));
          CK(cudaStreamSynchronize(stream_));
          CK(cudaMemcpy(&status_, st_, sizeof(status_), cudaMemcpyDeviceToHost));
          drain();
        }
        break;
      }
    }
    sync_all(issued, completed);
  }

  // The caller's plan buffer is overwritten in full; fresh host memory (a
  // numpy zeros array, a plain malloc) pays a page fault per 4 KB page on its
  // first write. Host threads therefore write it while the GPU iterates, in
  // 2 MiB pieces, until the solve ends; the copy back (pdot_transfer.cu) then
  // finds those pages present and faults the rest itself, in parallel.
  // Page-locked buffers are resident already and are left alone.
  struct Prefault {
    std::vector<std::thread> threads;
    std::atomic<bool> stop{false};
    Prefault(double* p, size_t count) {
      if (!p || count < (size_t(1) << 22) || pdot::host_is_pinned(p)) return;  // small plans: not worth a thread
      const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
      const size_t parts = std::min<size_t>(8, std::max<size_t>(1, hw / 2));
      const size_t per = (count + parts - 1) / parts;
      for (size_t k = 0; k < parts; ++k) {
        const size_t lo = k * per, hi = std::min(count, lo + per);
        if (lo >= hi) continue;
        threads.emplace_back([this, p, lo, hi] {
          const size_t piece = size_t(1) << 18;  // doubles (2 MiB)
          for (size_t a = lo; a < hi && !stop.load(std::memory_order_relaxed); a += piece)
            memset(p + a, 0, (std::min(hi, a + piece) - a) * sizeof(double));
        });
      }
    }
    void finish() {
      stop.store(true);
      for (std::thread& t : threads) t.join();
      threads.clear();
    }
    ~Prefault() { finish(); }
  };

  void finish(pdot_saddle_point_output* out) {
    {
      Prefault touch(out->primal_solution, (size_t)g_.m * (size_t)g_.n);
      while (!status_.done) iterate(int64_t(1) << 40);
      touch.finish();
    }
    // gpu_to_cpu!, src/io.jl:41-53 (average, or current if no average exists)
    const int xb = status_.out_current ? status_.buf : (status_.buf ^ 1);
    const size_t N = (size_t)g_.m * (size_t)g_.n;
    if (out->primal_solution) {
      if (!g_.plan_f32) {
        const double* X = static_cast<const double*>(X_[xb]);
        CK(pdot::copy_to_host(out->primal_solution, N,
                              [X](size_t off, size_t, int, cudaStream_t) { return X + off; }, stream_));
      } else {
        // widen the FP32 plan chunk by chunk into two device buffers
        const size_t chunk = std::min<size_t>(N, pdot::kTransferChunk);
        DeviceTemp tmp;
        CK(cudaMalloc(&tmp.p, 2 * std::max<size_t>(chunk, 1) * sizeof(double)));
        const float* Xf = static_cast<const float*>(X_[xb]);
        double* buf = tmp.get<double>();
        CK(pdot::copy_to_host(out->primal_solution, N,
                              [Xf, buf, chunk](size_t off, size_t cnt, int slot, cudaStream_t s) -> const double* {
                                double* d = buf + (size_t)slot * chunk;
                                pdot::launch_widen(Xf + off, d, cnt, s);
                                return d;
                              },
                              stream_));
      }
    }
    if (out->dual_source_solution)
      CK(cudaMemcpy(out->dual_source_solution, u_[xb], g_.m * sizeof(double), cudaMemcpyDeviceToHost));
    if (out->dual_target_solution)
      CK(cudaMemcpy(out->dual_target_solution, v_[xb], g_.n * sizeof(double), cudaMemcpyDeviceToHost));
    out->termination_reason = status_.termination_reason;
    out->iteration_count = (int32_t)(status_.iteration - 1);
    out->iteration_stats_count = (int64_t)records_.size();
    if (out->iteration_stats) {
      const int64_t k = std::min<int64_t>((int64_t)records_.size(), out->iteration_stats_capacity);
      for (int64_t i = 0; i < k; ++i) out->iteration_stats[i] = records_[i];
    }
    memset(&out->final_stats, 0, sizeof(out->final_stats));
    if (!records_.empty()) {
      out->final_stats = records_.back();
      out->solve_time_sec = records_.back().cumulative_time_sec;
    } else {
      out->solve_time_sec = 0.0;  // invalid problem: no evaluation ran
    }
  }

  void fill_status(pdot_solver_status* s) const {
    memset(s, 0, sizeof(*s));
    s->iteration = status_.iteration;
    s->total_number_iterations = status_.total_iters;
    s->done = status_.done;
    s->termination_reason = status_.termination_reason;
    s->step_size = status_.step_size;
    s->primal_weight = status_.primal_weight;
    s->cumulative_kkt_matrix_passes = status_.kkt_passes;
    s->iteration_stats_count = (int64_t)records_.size();
    s->primal_passes = status_.primal_passes;
    s->primal_passes_fresh_average = status_.fresh_passes;
    s->timed_primal_passes = timed_primal_;
    s->primal_pass_ms = primal_ms_;
    s->dual_step_ms = dual_ms_;
    s->evaluation_ms = eval_ms_;
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

  // A chunk starting here may be the captured graph or the persistent chunk
  // kernel: evaluation at its first iteration only, and no forced evaluation
  // (iteration_limit + 1) inside.
  bool regular_start(long long it) const {
    if (!(graph_exec_ || persistent_) || it <= 10 || (it - 1) % freq_ != 0) return false;
    for (long long k = it + 1; k < it + freq_; ++k)
      if (is_eval(k)) return false;
    return true;
  }

  TimedLaunch take_timer(int kind) {
    TimedLaunch t;
    if (!spare_.empty()) {
      t = spare_.back();
      spare_.pop_back();
    } else {
      CK(cudaEventCreate(&t.start));
      CK(cudaEventCreate(&t.stop));
    }
    t.kind = kind;
    return t;
  }

  template <typename L>
  void timed(int slot, int kind, L&& launch) {
    if (!time_kernels_) {
      CK(launch());
      return;
    }
    TimedLaunch t = take_timer(kind);
    CK(cudaEventRecord(t.start, stream_));
    CK(launch());
    CK(cudaEventRecord(t.stop, stream_));
    timed_[slot].push_back(t);
  }

  void enqueue_iteration(long long it, int slot) {
    if (is_eval(it)) timed(slot, kTimedEval, [&] { return pdot::launch_eval(B_, g_, cfg_, stream_); });
    const int xsums = is_eval(it + 1) ? 1 : 0;
    timed(slot, kTimedPrimal, [&] { return pdot::launch_primal(B_, g_, stream_, xsums); });
    timed(slot, kTimedDual, [&] { return pdot::launch_dual(B_, g_, cfg_, stream_); });
  }

  // Enqueues up to `budget` loop bodies starting at host_it_; returns how many.
  int64_t enqueue_chunk(int64_t budget, int slot) {
    if (regular_start(host_it_) && budget >= freq_) {
      if (persistent_)
        CK(pdot::launch_chunk(B_, g_, cfg_, stream_, (int)freq_));
      else
        CK(cudaGraphLaunch(graph_exec_, stream_));
      host_it_ += freq_;
      return freq_;
    }
    int64_t k = 0;
    do {
      enqueue_iteration(host_it_, slot);
      ++host_it_;
      ++k;
    } while (k < freq_ && k < budget && !regular_start(host_it_));
    return k;
  }

  void collect_timings(int slot) {
    for (TimedLaunch& t : timed_[slot]) {
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, t.start, t.stop));
      if (t.kind == kTimedPrimal) {
        primal_ms_ += ms;
        ++timed_primal_;
      } else if (t.kind == kTimedDual) {
        dual_ms_ += ms;
      } else {
        eval_ms_ += ms;
      }
      spare_.push_back(t);
    }
    timed_[slot].clear();
  }

  void sync_all(int issued, int& completed) {
    while (completed < issued) {
      const int slot = completed % kInFlight;
      CK(cudaEventSynchronize(ev_[slot]));
      collect_timings(slot);
      ++completed;
    }
    CK(cudaStreamSynchronize(stream_));
    CK(cudaMemcpy(&status_, st_, sizeof(status_), cudaMemcpyDeviceToHost));
    drain();
  }

  void capture_regular_chunk() {
    cudaGraph_t graph = nullptr;
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = pdot::launch_eval(B_, g_, cfg_, stream_);
    // the chunk's last step precedes the next chunk's evaluation
    for (long long k = 0; k < freq_ && e == cudaSuccess; ++k)
      e = pdot::launch_step(B_, g_, cfg_, stream_, k == freq_ - 1 ? 1 : 0);
    cudaError_t e2 = cudaStreamEndCapture(stream_, &graph);
    CK(e);
    CK(e2);
    cudaError_t e3 = cudaGraphInstantiate(&graph_exec_, graph, 0);
    cudaGraphDestroy(graph);
    CK(e3);
  }

  void drain() {
    const long long total = status_.num_stats;
    if (total <= drained_) return;
    if (total - drained_ > kRingCap) fail(PDOT_ERR_CUDA, "iteration-stats ring overflow");
    for (long long k = drained_; k < total; ++k) {
      pdot_iteration_stats rec;
      CK(cudaMemcpy(&rec, ring_ + (k % kRingCap), sizeof(rec), cudaMemcpyDeviceToHost));
      records_.push_back(rec);
    }
    drained_ = total;
  }

  int device_ = 0;
  bool use_graph_ = true, time_kernels_ = false;
  bool persistent_ = false;  // regular chunks run as one persistent launch
  pdot_pdhg_parameters params_;
  pdot::Geometry g_{};
  pdot::SolveConfig cfg_{};
  long long freq_ = 128, limit_ = 0;
  long long host_it_ = 1, drained_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev_[kInFlight] = {};
  cudaGraphExec_t graph_exec_ = nullptr;
  std::vector<TimedLaunch> timed_[kInFlight];
  std::vector<TimedLaunch> spare_;
  double primal_ms_ = 0.0, dual_ms_ = 0.0, eval_ms_ = 0.0;
  long long timed_primal_ = 0;
  std::vector<void*> allocs_;
  pdot::CostSource cost_{};
  const double* a_ = nullptr;
  const double* b_ = nullptr;
  double* warm_u_ = nullptr;
  double* warm_v_ = nullptr;
  void* warm_x_ = nullptr;
  double* warm_r_ = nullptr;
  double* warm_c_ = nullptr;
  double plan_eps_ = 0.0;
  int plan_iters_ = 0;
  bool warm_zero_ = false;
  pdot::WarmPlanArgs wp_{};
  void* X_[2] = {};
  size_t xbytes_ = sizeof(double);
  double* u_[2] = {};
  double* v_[2] = {};
  double* r_[2] = {};
  double* c_[2] = {};
  double* work_ = nullptr;
  pdot::DevState* st_ = nullptr;
  pdot_iteration_stats* ring_ = nullptr;
  pdot::DevState* host_status_ = nullptr;
  pdot::DevState status_{};
  std::vector<pdot_iteration_stats> records_;
  pdot::Buffers B_{};
};


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
    read_options(*problem, options);
    require_sm100(options ? options->device : 0);
    Solver solver(*problem, false, *params, options);
    solver.finish(output);
  });
}

struct pdot_solver {
  Solver* impl;
};

static int create_solver(const pdot_problem* problem, const pdot_pdhg_parameters* params,
                         const pdot_solver_options* options, pdot_solver** out, bool device_inputs) {
  return guarded([&] {
    validate(problem, params);
    if (!out) fail(PDOT_ERR_INVALID_ARGUMENT, "null solver handle");
    *out = nullptr;
    read_options(*problem, options);
    require_sm100(options ? options->device : 0);
    Solver* s = new Solver(*problem, device_inputs, *params, options);
    *out = new pdot_solver{s};
  });
}

int pdot_solver_create(const pdot_problem* problem, const pdot_pdhg_parameters* params,
                       const pdot_solver_options* options, pdot_solver** solver) {
  return create_solver(problem, params, options, solver, false);
}

int pdot_solver_create_device(const pdot_problem* device_problem, const pdot_pdhg_parameters* params,
                              const pdot_solver_options* options, pdot_solver** solver) {
  return create_solver(device_problem, params, options, solver, true);
}

int pdot_solver_reset(pdot_solver* solver) {
  return guarded([&] {
    if (!solver) fail(PDOT_ERR_INVALID_ARGUMENT, "null solver");
    solver->impl->reset();
  });
}

int pdot_solver_iterate(pdot_solver* solver, int64_t max_iterations, pdot_solver_status* status) {
  return guarded([&] {
    if (!solver) fail(PDOT_ERR_INVALID_ARGUMENT, "null solver");
    if (max_iterations < 0) fail(PDOT_ERR_INVALID_ARGUMENT, "negative iteration count");
    solver->impl->iterate(max_iterations);
    if (status) solver->impl->fill_status(status);
  });
}

int pdot_solver_finish(pdot_solver* solver, pdot_saddle_point_output* output) {
  return guarded([&] {
    if (!solver || !output) fail(PDOT_ERR_INVALID_ARGUMENT, "null solver or output");
    solver->impl->finish(output);
  });
}

void* pdot_solver_stream(pdot_solver* solver) { return solver ? (void*)solver->impl->stream() : nullptr; }

void pdot_solver_destroy(pdot_solver* solver) {
  if (!solver) return;
  delete solver->impl;
  delete solver;
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

int pdot_rounding_f64(int64_t m, int64_t n, const double* source, const double* target, double* plan,
                      void* stream) {
  return guarded([&] {
    if (m < 1 || n < 1) fail(PDOT_ERR_INVALID_ARGUMENT, "empty matrix");
    if (!source || !target || !plan) fail(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* work = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void**>(&work), pdot::rounding_workspace_doubles(m, n) * sizeof(double), s));
    const cudaError_t e = pdot::launch_rounding(m, n, source, target, plan, work, s);
    const cudaError_t e2 = cudaFreeAsync(work, s);
    CK(e);
    CK(e2);
  });
}

int pdot_rounding_host(int64_t m, int64_t n, const double* source, const double* target, double* plan,
                       int32_t device) {
  return guarded([&] {
    if (m < 1 || n < 1) fail(PDOT_ERR_INVALID_ARGUMENT, "empty matrix");
    if (!source || !target || !plan) fail(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
    require_sm100(device);
    CK(cudaSetDevice(device));
    const size_t N = (size_t)m * (size_t)n;
    double *dX = nullptr, *da = nullptr, *db = nullptr, *work = nullptr;
    const size_t wbytes = pdot::rounding_workspace_doubles(m, n) * sizeof(double);
    cudaError_t e = cudaMalloc(&dX, N * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&da, m * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&db, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&work, wbytes);
    if (e == cudaSuccess) e = cudaMemcpy(dX, plan, N * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(da, source, m * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(db, target, n * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = pdot::launch_rounding(m, n, da, db, dX, work, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(plan, dX, N * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(dX);
    cudaFree(da);
    cudaFree(db);
    cudaFree(work);
    CK(e);
  });
}

int pdot_sqeuclid_cost_f64(int64_t m, int64_t n, int32_t dim, const double* source_points,
                           const double* target_points, int32_t normalise, double* cost, void* stream) {
  return guarded([&] {
    if (m < 1 || n < 1 || dim < 1) fail(PDOT_ERR_INVALID_ARGUMENT, "empty problem");
    if (!source_points || !target_points || !cost) fail(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* work = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void**>(&work), pdot::sqeuclid_workspace_doubles() * sizeof(double), s));
    const cudaError_t e = pdot::launch_sqeuclid_cost(m, n, dim, source_points, target_points, normalise, cost, work, s);
    const cudaError_t e2 = cudaFreeAsync(work, s);
    CK(e);
    CK(e2);
  });
}

}  // extern "C"
