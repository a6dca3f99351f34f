// pdot_warmplan.cu — a warm-start plan recovered from warm-start duals (an
// addition; the reference always starts at zero, src/solver_gpu.jl:428-441).
//
// Given duals (u0, v0) and eps > 0, rounds of log-domain balancing
//   f_i = eps (log a_i - LSE_j((g_j - C_ij) / eps))        (rows sum to a)
//   g_j = eps (log b_j - LSE_i((f_i - C_ij) / eps))        (columns sum to b)
// start from (f, g) = (u0, v0); the plan is X_ij = exp((f_i + g_j - C_ij) / eps)
// and its row and column sums r, c. The solver keeps (u0, v0) as its duals.
// One warp per row or column; every sum in a fixed order, so the result is
// deterministic. The balancing rounds take their exponentials in FP32 (the
// plan is only a starting point); the plan entries and their sums are FP64
// (narrowed to the plan's storage type before they are summed).
#include <cmath>
#include <cstdint>

#include "pdot_device.cuh"

namespace pdot {
namespace {

constexpr int kWpThreads = 256;
constexpr int kWpWarps = kWpThreads / 32;

__device__ __forceinline__ int find_instance(const long long* prefix, int count, long long q) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= q)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// The solver's cost entry C_ij of instance I (coordinate costs in FP32 as the
// primal pass computes them, times the instance's cost scale).
__device__ __forceinline__ double cost_at(const WarmPlanArgs& A, const PlanInstance& I, float scale, int64_t i,
                                          int64_t j) {
  const int64_t e = I.x_off + i + j * I.ld;
  if (A.kind == PDOT_COST_F64) return static_cast<const double*>(A.C)[e];
  if (A.kind == PDOT_COST_F32) return (double)static_cast<const float*>(A.C)[e];
  if (A.kind == PDOT_COST_BF16) return (double)__bfloat162float(static_cast<const __nv_bfloat16*>(A.C)[e]);
  const float* x = A.xs + (I.row_off + i) * A.dim;
  const float* y = A.ys + (I.col_off + j) * A.dim;
  const bool l1 = is_l1_cost(A.kind);
  float acc = 0.0f;
  for (int d = 0; d < A.dim; ++d) {
    const float t = __ldg(x + d) - __ldg(y + d);
    acc = l1 ? acc + fabsf(t) : acc + t * t;
  }
  return (double)(acc * scale);
}

// log-sum-exp accumulator: value = mx + log(s)
struct Lse {
  double mx = -INFINITY;
  float s = 0.0f;
  __device__ __forceinline__ void add(double x) {
    if (x > mx) {
      s = (mx == -INFINITY ? 0.0f : s * expf((float)(mx - x))) + 1.0f;
      mx = x;
    } else if (x > -INFINITY) {
      s += expf((float)(x - mx));
    }
  }
  __device__ __forceinline__ void merge_warp() {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double om = __shfl_xor_sync(0xffffffffu, mx, o);
      const float os = __shfl_xor_sync(0xffffffffu, s, o);
      const double M = om > mx ? om : mx;
      if (M == -INFINITY) continue;
      s = (mx == -INFINITY ? 0.0f : s * expf((float)(mx - M))) + (om == -INFINITY ? 0.0f : os * expf((float)(om - M)));
      mx = M;
    }
  }
};

// One balancing half-round: rows (by_rows) update f from g, columns g from f.
// `first` reads the other side from the warm duals.
__global__ void __launch_bounds__(kWpThreads) k_wp_balance(WarmPlanArgs A, int by_rows, int first) {
  const long long total = by_rows ? A.total_rows : A.total_cols;
  const long long* prefix = by_rows ? A.row_prefix : A.col_prefix;
  const int lane = threadIdx.x & 31;
  for (long long q = (long long)blockIdx.x * kWpWarps + (threadIdx.x >> 5); q < total;
       q += (long long)gridDim.x * kWpWarps) {
    const int k = find_instance(prefix, A.num, q);
    const PlanInstance I = A.inst[k];
    if (!I.active) continue;
    const float scale = (float)A.st[k].cost_scale;
    const double inv = 1.0 / A.eps;
    Lse acc;
    if (by_rows) {
      const int64_t i = q - I.row_off;
      const double* g = first ? A.v0 : A.g;
      for (int64_t j = lane; j < I.n; j += 32) acc.add((g[I.col_off + j] - cost_at(A, I, scale, i, j)) * inv);
      acc.merge_warp();
      if (lane == 0) {
        const double lse = acc.mx + log((double)acc.s);
        A.f[q] = acc.mx == -INFINITY ? -INFINITY : A.eps * (log(A.a[q]) - lse);
      }
    } else {
      const int64_t j = q - I.col_off;
      const double* f = first ? A.u0 : A.f;
      for (int64_t i = lane; i < I.m; i += 32) acc.add((f[I.row_off + i] - cost_at(A, I, scale, i, j)) * inv);
      acc.merge_warp();
      if (lane == 0) {
        const double lse = acc.mx + log((double)acc.s);
        A.g[q] = acc.mx == -INFINITY ? -INFINITY : A.eps * (log(A.b[q]) - lse);
      }
    }
  }
}

template <typename TX>
__device__ __forceinline__ double plan_entry(const WarmPlanArgs& A, const PlanInstance& I, float scale, int64_t i,
                                             int64_t j) {
  const double x = exp((A.f[I.row_off + i] + A.g[I.col_off + j] - cost_at(A, I, scale, i, j)) / A.eps);
  return (double)(TX)x;
}

// The plan by columns (stored, with the column sums), then the row sums of
// the same stored values.
template <typename TX>
__global__ void __launch_bounds__(kWpThreads) k_wp_plan(WarmPlanArgs A, int by_rows) {
  const long long total = by_rows ? A.total_rows : A.total_cols;
  const long long* prefix = by_rows ? A.row_prefix : A.col_prefix;
  const int lane = threadIdx.x & 31;
  TX* X = static_cast<TX*>(A.X);
  for (long long q = (long long)blockIdx.x * kWpWarps + (threadIdx.x >> 5); q < total;
       q += (long long)gridDim.x * kWpWarps) {
    const int k = find_instance(prefix, A.num, q);
    const PlanInstance I = A.inst[k];
    if (!I.active) continue;
    const float scale = (float)A.st[k].cost_scale;
    double s = 0.0;
    if (by_rows) {
      const int64_t i = q - I.row_off;
      for (int64_t j = lane; j < I.n; j += 32) s += plan_entry<TX>(A, I, scale, i, j);
    } else {
      const int64_t j = q - I.col_off;
      for (int64_t i = lane; i < I.m; i += 32) {
        const double x = plan_entry<TX>(A, I, scale, i, j);
        X[I.x_off + i + j * I.ld] = (TX)x;
        s += x;
      }
    }
    s = warp_sum(s);
    if (lane == 0) (by_rows ? A.r : A.c)[q] = s;
  }
}

__global__ void k_wp_copy(const double* __restrict__ src, double* __restrict__ dst, long long count) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < count; e += (long long)gridDim.x * blockDim.x)
    dst[e] = src[e];
}

int wp_grid(long long warps) {
  long long g = (warps + kWpWarps - 1) / kWpWarps;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

cudaError_t launch_warm_plan(const WarmPlanArgs& A, int iterations, cudaStream_t s) {
  // every array the kernels read or write must be in place
  const bool stored = A.kind == PDOT_COST_F64 || A.kind == PDOT_COST_F32 || A.kind == PDOT_COST_BF16;
  if (!A.inst || A.num < 1 || !A.row_prefix || !A.col_prefix || !A.st || !A.a || !A.b || !A.u0 || !A.v0 || !A.f ||
      !A.g || !A.X || !A.r || !A.c || !(A.eps > 0.0) || (stored ? !A.C : (!A.xs || !A.ys || A.dim < 1)))
    return cudaErrorInvalidValue;
  const int rg = wp_grid(A.total_rows), cg = wp_grid(A.total_cols);
  if (iterations <= 0) {
    // the plan from the warm duals themselves
    k_wp_copy<<<rg, kWpThreads, 0, s>>>(A.u0, A.f, A.total_rows);
    k_wp_copy<<<cg, kWpThreads, 0, s>>>(A.v0, A.g, A.total_cols);
  }
  for (int it = 0; it < iterations; ++it) {
    k_wp_balance<<<rg, kWpThreads, 0, s>>>(A, 1, it == 0);
    k_wp_balance<<<cg, kWpThreads, 0, s>>>(A, 0, 0);
  }
  if (A.plan_f32) {
    k_wp_plan<float><<<cg, kWpThreads, 0, s>>>(A, 0);
    k_wp_plan<float><<<rg, kWpThreads, 0, s>>>(A, 1);
  } else {
    k_wp_plan<double><<<cg, kWpThreads, 0, s>>>(A, 0);
    k_wp_plan<double><<<rg, kWpThreads, 0, s>>>(A, 1);
  }
  return cudaGetLastError();
}

}  // namespace pdot
