// pdot_aux.cu — the device passes around a solve: the feasibility rounding of
// a plan and the construction of a squared-Euclidean cost from coordinates.
//
// rounding (src/utils_gpu.jl:296-318): scale the rows by min(1, a / rowsum),
// then the columns by min(1, b / colsum) (a NaN ratio counts as 0), then add
// the rank-one correction err_r * err_c^T with err_r = a - rowsum normalised
// by its 1-norm (when that is not zero) and err_c = b - colsum. Sums are
// two-stage and in a fixed order; each product is rounded as the reference's
// `Diagonal(d) * X`, `X * Diagonal(d)` and `X .+= err_r * err_c'` round it.
#include <cstdint>

#include "pdot_common.cuh"

namespace pdot {
namespace {

constexpr int kAuxThreads = 256;
constexpr int kColChunk = 64;  // columns per CTA of the strided (row) sums

// Row sums, stage one: CTA (rb, cb) sums columns [cb*kColChunk, ...) for rows
// rb*256 + t; partial[cb * m + i]. Consecutive threads read consecutive rows.
__global__ void k_row_partials(int64_t m, int64_t n, const double* __restrict__ X, double* __restrict__ part) {
  const int64_t i = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.y * kColChunk;
  const int64_t j1 = (j0 + kColChunk < n) ? j0 + kColChunk : n;
  if (i >= m) return;
  double s = 0.0;
  for (int64_t j = j0; j < j1; ++j) s += X[i + j * m];
  part[(int64_t)blockIdx.y * m + i] = s;
}

// Column sums: one CTA per column, a fixed-order tree over the contiguous rows.
__global__ void k_col_sums(int64_t m, const double* __restrict__ X, double* __restrict__ out) {
  __shared__ double sh[kAuxThreads];
  const int64_t j = blockIdx.x;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += kAuxThreads) s += X[i + j * m];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kAuxThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = sh[0];
}

__device__ __forceinline__ double row_sum(const double* part, int64_t m, int chunks, int64_t i) {
  double s = 0.0;
  for (int c = 0; c < chunks; ++c) s += part[(int64_t)c * m + i];
  return s;
}

// min(1, dist / sum) with a NaN ratio replaced by 0 (src/utils_gpu.jl:302,305)
__device__ __forceinline__ double scale_of(double dist, double sum) {
  double t = __ddiv_rn(dist, sum);
  if (t != t) t = 0.0;
  return t < 1.0 ? t : 1.0;
}

__global__ void k_row_scales(int64_t m, int chunks, const double* __restrict__ part, const double* __restrict__ a,
                             double* __restrict__ scale) {
  const int64_t i = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x;
  if (i < m) scale[i] = scale_of(a[i], row_sum(part, m, chunks, i));
}

__global__ void k_col_scales(int64_t n, const double* __restrict__ sums, const double* __restrict__ b,
                             double* __restrict__ scale) {
  const int64_t j = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x;
  if (j < n) scale[j] = scale_of(b[j], sums[j]);
}

// X_ij *= row_scale_i (by_row) or col_scale_j
__global__ void k_scale(int64_t m, int64_t n, double* __restrict__ X, const double* __restrict__ scale, int by_row) {
  const int64_t N = m * n;
  for (int64_t e = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x; e < N; e += (int64_t)gridDim.x * kAuxThreads) {
    const int64_t j = e / m, i = e - j * m;
    X[e] = __dmul_rn(by_row ? scale[i] : scale[j], X[e]);
  }
}

// err_r = a - rowsum
__global__ void k_err_rows(int64_t m, int chunks, const double* __restrict__ part, const double* __restrict__ a,
                           double* __restrict__ er) {
  const int64_t i = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x;
  if (i < m) er[i] = __dsub_rn(a[i], row_sum(part, m, chunks, i));
}

// ||err_r||_1 in one CTA (fixed order)
__global__ void k_norm1(int64_t m, const double* __restrict__ er, double* __restrict__ norm1) {
  __shared__ double sh[kAuxThreads];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += kAuxThreads) s += fabs(er[i]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kAuxThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *norm1 = sh[0];
}

// X += (err_r / ||err_r||_1) * (b - colsum)^T
__global__ void k_rank_one(int64_t m, int64_t n, double* __restrict__ X, const double* __restrict__ er,
                           const double* __restrict__ norm1, const double* __restrict__ colsum,
                           const double* __restrict__ b) {
  const double nrm = *norm1;
  const int64_t N = m * n;
  for (int64_t e = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x; e < N; e += (int64_t)gridDim.x * kAuxThreads) {
    const int64_t j = e / m, i = e - j * m;
    const double r = nrm != 0.0 ? __ddiv_rn(er[i], nrm) : er[i];
    const double c = __dsub_rn(b[j], colsum[j]);
    X[e] = __dadd_rn(X[e], __dmul_rn(r, c));
  }
}

// C_ij = ||x_i - y_j||^2 in FP64, then divided by its maximum when `normalise`.
__global__ void k_sqeuclid(int64_t m, int64_t n, int dim, const double* __restrict__ xs,
                           const double* __restrict__ ys, double* __restrict__ C) {
  const int64_t N = m * n;
  for (int64_t e = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x; e < N; e += (int64_t)gridDim.x * kAuxThreads) {
    const int64_t j = e / m, i = e - j * m;
    double s = 0.0;
    for (int d = 0; d < dim; ++d) {
      const double t = __dsub_rn(xs[i * dim + d], ys[j * dim + d]);
      s = __dadd_rn(s, __dmul_rn(t, t));
    }
    C[e] = s;
  }
}

__global__ void k_max_partials(int64_t N, const double* __restrict__ C, double* __restrict__ part) {
  __shared__ double sh[kAuxThreads];
  double mx = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x; e < N; e += (int64_t)gridDim.x * kAuxThreads)
    mx = fmax(mx, C[e]);
  sh[threadIdx.x] = mx;
  __syncthreads();
  for (int w = kAuxThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_divide_by_max(int64_t N, double* __restrict__ C, const double* __restrict__ part, int parts) {
  double mx = 0.0;
  for (int k = 0; k < parts; ++k) mx = fmax(mx, part[k]);
  if (!(mx > 0.0)) return;
  for (int64_t e = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x; e < N; e += (int64_t)gridDim.x * kAuxThreads)
    C[e] = __ddiv_rn(C[e], mx);
}

// Row and column sums of a plan in storage type TX (the sums of a warm-start
// plan): row partials over column chunks, then their fixed-order total; one CTA
// per column for the column sums.
template <typename TX>
__global__ void k_plan_row_partials(int64_t m, int64_t n, const TX* __restrict__ X, double* __restrict__ part) {
  const int64_t i = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.y * kColChunk;
  const int64_t j1 = (j0 + kColChunk < n) ? j0 + kColChunk : n;
  if (i >= m) return;
  double s = 0.0;
  for (int64_t j = j0; j < j1; ++j) s += (double)X[i + j * m];
  part[(int64_t)blockIdx.y * m + i] = s;
}

template <typename TX>
__global__ void k_plan_col_sums(int64_t m, const TX* __restrict__ X, double* __restrict__ out) {
  __shared__ double sh[kAuxThreads];
  const int64_t j = blockIdx.x;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += kAuxThreads) s += (double)X[i + j * m];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kAuxThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = sh[0];
}

__global__ void k_plan_row_totals(int64_t m, int chunks, const double* __restrict__ part, double* __restrict__ r) {
  const int64_t i = (int64_t)blockIdx.x * kAuxThreads + threadIdx.x;
  if (i < m) r[i] = row_sum(part, m, chunks, i);
}

int grid_for(int64_t count) {
  int64_t g = (count + kAuxThreads - 1) / kAuxThreads;
  return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

}  // namespace

size_t rounding_workspace_doubles(int64_t m, int64_t n) {
  const int64_t chunks = (n + kColChunk - 1) / kColChunk;
  return (size_t)chunks * m + 2 * (size_t)m + 2 * (size_t)n + 1;
}

cudaError_t launch_rounding(int64_t m, int64_t n, const double* a, const double* b, double* X, double* work,
                            cudaStream_t s) {
  const int chunks = (int)((n + kColChunk - 1) / kColChunk);
  double* part = work;
  double* rscale = part + (size_t)chunks * m;  // row scales, later err_r
  double* colsum = rscale + m;                 // column sums
  double* cscale = colsum + n;
  double* norm1 = cscale + n;
  const dim3 rgrid((unsigned)((m + kAuxThreads - 1) / kAuxThreads), (unsigned)chunks);
  const int rb = (int)((m + kAuxThreads - 1) / kAuxThreads), cbk = (int)((n + kAuxThreads - 1) / kAuxThreads);
  const int eg = grid_for(m * n);
  k_row_partials<<<rgrid, kAuxThreads, 0, s>>>(m, n, X, part);
  k_row_scales<<<rb, kAuxThreads, 0, s>>>(m, chunks, part, a, rscale);
  k_scale<<<eg, kAuxThreads, 0, s>>>(m, n, X, rscale, 1);
  k_col_sums<<<(unsigned)n, kAuxThreads, 0, s>>>(m, X, colsum);
  k_col_scales<<<cbk, kAuxThreads, 0, s>>>(n, colsum, b, cscale);
  k_scale<<<eg, kAuxThreads, 0, s>>>(m, n, X, cscale, 0);
  k_row_partials<<<rgrid, kAuxThreads, 0, s>>>(m, n, X, part);
  k_err_rows<<<rb, kAuxThreads, 0, s>>>(m, chunks, part, a, rscale);
  k_norm1<<<1, kAuxThreads, 0, s>>>(m, rscale, norm1);
  k_col_sums<<<(unsigned)n, kAuxThreads, 0, s>>>(m, X, colsum);
  k_rank_one<<<eg, kAuxThreads, 0, s>>>(m, n, X, rscale, norm1, colsum, b);
  return cudaGetLastError();
}

size_t plan_sums_workspace_doubles(int64_t m, int64_t n) {
  return (size_t)((n + kColChunk - 1) / kColChunk) * (size_t)m;
}

cudaError_t launch_plan_sums(int64_t m, int64_t n, const void* X, int plan_f32, double* r, double* c, double* work,
                             cudaStream_t s) {
  const int chunks = (int)((n + kColChunk - 1) / kColChunk);
  const dim3 rgrid((unsigned)((m + kAuxThreads - 1) / kAuxThreads), (unsigned)chunks);
  const int rb = (int)((m + kAuxThreads - 1) / kAuxThreads);
  if (plan_f32) {
    k_plan_row_partials<float><<<rgrid, kAuxThreads, 0, s>>>(m, n, static_cast<const float*>(X), work);
    k_plan_col_sums<float><<<(unsigned)n, kAuxThreads, 0, s>>>(m, static_cast<const float*>(X), c);
  } else {
    k_plan_row_partials<double><<<rgrid, kAuxThreads, 0, s>>>(m, n, static_cast<const double*>(X), work);
    k_plan_col_sums<double><<<(unsigned)n, kAuxThreads, 0, s>>>(m, static_cast<const double*>(X), c);
  }
  k_plan_row_totals<<<rb, kAuxThreads, 0, s>>>(m, chunks, work, r);
  return cudaGetLastError();
}

size_t sqeuclid_workspace_doubles() { return 148 * 4; }

cudaError_t launch_sqeuclid_cost(int64_t m, int64_t n, int dim, const double* xs, const double* ys, int normalise,
                                 double* C, double* work, cudaStream_t s) {
  const int64_t N = m * n;
  const int eg = grid_for(N);
  k_sqeuclid<<<eg, kAuxThreads, 0, s>>>(m, n, dim, xs, ys, C);
  if (normalise) {
    const int parts = 148 * 4;
    k_max_partials<<<parts, kAuxThreads, 0, s>>>(N, C, work);
    k_divide_by_max<<<eg, kAuxThreads, 0, s>>>(N, C, work, parts);
  }
  return cudaGetLastError();
}

}  // namespace pdot
