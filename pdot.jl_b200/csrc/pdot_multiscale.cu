// pdot_multiscale.cu — device passes of the coarse-to-fine warm start for
// point clouds (pdot/multiscale.py): the largest squared distance between two
// point sets, which normalises the squared-Euclidean cost, and the
// semi-discrete c-transform that extends duals known on coarse cells to every
// point, u_i = min_J (scale * ||x_i - c_J||^2 - V_J).
//
// Both are brute force over pairs with the second set staged through shared
// memory in tiles: at 20000 x 15000 points that is 3e8 pairs, a fraction of a
// millisecond, where the same loops on the host took over a second.
#include <cfloat>
#include <cmath>

#include "pdot_common.cuh"

namespace pdot {
namespace {

constexpr int kTile = 256;  // points of the second set per shared-memory tile (= threads per CTA)

// Thread i keeps max_j ||x_i - y_j||^2 (FP64 from FP32 coordinates); a CTA
// reduces its threads and one atomicMax on the bit pattern combines the CTAs
// (non-negative doubles order like their bit patterns).
template <int D>
__global__ void __launch_bounds__(kTile) k_max_sqdist(int64_t m, int64_t n, const float* __restrict__ xs,
                                                      const float* __restrict__ ys,
                                                      unsigned long long* __restrict__ out_bits) {
  __shared__ float ty[kTile * D];
  __shared__ double red[kTile / 32];
  const int64_t i = (int64_t)blockIdx.x * kTile + threadIdx.x;
  double xi[D];
#pragma unroll
  for (int d = 0; d < D; ++d) xi[d] = i < m ? (double)xs[i * D + d] : 0.0;
  double best = 0.0;
  for (int64_t j0 = 0; j0 < n; j0 += kTile) {
    const int64_t cnt = (n - j0) < kTile ? (n - j0) : kTile;
    __syncthreads();
    for (int t = threadIdx.x; t < cnt * D; t += kTile) ty[t] = ys[j0 * D + t];
    __syncthreads();
    if (i < m)
      for (int t = 0; t < cnt; ++t) {
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const double e = xi[d] - (double)ty[t * D + d];
          s += e * e;
        }
        best = s > best ? s : best;
      }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_xor_sync(0xffffffffu, best, o);
    best = y > best ? y : best;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = red[0];
    for (int w = 1; w < kTile / 32; ++w) b = red[w] > b ? red[w] : b;
    atomicMax(out_bits, (unsigned long long)__double_as_longlong(b));
  }
}

// out_i = min_J (scale * ||p_i - c_J||^2 - dual_J), p in FP32, centres and
// duals in FP64, arithmetic in FP64.
template <int D>
__global__ void __launch_bounds__(kTile) k_c_transform(int64_t np, int64_t nc, const float* __restrict__ pts,
                                                       const double* __restrict__ centres,
                                                       const double* __restrict__ duals, double scale,
                                                       double* __restrict__ out) {
  __shared__ double tc[kTile * D];
  __shared__ double tv[kTile];
  const int64_t i = (int64_t)blockIdx.x * kTile + threadIdx.x;
  double p[D];
#pragma unroll
  for (int d = 0; d < D; ++d) p[d] = i < np ? (double)pts[i * D + d] : 0.0;
  double best = INFINITY;
  for (int64_t j0 = 0; j0 < nc; j0 += kTile) {
    const int64_t cnt = (nc - j0) < kTile ? (nc - j0) : kTile;
    __syncthreads();
    for (int t = threadIdx.x; t < cnt * D; t += kTile) tc[t] = centres[j0 * D + t];
    for (int t = threadIdx.x; t < cnt; t += kTile) tv[t] = duals[j0 + t];
    __syncthreads();
    if (i < np)
      for (int t = 0; t < cnt; ++t) {
        double s = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const double e = p[d] - tc[t * D + d];
          s += e * e;
        }
        const double val = scale * s - tv[t];
        best = val < best ? val : best;
      }
  }
  if (i < np) out[i] = best;
}

int report(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

}  // namespace
}  // namespace pdot

extern "C" int pdot_points_max_sqdist(int64_t m, int64_t n, int32_t dim, const float* source_points,
                                      const float* target_points, double* out, void* stream) {
  using namespace pdot;
  set_last_error("");
  if (m < 1 || n < 1) return report(PDOT_ERR_INVALID_ARGUMENT, "empty point set");
  if (dim < 1 || dim > 3) return report(PDOT_ERR_INVALID_ARGUMENT, "point dimension must be 1..3");
  if (!source_points || !target_points || !out) return report(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
  if (e != cudaSuccess) return report(PDOT_ERR_CUDA, cudaGetErrorString(e));
  const unsigned blocks = (unsigned)((m + kTile - 1) / kTile);
  auto* bits = reinterpret_cast<unsigned long long*>(out);
  if (dim == 1)
    k_max_sqdist<1><<<blocks, kTile, 0, s>>>(m, n, source_points, target_points, bits);
  else if (dim == 2)
    k_max_sqdist<2><<<blocks, kTile, 0, s>>>(m, n, source_points, target_points, bits);
  else
    k_max_sqdist<3><<<blocks, kTile, 0, s>>>(m, n, source_points, target_points, bits);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report(PDOT_ERR_CUDA, cudaGetErrorString(e));
  return PDOT_OK;
}

extern "C" int pdot_points_c_transform(int64_t num_points, int64_t num_centres, int32_t dim, const float* points,
                                       const double* centres, const double* duals, double scale, double* out,
                                       void* stream) {
  using namespace pdot;
  set_last_error("");
  if (num_points < 1 || num_centres < 1) return report(PDOT_ERR_INVALID_ARGUMENT, "empty point set");
  if (dim < 1 || dim > 3) return report(PDOT_ERR_INVALID_ARGUMENT, "point dimension must be 1..3");
  if (!points || !centres || !duals || !out) return report(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (!std::isfinite(scale)) return report(PDOT_ERR_INVALID_ARGUMENT, "scale must be finite");
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned blocks = (unsigned)((num_points + kTile - 1) / kTile);
  if (dim == 1)
    k_c_transform<1><<<blocks, kTile, 0, s>>>(num_points, num_centres, points, centres, duals, scale, out);
  else if (dim == 2)
    k_c_transform<2><<<blocks, kTile, 0, s>>>(num_points, num_centres, points, centres, duals, scale, out);
  else
    k_c_transform<3><<<blocks, kTile, 0, s>>>(num_points, num_centres, points, centres, duals, scale, out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return report(PDOT_ERR_CUDA, cudaGetErrorString(e));
  return PDOT_OK;
}
