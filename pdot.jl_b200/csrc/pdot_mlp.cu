// pdot_mlp.cu — the network of the learned warm start: an MLP
// input -> hidden -> hidden -> output with GELU, BF16 weights (FP32 master
// copies and AdamW state), BF16 activations and FP32 accumulation.
//
// Every matrix product runs on the 5th-generation tensor cores through one
// hand-written kernel, k_gemm: D[M x N] = A[M x K] . B[N x K]^T with A and B
// BF16 and K-major (K contiguous). TMA moves 128 x 64 tiles of A and B into
// shared memory with the 128-byte swizzle, one thread issues tcgen05.mma
// (M = 128, N = 128, K = 16 per instruction) into a TMEM accumulator, each
// stage of the 4-deep ring is released by tcgen05.commit on its mbarrier, and
// the four warps read the accumulator back with tcgen05.ld for a fused
// epilogue (bias, GELU or the GELU derivative) that also writes the transposed
// BF16 copy the backward products read. With every operand K-major:
//
//   forward   Z1 = X  W1^T + b1, H1 = gelu(Z1)     A = X  [B x I],  B = W1 [H x I]
//             Z2 = H1 W2^T + b2, H2 = gelu(Z2)     A = H1,          B = W2
//             Y  = H2 W3^T + b3                    A = H2,          B = W3 [O x H]
//   backward  dW3 = dY^T H2                        A = dY^T [O x B], B = H2^T [H x B]
//             dZ2 = (dY W3) * gelu'(Z2)            A = dY [B x O],   B = W3^T [H x O]
//             dW2 = dZ2^T H1,  dZ1 = (dZ2 W2) * gelu'(Z1),  dW1 = dZ1^T X
//
// The loss is the mean squared error over the output entries of the real rows
// of the batch. All reductions (loss, bias gradients) are in a fixed order.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "pdot_device.cuh"

namespace pdot {
namespace {

// Build knob: PDOT_MLP_SPLIT_K 0 runs every product as one tile per CTA.
#ifndef PDOT_MLP_SPLIT_K
#define PDOT_MLP_SPLIT_K 1
#endif
constexpr int kGemmThreads = 128;
constexpr int kBM = 128;  // rows of A per tile (= TMEM lanes)
constexpr int kBN = 128;  // rows of B per tile (= accumulator columns)
constexpr int kBK = 64;   // K per stage: one 128-byte swizzle row of BF16
constexpr int kUmmaK = 16;
constexpr int kStages = 4;
constexpr int kTileABytes = kBM * kBK * 2;
constexpr int kTileBBytes = kBN * kBK * 2;
constexpr int kStageBytes = kTileABytes + kTileBBytes;
constexpr int kGemmSmem = kStages * kStageBytes + 1024 + 256;

enum { EPI_F32 = 0, EPI_BIAS_GELU = 1, EPI_BIAS = 2, EPI_GELU_BWD = 3 };

// Error codes a kernel leaves in the error word.
enum { kErrWaitFull = 1, kErrWaitEmpty = 2, kErrWaitDone = 3 };

struct Epi {
  float* f32;                  // row-major M x N (ld_f32)
  __nv_bfloat16* bf16;         // row-major M x N (ld_bf16)
  __nv_bfloat16* bf16_t;       // transposed: entry (r, c) at [c * ld_t + r]
  const float* bias;           // N
  const float* z;              // saved pre-activation, row-major (ld_z)
  int64_t ld_f32, ld_bf16, ld_t, ld_z;
  float* part;                 // split K: slice z of the partial products at part + z * M * N (row-major M x N)
  int64_t part_m, part_n;      // M and N of the product
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor of a K-major operand tile written by TMA with
// the 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart
// (stride byte offset), descriptor version 1, layout SWIZZLE_128B (2).
__device__ __forceinline__ uint64_t sw128_kmajor_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;            // leading byte offset (unused by swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;  // stride byte offset
  d |= (uint64_t)1 << 46;            // version
  d |= (uint64_t)2 << 61;            // SWIZZLE_128B
  return d;
}

// Instruction descriptor: kind::f16 with BF16 A and B, FP32 accumulator,
// both K-major, N = kBN, M = kBM.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// D (+)= A B^T for one K = 16 step; no output lane disabled.
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  const uint32_t z = 0u;
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// GELU with the error function, and its derivative.
__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// The fused epilogue of W (a multiple of 4) accumulator columns [col, col + W)
// of one row.
template <int EPI, int W>
__device__ __forceinline__ void epilogue_cols(const Epi& ep, int64_t row, int64_t col, float (&v)[W]) {
  if (EPI == EPI_BIAS_GELU || EPI == EPI_BIAS) {
#pragma unroll
    for (int k = 0; k < W; ++k) v[k] += __ldg(ep.bias + col + k);
  }
  if (EPI == EPI_GELU_BWD) {
    const float* zr = ep.z + row * ep.ld_z + col;
#pragma unroll
    for (int k = 0; k < W; k += 4) {
      const float4 z4 = *reinterpret_cast<const float4*>(zr + k);
      v[k] *= gelu_grad(z4.x);
      v[k + 1] *= gelu_grad(z4.y);
      v[k + 2] *= gelu_grad(z4.z);
      v[k + 3] *= gelu_grad(z4.w);
    }
  }
  float* fo = ep.f32 + row * ep.ld_f32 + col;
#pragma unroll
  for (int k = 0; k < W; k += 4) *reinterpret_cast<float4*>(fo + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
  if (EPI == EPI_BIAS_GELU || EPI == EPI_GELU_BWD) {
    __align__(16) __nv_bfloat16 h[W];
#pragma unroll
    for (int k = 0; k < W; ++k) h[k] = __float2bfloat16_rn(EPI == EPI_BIAS_GELU ? gelu(v[k]) : v[k]);
    if (ep.bf16) {
      __nv_bfloat16* bo = ep.bf16 + row * ep.ld_bf16 + col;
#pragma unroll
      for (int k = 0; k < W; k += 4) *reinterpret_cast<uint2*>(bo + k) = *reinterpret_cast<const uint2*>(h + k);
    }
#pragma unroll
    for (int k = 0; k < W; ++k) ep.bf16_t[(col + k) * ep.ld_t + row] = h[k];
  }
}

// One 128 x 128 tile of D = A B^T per CTA; K a multiple of kBK. With
// gridDim.z = S > 1 (split K), CTA z multiplies the K blocks
// [z * KB / S, (z + 1) * KB / S) and writes its raw partial tile to slice z of
// ep.part; k_splitk_finish then adds the slices in order and runs the
// epilogue. Products with few output tiles (the batch is 256 rows) thus
// spread over the SMs instead of 16 of them.
template <int EPI>
__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, int K, Epi ep, int* err) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_addr(smem_raw);
  const uint32_t tiles = (raw + 1023u) & ~1023u;  // the swizzle atoms need 1024-byte alignment
  const uint32_t bars = tiles + kStages * kStageBytes;
  auto full = [&](int s) { return bars + 8u * s; };
  auto empty = [&](int s) { return bars + 8u * (kStages + s); };
  const uint32_t done = bars + 8u * (2 * kStages);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_raw + (bars - raw) + 8 * (2 * kStages + 1));
  __shared__ int s_err;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int kb_all = K / kBK;
  const int kb0 = (int)((long long)blockIdx.z * kb_all / gridDim.z);
  const int kblocks = (int)((long long)(blockIdx.z + 1) * kb_all / gridDim.z) - kb0;
  if (threadIdx.x == 0) {
    s_err = 0;
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    mbar_init(done, 1);
    fence_mbar_init();
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(kBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // producer: TMA loads of the A and B tiles of each K block
    int issued = 0;
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb % kStages;
      if (kb >= kStages && !mbar_wait_bounded(empty(s), ((kb / kStages) & 1) ^ 1)) {
        atomicCAS(&s_err, 0, kErrWaitEmpty);
        break;
      }
      mbar_expect_tx(full(s), kStageBytes);
      tma_load_2d(tiles + s * kStageBytes, &ta, full(s), (kb0 + kb) * kBK, m0);
      tma_load_2d(tiles + s * kStageBytes + kTileABytes, &tb, full(s), (kb0 + kb) * kBK, n0);
      issued = kb + 1;
    }
    // every copy issued has landed before the CTA may leave (already true on
    // the normal path, where the MMAs consumed them)
    for (int kb = (issued > kStages ? issued - kStages : 0); kb < issued; ++kb)
      if (!mbar_wait_bounded(full(kb % kStages), (kb / kStages) & 1)) atomicCAS(&s_err, 0, kErrWaitFull);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    for (int kb = 0; kb < kblocks; ++kb) {
      const int s = kb % kStages;
      if (!mbar_wait_bounded(full(s), (kb / kStages) & 1)) {
        atomicCAS(&s_err, 0, kErrWaitFull);
        break;
      }
      tc_fence_after();
      const uint64_t da = sw128_kmajor_desc(tiles + s * kStageBytes);
      const uint64_t db = sw128_kmajor_desc(tiles + s * kStageBytes + kTileABytes);
#pragma unroll
      for (int kk = 0; kk < kBK / kUmmaK; ++kk)  // +32 bytes along the swizzled row per K step
        umma_bf16(tmem, da + (uint64_t)(2 * kk), db + (uint64_t)(2 * kk), (kb | kk) != 0 ? 1u : 0u);
      umma_commit(empty(s));
    }
    umma_commit(done);
  }
  __syncwarp();
  if (!mbar_wait_bounded(done, 0)) atomicCAS(&s_err, 0, kErrWaitDone);
  __syncwarp();
  tc_fence_after();

  // epilogue: thread (warp w, lane l) owns accumulator row 32 w + l
  const int64_t row = m0 + warp * 32 + lane;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const bool split = gridDim.z > 1;
#pragma unroll 1
  for (int c0 = 0; c0 < kBN; c0 += 16) {
    float v[16];
    tmem_ld16(lane_base + (uint32_t)c0, v);
    const int64_t col = n0 + c0;
    if (split) {
      float* po = ep.part + ((int64_t)blockIdx.z * ep.part_m + row) * ep.part_n + col;
#pragma unroll
      for (int k = 0; k < 16; k += 4) *reinterpret_cast<float4*>(po + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
    } else {
      epilogue_cols<EPI, 16>(ep, row, col, v);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN) : "memory");
  }
  if (threadIdx.x == 0 && s_err != 0) atomicCAS(err, 0, s_err);
}

// Split K: D = the sum of the S partial slices in order z = 0, 1, ..., then the
// epilogue; a thread per (row, 4 columns), consecutive threads on consecutive
// rows (the transposed BF16 copy's stores coalesce). The slices' loads are
// issued together (S <= kMaxSplit), the additions keep their order.
constexpr int kMaxSplit = 16;
template <int EPI>
__global__ void __launch_bounds__(256) k_splitk_finish(Epi ep, int S) {
  const int64_t M = ep.part_m, N = ep.part_n, total = M * (N / 4);
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = t % M, col = (t / M) * 4;
    float4 q[kMaxSplit];
#pragma unroll
    for (int z = 0; z < kMaxSplit; ++z)
      if (z < S) q[z] = __ldcs(reinterpret_cast<const float4*>(ep.part + ((int64_t)z * M + row) * N + col));
    float v[4] = {q[0].x, q[0].y, q[0].z, q[0].w};
#pragma unroll
    for (int z = 1; z < kMaxSplit; ++z)
      if (z < S) v[0] += q[z].x, v[1] += q[z].y, v[2] += q[z].z, v[3] += q[z].w;
    epilogue_cols<EPI, 4>(ep, row, col, v);
  }
}

constexpr int kEw = 256;  // threads of the elementwise kernels

// x[r, k] = bf16((log(max(h, 1e-30)) + shift) * scale) for real rows, 0 for the
// padding rows up to bp; also the transposed copy xt (leading dimension ld_t).
__global__ void k_features(const double* __restrict__ hist, int64_t batch, int64_t bp, int64_t dim, double shift,
                           double scale, __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ xt,
                           int64_t ld_t) {
  const int64_t N = bp * dim;
  for (int64_t e = (int64_t)blockIdx.x * kEw + threadIdx.x; e < N; e += (int64_t)gridDim.x * kEw) {
    const int64_t r = e / dim, k = e - r * dim;
    double f = 0.0;
    if (r < batch) {
      const double h = hist[e];
      f = (log(h > 1e-30 ? h : 1e-30) + shift) * scale;
    }
    const __nv_bfloat16 b = __double2bfloat16(f);
    x[e] = b;
    xt[k * ld_t + r] = b;
  }
}

// dY = 2 (Y - T) / (batch * O) on real rows (0 on padding), its BF16 copy and
// transpose, and per-CTA partial sums of (Y - T)^2.
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, int64_t batch, int64_t bp,
                       int64_t dim, float* __restrict__ dy, __nv_bfloat16* __restrict__ dyb,
                       __nv_bfloat16* __restrict__ dyt, int64_t ld_t, double* __restrict__ part) {
  const int64_t N = bp * dim;
  const float g = 2.0f / (float)(batch * dim);
  double acc = 0.0;
  for (int64_t e = (int64_t)blockIdx.x * kEw + threadIdx.x; e < N; e += (int64_t)gridDim.x * kEw) {
    const int64_t r = e / dim, k = e - r * dim;
    float d = 0.0f;
    if (r < batch) {
      const float diff = y[e] - t[e];
      acc += (double)diff * (double)diff;
      d = g * diff;
    }
    dy[e] = d;
    const __nv_bfloat16 b = __float2bfloat16_rn(d);
    dyb[e] = b;
    dyt[k * ld_t + r] = b;
  }
  __shared__ double sh[kEw];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kEw / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

__global__ void k_loss_total(const double* __restrict__ part, int parts, int64_t count, double* __restrict__ loss) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int k = 0; k < parts; ++k) s += part[k];
  *loss = s / (double)count;
}

// out[c] = sum over the first `rows` rows of in[r, c] (bias gradients)
__global__ void k_colsum(const float* __restrict__ in, int64_t rows, int64_t cols, float* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * kEw + threadIdx.x;
  if (c >= cols) return;
  double s = 0.0;
  for (int64_t r = 0; r < rows; ++r) s += (double)in[r * cols + c];
  out[c] = (float)s;
}

// AdamW on one tensor (rows x cols; a bias has rows = 1 and no BF16 copies):
// m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2,
// p -= lr (m / (1 - b1^t) / (sqrt(v / (1 - b2^t)) + eps) + wd p);
// then the BF16 copy and its transpose.
__global__ void k_adamw(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                        float* __restrict__ v, int64_t rows, int64_t cols, float lr, float b1, float b2, float eps,
                        float wd, float c1, float c2, __nv_bfloat16* __restrict__ pb,
                        __nv_bfloat16* __restrict__ pt) {
  const int64_t N = rows * cols;
  for (int64_t e = (int64_t)blockIdx.x * kEw + threadIdx.x; e < N; e += (int64_t)gridDim.x * kEw) {
    const float gr = g[e];
    const float mm = b1 * m[e] + (1.0f - b1) * gr;
    const float vv = b2 * v[e] + (1.0f - b2) * gr * gr;
    m[e] = mm;
    v[e] = vv;
    const float upd = (mm / c1) / (sqrtf(vv / c2) + eps) + wd * p[e];
    const float np = p[e] - lr * upd;
    p[e] = np;
    if (pb) {
      const __nv_bfloat16 b = __float2bfloat16_rn(np);
      pb[e] = b;
      const int64_t r = e / cols, c = e - r * cols;
      pt[c * rows + r] = b;
    }
  }
}

// BF16 copies (and transposes) of the weight matrices from the FP32 masters.
__global__ void k_to_bf16(const float* __restrict__ p, int64_t rows, int64_t cols, __nv_bfloat16* __restrict__ pb,
                          __nv_bfloat16* __restrict__ pt) {
  const int64_t N = rows * cols;
  for (int64_t e = (int64_t)blockIdx.x * kEw + threadIdx.x; e < N; e += (int64_t)gridDim.x * kEw) {
    const __nv_bfloat16 b = __float2bfloat16_rn(p[e]);
    pb[e] = b;
    const int64_t r = e / cols, c = e - r * cols;
    pt[c * rows + r] = b;
  }
}

int ew_grid(int64_t n) {
  int64_t g = (n + kEw - 1) / kEw;
  return (int)(g < 1 ? 1 : (g > 148 * 8 ? 148 * 8 : g));
}

}  // namespace
}  // namespace pdot

// ---------------------------------------------------------------------------
// Host side
namespace {

struct MlpFailure {
  int code;
  std::string msg;
};

[[noreturn]] void mfail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw MlpFailure{code, buf};
}

void mck(cudaError_t e, const char* what, int line) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    mfail(e == cudaErrorMemoryAllocation ? PDOT_ERR_OUT_OF_MEMORY : PDOT_ERR_CUDA, "%s failed: %s (pdot_mlp.cu:%d)",
          what, cudaGetErrorString(e), line);
  }
}
#define MCK(x) mck((x), #x, __LINE__)

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static std::mutex mu;
  static EncodeTiledFn fn = nullptr;
  std::lock_guard<std::mutex> lock(mu);
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p) {
      cudaGetLastError();
      mfail(PDOT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    }
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Tensor map of a row-major BF16 matrix [rows x cols] read in 128 x 64 boxes
// with the 128-byte swizzle (cols a multiple of 64, rows of 128).
CUtensorMap make_map(const __nv_bfloat16* base, int64_t rows, int64_t cols) {
  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  const cuuint32_t box[2] = {(cuuint32_t)pdot::kBK, (cuuint32_t)pdot::kBM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(base), dims,
                                 strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) mfail(PDOT_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d) for a %lld x %lld matrix", (int)r,
                               (long long)rows, (long long)cols);
  return map;
}

using bf16 = __nv_bfloat16;

}  // namespace

struct pdot_mlp {
  int device = 0;
  int64_t I = 0, H = 0, O = 0, Bp = 0;  // dimensions; Bp = batch capacity (multiple of 128)
  int64_t P = 0;                        // parameters
  int64_t step = 0;                     // AdamW steps taken
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  // FP32 masters, gradients, AdamW moments (layout W1, b1, W2, b2, W3, b3)
  float *theta = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
  float *W[3] = {}, *b[3] = {}, *gW[3] = {}, *gb[3] = {};
  bf16 *Wb[3] = {}, *Wt[3] = {};
  // activations
  bf16 *x = nullptr, *xt = nullptr, *h1 = nullptr, *h1t = nullptr, *h2 = nullptr, *h2t = nullptr;
  float *z1 = nullptr, *z2 = nullptr, *y = nullptr;
  float *dy = nullptr, *dz2 = nullptr, *dz1 = nullptr;
  bf16 *dyb = nullptr, *dyt = nullptr, *dz2b = nullptr, *dz2t = nullptr, *dz1t = nullptr;
  double *loss_part = nullptr, *loss = nullptr;
  int* err = nullptr;
  float* part = nullptr;  // split-K partial products: at most one 128 x 128 tile per SM
  int sms = 148;
  int loss_parts = 0;
  int64_t batch = 0;  // rows of the current input
  // tensor maps of every GEMM operand
  CUtensorMap mx, mW[3], mh1, mh2, mdyt, mh2t, mdyb, mWt[3], mdz2t, mh1t, mdz2b, mdz1t, mxt;

  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    MCK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocs.push_back(p);
    MCK(cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), stream));
    return static_cast<T*>(p);
  }

  ~pdot_mlp() {
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : allocs) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }

  void sync_bf16() {
    const int64_t rows[3] = {H, H, O}, cols[3] = {I, H, H};
    for (int l = 0; l < 3; ++l)
      pdot::k_to_bf16<<<pdot::ew_grid(rows[l] * cols[l]), pdot::kEw, 0, stream>>>(W[l], rows[l], cols[l], Wb[l], Wt[l]);
    MCK(cudaGetLastError());
  }

  void check_err() {
    int e = 0;
    MCK(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    MCK(cudaStreamSynchronize(stream));
    if (e != 0) {
      MCK(cudaMemsetAsync(err, 0, sizeof(int), stream));
      mfail(PDOT_ERR_CUDA, "a tensor-core GEMM gave up waiting on its pipeline (code %d)", e);
    }
  }

  template <int EPI>
  void gemm(const CUtensorMap& a, const CUtensorMap& bm, int64_t M, int64_t N, int64_t K, const pdot::Epi& ep) {
    if (M % pdot::kBM || N % pdot::kBN || K % pdot::kBK || K <= 0)
      mfail(PDOT_ERR_INVALID_ARGUMENT, "GEMM shape %lld x %lld x %lld is not tiled by 128 x 128 x 64", (long long)M,
            (long long)N, (long long)K);
    MCK(cudaFuncSetAttribute(pdot::k_gemm<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, pdot::kGemmSmem));
    // split K where the tiles cover at most an eighth of the SMs (the batch's
    // 256-row products with a 1024-wide output), while the slices fill at
    // most every SM and each keeps at least two K blocks. Measured per launch
    // (ncu, cold cache) for 256 x 1024 x 2048: 8.9 us + 6.3 us for the
    // ordered sum and epilogue, against 22.5 us in one K loop; 256 x 2048 x
    // 1024 (32 tiles) split in four measured 16.6 us against 14.4 us, so it
    // stays whole, as do the weight gradients (64 and more tiles).
    const int64_t tiles = (N / pdot::kBN) * (M / pdot::kBM), kb = K / pdot::kBK;
    int S = 1;
    if (PDOT_MLP_SPLIT_K && tiles * 8 <= sms)
      while (tiles * S * 2 <= sms && kb / (S * 2) >= 2 && S * 2 <= pdot::kMaxSplit) S *= 2;
    const dim3 grid((unsigned)(N / pdot::kBN), (unsigned)(M / pdot::kBM), (unsigned)S);
    pdot::Epi e = ep;
    e.part = part;
    e.part_m = M;
    e.part_n = N;
    pdot::k_gemm<EPI><<<grid, pdot::kGemmThreads, pdot::kGemmSmem, stream>>>(a, bm, (int)K, e, err);
    MCK(cudaGetLastError());
    if (S > 1) {
      const int64_t threads = M * (N / 4);
      const int blocks = (int)std::min<int64_t>((threads + 255) / 256, (int64_t)sms * 8);
      pdot::k_splitk_finish<EPI><<<blocks, 256, 0, stream>>>(e, S);
      MCK(cudaGetLastError());
    }
  }

  int64_t padded(int64_t rows) const { return (rows + pdot::kBM - 1) / pdot::kBM * pdot::kBM; }

  void forward() {
    const int64_t bp = padded(batch);
    pdot::Epi e{};
    e.f32 = z1; e.ld_f32 = H; e.bf16 = h1; e.ld_bf16 = H; e.bf16_t = h1t; e.ld_t = Bp; e.bias = b[0];
    gemm<pdot::EPI_BIAS_GELU>(mx, mW[0], bp, H, I, e);
    e = pdot::Epi{};
    e.f32 = z2; e.ld_f32 = H; e.bf16 = h2; e.ld_bf16 = H; e.bf16_t = h2t; e.ld_t = Bp; e.bias = b[1];
    gemm<pdot::EPI_BIAS_GELU>(mh1, mW[1], bp, H, H, e);
    e = pdot::Epi{};
    e.f32 = y; e.ld_f32 = O; e.bias = b[2];
    gemm<pdot::EPI_BIAS>(mh2, mW[2], bp, O, H, e);
  }

  void backward(const float* target) {
    const int64_t bp = padded(batch);
    pdot::k_loss<<<loss_parts, pdot::kEw, 0, stream>>>(y, target, batch, bp, O, dy, dyb, dyt, Bp, loss_part);
    pdot::k_loss_total<<<1, 32, 0, stream>>>(loss_part, loss_parts, batch * O, loss);
    MCK(cudaGetLastError());
    // the transposed operands were written with leading dimension Bp; the
    // products over the batch read the first bp columns of them
    pdot::Epi e{};
    e.f32 = gW[2]; e.ld_f32 = H;
    gemm<pdot::EPI_F32>(mdyt, mh2t, O, H, bp, e);
    e = pdot::Epi{};
    e.f32 = dz2; e.ld_f32 = H; e.bf16 = dz2b; e.ld_bf16 = H; e.bf16_t = dz2t; e.ld_t = Bp; e.z = z2; e.ld_z = H;
    gemm<pdot::EPI_GELU_BWD>(mdyb, mWt[2], bp, H, O, e);
    e = pdot::Epi{};
    e.f32 = gW[1]; e.ld_f32 = H;
    gemm<pdot::EPI_F32>(mdz2t, mh1t, H, H, bp, e);
    e = pdot::Epi{};
    e.f32 = dz1; e.ld_f32 = H; e.bf16 = nullptr; e.bf16_t = dz1t; e.ld_t = Bp; e.z = z1; e.ld_z = H;
    gemm<pdot::EPI_GELU_BWD>(mdz2b, mWt[1], bp, H, H, e);
    e = pdot::Epi{};
    e.f32 = gW[0]; e.ld_f32 = I;
    gemm<pdot::EPI_F32>(mdz1t, mxt, H, I, bp, e);
    pdot::k_colsum<<<(unsigned)((O + pdot::kEw - 1) / pdot::kEw), pdot::kEw, 0, stream>>>(dy, bp, O, gb[2]);
    pdot::k_colsum<<<(unsigned)((H + pdot::kEw - 1) / pdot::kEw), pdot::kEw, 0, stream>>>(dz2, bp, H, gb[1]);
    pdot::k_colsum<<<(unsigned)((H + pdot::kEw - 1) / pdot::kEw), pdot::kEw, 0, stream>>>(dz1, bp, H, gb[0]);
    MCK(cudaGetLastError());
  }

  void adamw(float lr, float b1_, float b2_, float eps, float wd) {
    ++step;
    const float c1 = 1.0f - powf(b1_, (float)step), c2 = 1.0f - powf(b2_, (float)step);
    const int64_t rows[3] = {H, H, O}, cols[3] = {I, H, H};
    for (int l = 0; l < 3; ++l) {
      const int64_t off_w = W[l] - theta, off_b = b[l] - theta;
      pdot::k_adamw<<<pdot::ew_grid(rows[l] * cols[l]), pdot::kEw, 0, stream>>>(
          W[l], grad + off_w, m1 + off_w, m2 + off_w, rows[l], cols[l], lr, b1_, b2_, eps, wd, c1, c2, Wb[l], Wt[l]);
      pdot::k_adamw<<<pdot::ew_grid(rows[l]), pdot::kEw, 0, stream>>>(b[l], grad + off_b, m1 + off_b, m2 + off_b, 1,
                                                                      rows[l], lr, b1_, b2_, eps, 0.0f, c1, c2,
                                                                      nullptr, nullptr);
    }
    MCK(cudaGetLastError());
  }
};

namespace {

int mguarded(const std::function<void()>& f) {
  try {
    f();
    return PDOT_OK;
  } catch (const MlpFailure& e) {
    pdot::set_last_error(e.msg.c_str());
    return e.code;
  } catch (const std::bad_alloc&) {
    pdot::set_last_error("host allocation failed");
    return PDOT_ERR_OUT_OF_MEMORY;
  } catch (...) {
    pdot::set_last_error("unknown failure");
    return PDOT_ERR_CUDA;
  }
}

// splitmix64, for the initial weights
uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
}  // namespace

extern "C" int pdot_mlp_create(int32_t device, int64_t input_dim, int64_t hidden_dim, int64_t output_dim,
                               int64_t max_batch, uint64_t seed, pdot_mlp** out) {
  return mguarded([&] {
    if (!out) mfail(PDOT_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (input_dim <= 0 || hidden_dim <= 0 || output_dim <= 0 || input_dim % 128 || hidden_dim % 128 ||
        output_dim % 128)
      mfail(PDOT_ERR_INVALID_ARGUMENT, "the layer widths must be positive multiples of 128");
    if (max_batch <= 0 || max_batch > (1 << 20)) mfail(PDOT_ERR_INVALID_ARGUMENT, "max_batch must be 1..2^20");
    int count = 0;
    MCK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) mfail(PDOT_ERR_NO_DEVICE, "no CUDA device %d", device);
    cudaDeviceProp prop;
    MCK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) mfail(PDOT_ERR_NO_DEVICE, "the tensor-core kernels need an sm_100 device");
    MCK(cudaSetDevice(device));
    std::unique_ptr<pdot_mlp> m(new pdot_mlp);
    m->device = device;
    m->I = input_dim;
    m->H = hidden_dim;
    m->O = output_dim;
    m->Bp = (max_batch + 127) / 128 * 128;
    MCK(cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, device));
    MCK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
    const int64_t I = m->I, H = m->H, O = m->O, Bp = m->Bp;
    const int64_t sizes[6] = {H * I, H, H * H, H, O * H, O};
    int64_t P = 0;
    for (int64_t s : sizes) P += s;
    m->P = P;
    m->theta = m->alloc<float>(P);
    m->grad = m->alloc<float>(P);
    m->m1 = m->alloc<float>(P);
    m->m2 = m->alloc<float>(P);
    int64_t off = 0;
    for (int l = 0; l < 3; ++l) {
      m->W[l] = m->theta + off;
      m->gW[l] = m->grad + off;
      off += sizes[2 * l];
      m->b[l] = m->theta + off;
      m->gb[l] = m->grad + off;
      off += sizes[2 * l + 1];
    }
    const int64_t rows[3] = {H, H, O}, cols[3] = {I, H, H};
    for (int l = 0; l < 3; ++l) {
      m->Wb[l] = m->alloc<bf16>(rows[l] * cols[l]);
      m->Wt[l] = m->alloc<bf16>(rows[l] * cols[l]);
    }
    m->x = m->alloc<bf16>(Bp * I);
    m->xt = m->alloc<bf16>(I * Bp);
    m->z1 = m->alloc<float>(Bp * H);
    m->h1 = m->alloc<bf16>(Bp * H);
    m->h1t = m->alloc<bf16>(H * Bp);
    m->z2 = m->alloc<float>(Bp * H);
    m->h2 = m->alloc<bf16>(Bp * H);
    m->h2t = m->alloc<bf16>(H * Bp);
    m->y = m->alloc<float>(Bp * O);
    m->dy = m->alloc<float>(Bp * O);
    m->dyb = m->alloc<bf16>(Bp * O);
    m->dyt = m->alloc<bf16>(O * Bp);
    m->dz2 = m->alloc<float>(Bp * H);
    m->dz2b = m->alloc<bf16>(Bp * H);
    m->dz2t = m->alloc<bf16>(H * Bp);
    m->dz1 = m->alloc<float>(Bp * H);
    m->dz1t = m->alloc<bf16>(H * Bp);
    m->loss_parts = pdot::ew_grid(Bp * O);
    m->loss_part = m->alloc<double>(m->loss_parts);
    m->loss = m->alloc<double>(1);
    m->err = m->alloc<int>(1);
    m->part = m->alloc<float>((size_t)m->sms * pdot::kBM * pdot::kBN);
    // initial weights and biases uniform in +-1/sqrt(fan_in)
    std::vector<float> h(P);
    uint64_t s = seed;
    const int64_t fan[6] = {I, I, H, H, H, H};
    off = 0;
    for (int k = 0; k < 6; ++k) {
      const double bound = 1.0 / std::sqrt((double)fan[k]);
      for (int64_t e = 0; e < sizes[k]; ++e) {
        const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
        h[off + e] = (float)((2.0 * u - 1.0) * bound);
      }
      off += sizes[k];
    }
    MCK(cudaMemcpyAsync(m->theta, h.data(), P * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    m->sync_bf16();
    // tensor maps: activations have Bp rows (products over the batch read the
    // transposed copies, Bp columns), weights their own shapes
    m->mx = make_map(m->x, Bp, I);
    m->mxt = make_map(m->xt, I, Bp);
    m->mh1 = make_map(m->h1, Bp, H);
    m->mh1t = make_map(m->h1t, H, Bp);
    m->mh2 = make_map(m->h2, Bp, H);
    m->mh2t = make_map(m->h2t, H, Bp);
    m->mdyb = make_map(m->dyb, Bp, O);
    m->mdyt = make_map(m->dyt, O, Bp);
    m->mdz2b = make_map(m->dz2b, Bp, H);
    m->mdz2t = make_map(m->dz2t, H, Bp);
    m->mdz1t = make_map(m->dz1t, H, Bp);
    for (int l = 0; l < 3; ++l) {
      m->mW[l] = make_map(m->Wb[l], rows[l], cols[l]);
      m->mWt[l] = make_map(m->Wt[l], cols[l], rows[l]);
    }
    MCK(cudaStreamSynchronize(m->stream));
    *out = m.release();
  });
}

extern "C" int pdot_mlp_destroy(pdot_mlp* m) {
  delete m;
  return PDOT_OK;
}

extern "C" int64_t pdot_mlp_num_parameters(const pdot_mlp* m) { return m ? m->P : 0; }

extern "C" void* pdot_mlp_stream(pdot_mlp* m) { return m ? (void*)m->stream : nullptr; }

extern "C" int pdot_mlp_get_parameters(pdot_mlp* m, float* host, int64_t count) {
  return mguarded([&] {
    if (!m || !host || count != m->P) mfail(PDOT_ERR_INVALID_ARGUMENT, "bad arguments");
    MCK(cudaSetDevice(m->device));
    MCK(cudaMemcpyAsync(host, m->theta, count * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
  });
}

extern "C" int pdot_mlp_set_parameters(pdot_mlp* m, const float* host, int64_t count) {
  return mguarded([&] {
    if (!m || !host || count != m->P) mfail(PDOT_ERR_INVALID_ARGUMENT, "bad arguments");
    MCK(cudaSetDevice(m->device));
    MCK(cudaMemcpyAsync(m->theta, host, count * sizeof(float), cudaMemcpyHostToDevice, m->stream));
    MCK(cudaMemsetAsync(m->m1, 0, count * sizeof(float), m->stream));
    MCK(cudaMemsetAsync(m->m2, 0, count * sizeof(float), m->stream));
    m->step = 0;
    m->sync_bf16();
    MCK(cudaStreamSynchronize(m->stream));
  });
}

extern "C" int pdot_mlp_get_gradients(pdot_mlp* m, float* host, int64_t count) {
  return mguarded([&] {
    if (!m || !host || count != m->P) mfail(PDOT_ERR_INVALID_ARGUMENT, "bad arguments");
    MCK(cudaSetDevice(m->device));
    MCK(cudaMemcpyAsync(host, m->grad, count * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
    MCK(cudaStreamSynchronize(m->stream));
  });
}

extern "C" int pdot_mlp_set_input(pdot_mlp* m, int64_t batch, const double* histograms, double shift, double scale) {
  return mguarded([&] {
    if (!m || !histograms) mfail(PDOT_ERR_INVALID_ARGUMENT, "bad arguments");
    if (batch < 1 || batch > m->Bp) mfail(PDOT_ERR_INVALID_ARGUMENT, "batch must be 1..%lld", (long long)m->Bp);
    MCK(cudaSetDevice(m->device));
    m->batch = batch;
    const int64_t bp = m->padded(batch);
    // rows past bp stay as they are: no product reads them
    pdot::k_features<<<pdot::ew_grid(bp * m->I), pdot::kEw, 0, m->stream>>>(histograms, batch, bp, m->I, shift, scale,
                                                                           m->x, m->xt, m->Bp);
    MCK(cudaGetLastError());
  });
}

extern "C" int pdot_mlp_forward(pdot_mlp* m, float* out) {
  return mguarded([&] {
    if (!m || m->batch < 1) mfail(PDOT_ERR_INVALID_ARGUMENT, "no input set");
    MCK(cudaSetDevice(m->device));
    m->forward();
    if (out)
      MCK(cudaMemcpyAsync(out, m->y, m->batch * m->O * sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
    m->check_err();
  });
}

extern "C" int pdot_mlp_backward(pdot_mlp* m, const float* target, double* loss) {
  return mguarded([&] {
    if (!m || !target || m->batch < 1) mfail(PDOT_ERR_INVALID_ARGUMENT, "bad arguments");
    MCK(cudaSetDevice(m->device));
    m->backward(target);
    if (loss) MCK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    m->check_err();
  });
}

extern "C" int pdot_mlp_adamw(pdot_mlp* m, float lr, float beta1, float beta2, float eps, float weight_decay) {
  return mguarded([&] {
    if (!m) mfail(PDOT_ERR_INVALID_ARGUMENT, "null network");
    MCK(cudaSetDevice(m->device));
    m->adamw(lr, beta1, beta2, eps, weight_decay);
  });
}

extern "C" int pdot_mlp_train_step(pdot_mlp* m, const float* target, float lr, float weight_decay, double* loss) {
  return mguarded([&] {
    if (!m || !target || m->batch < 1) mfail(PDOT_ERR_INVALID_ARGUMENT, "bad arguments");
    MCK(cudaSetDevice(m->device));
    m->forward();
    m->backward(target);
    m->adamw(lr, 0.9f, 0.999f, 1e-8f, weight_decay);
    if (loss) {
      MCK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
      m->check_err();
    }
  });
}
