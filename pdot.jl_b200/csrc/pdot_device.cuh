// pdot_device.cuh — device code shared by the solver kernels (pdot_kernels.cu)
// and the batched solver (pdot_batch.cu): reductions, vector loads, the cost
// sources, the per-entry primal update, the dual-step entry, the adaptive
// step-size rule and the evaluation / restart / termination control.
//
// Everything here has internal linkage: each translation unit gets its own copy.
#pragma once

#include <cfloat>
#include <cmath>
#include <cuda_bf16.h>
#include <utility>

#include "pdot_common.cuh"

namespace pdot {
namespace {

__device__ __forceinline__ double nanmax(double a, double b) { return (b > a || b != b) ? b : a; }

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Base.max(x, 0.0): NaN propagates, -0.0 becomes 0.0.
__device__ __forceinline__ double jl_max0(double x) { return x > 0.0 ? x : (x != x ? x : 0.0); }
// |min(x, 0.0)| with NaN propagating.
__device__ __forceinline__ double neg_part(double x) { return x < 0.0 ? -x : (x != x ? x : 0.0); }
// Base.min(x, y) for Float64.
__device__ __forceinline__ double jl_min(double x, double y) {
  if (x != x) return x;
  if (y != y) return y;
  return y < x ? y : x;
}
// x^y for the step-size rule; integral exponents 1 and 2 are exact as in Julia.
__device__ __forceinline__ double powd(double x, double y) {
  if (y == 1.0) return x;
  if (y == 2.0) return x * x;
  return pow(x, y);
}

// Deterministic block reduction of K values (bit k of maxmask: max, else sum),
// result written by thread 0 to out[0..K). Blocks have 256 threads.
template <int K>
__device__ __forceinline__ void block_reduce(double (&vals)[K], unsigned maxmask, double* out) {
  __shared__ double sh[kWarps][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = vals[k];
    const bool mx = (maxmask >> k) & 1u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double y = __shfl_xor_sync(0xffffffffu, x, o);
      x = mx ? nanmax(x, y) : x + y;
    }
    if (lane == 0) sh[warp][k] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const bool mx = (maxmask >> k) & 1u;
      double acc = sh[0][k];
      for (int w = 1; w < kWarps; ++w) acc = mx ? nanmax(acc, sh[w][k]) : acc + sh[w][k];
      out[k] = acc;
    }
  }
  __syncthreads();
}

// One warp reduces `count` records of K partials in a fixed order; lane 0 holds
// the result. Reads go through L2 (the partials were written by other CTAs).
// Lane l visits records l, l + 32, ... and takes all K values of a record at
// once, so the loads of a record are independent; each value's additions keep
// their order (record by record, then the shuffle tree).
template <int K>
__device__ __forceinline__ void warp_reduce_partials(const double* part, int64_t first, int64_t count,
                                                     unsigned maxmask, double (&out)[K]) {
  const int lane = threadIdx.x & 31;
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int64_t c = lane; c < count; c += 32) {
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = __ldcg(part + (first + c) * K + k);
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = ((maxmask >> k) & 1u) ? nanmax(acc[k], v[k]) : acc[k] + v[k];
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const bool mx = (maxmask >> k) & 1u;
    double a = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double y = __shfl_xor_sync(0xffffffffu, a, o);
      a = mx ? nanmax(a, y) : a + y;
    }
    out[k] = a;
  }
}

// sum_{c < count} q[c * stride], added in order c = 0, 1, ... The loads are
// issued eight at a time ahead of the (still sequential) additions: the second
// stage of a row sum of a small problem visits many CTA slots, and one
// dependent L2 round trip per slot made it a latency chain.
__device__ __forceinline__ double sum_strided(const double* q, int64_t count, int64_t stride) {
  double s = 0.0;
  int64_t c = 0;
  for (; c + 8 <= count; c += 8) {
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = q[(c + k) * stride];
#pragma unroll
    for (int k = 0; k < 8; ++k) s += v[k];
  }
  for (; c < count; ++c) s += q[c * stride];
  return s;
}

// Last-of-`count` election for a finish step: every CTA (or virtual block of
// a persistent launch) takes a ticket once; the one that takes the last sees
// the others' writes.
__device__ __forceinline__ bool elect_last_of(unsigned int* ticket, unsigned int count) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == count - 1);
  __syncthreads();
  if (last) __threadfence();
  return last;
}
__device__ __forceinline__ bool elect_last_cta(unsigned int* ticket) { return elect_last_of(ticket, gridDim.x); }

__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---- vector loads and stores of R consecutive rows (R*sizeof(T) bytes) -------
// Values stay in their storage type in registers and are widened to FP64 at use.
template <int BYTES>
struct VecWord;
template <>
struct VecWord<16> {
  using type = uint4;
};
template <>
struct VecWord<8> {
  using type = uint2;
};
template <>
struct VecWord<4> {
  using type = unsigned int;
};
template <>
struct VecWord<2> {
  using type = unsigned short;
};

template <typename T, int R>
__device__ __forceinline__ void vld(const T* p, T (&v)[R]) {
  if constexpr (R == 1) {
    v[0] = *p;
  } else if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < R / 2; ++h) {
      const double2 t = reinterpret_cast<const double2*>(p)[h];
      v[2 * h] = t.x;
      v[2 * h + 1] = t.y;
    }
  } else if constexpr (sizeof(T) == 4 && R == 4) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  } else {
    using W = typename VecWord<sizeof(T) * R>::type;
    const W w = *reinterpret_cast<const W*>(p);
    memcpy(v, &w, sizeof(W));
  }
}
template <typename T, int R>
__device__ __forceinline__ void vldg(const T* p, T (&v)[R]) {
  if constexpr (R == 1) {
    v[0] = __ldg(p);
  } else if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < R / 2; ++h) {
      const double2 t = __ldg(reinterpret_cast<const double2*>(p) + h);
      v[2 * h] = t.x;
      v[2 * h + 1] = t.y;
    }
  } else if constexpr (sizeof(T) == 4 && R == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  } else {
    using W = typename VecWord<sizeof(T) * R>::type;
    const W w = __ldg(reinterpret_cast<const W*>(p));
    memcpy(v, &w, sizeof(W));
  }
}
// The same through L2 only (ld.global.cg): for data that other CTAs of the
// same launch wrote (the persistent chunk kernel), where the read-only path
// of vldg is not coherent.
template <typename T, int R>
__device__ __forceinline__ void vldcg(const T* p, T (&v)[R]) {
  if constexpr (R == 1) {
    if constexpr (sizeof(T) == 2) {
      const unsigned short w = __ldcg(reinterpret_cast<const unsigned short*>(p));
      memcpy(v, &w, 2);
    } else {
      v[0] = __ldcg(p);
    }
  } else if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < R / 2; ++h) {
      const double2 t = __ldcg(reinterpret_cast<const double2*>(p) + h);
      v[2 * h] = t.x;
      v[2 * h + 1] = t.y;
    }
  } else if constexpr (sizeof(T) == 4 && R == 4) {
    const float4 t = __ldcg(reinterpret_cast<const float4*>(p));
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  } else {
    using W = typename VecWord<sizeof(T) * R>::type;
    const W w = __ldcg(reinterpret_cast<const W*>(p));
    memcpy(v, &w, sizeof(W));
  }
}
template <typename T, int R>
__device__ __forceinline__ void vst(T* p, const T (&v)[R]) {
  if constexpr (R == 1) {
    *p = v[0];
  } else if constexpr (sizeof(T) == 8) {
#pragma unroll
    for (int h = 0; h < R / 2; ++h) reinterpret_cast<double2*>(p)[h] = make_double2(v[2 * h], v[2 * h + 1]);
  } else if constexpr (sizeof(T) == 4 && R == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
    using W = typename VecWord<sizeof(T) * R>::type;
    W w;
    memcpy(&w, v, sizeof(W));
    *reinterpret_cast<W*>(p) = w;
  }
}

__device__ __forceinline__ double widen(double x) { return x; }
__device__ __forceinline__ double widen(float x) { return (double)x; }
__device__ __forceinline__ double widen(__nv_bfloat16 x) { return (double)__bfloat162float(x); }

// Round an FP64 value to the plan's storage type.
template <typename TX>
__device__ __forceinline__ TX narrow(double x);
template <>
__device__ __forceinline__ double narrow<double>(double x) {
  return x;
}
template <>
__device__ __forceinline__ float narrow<float>(double x) {
  return __double2float_rn(x);
}

// ---- cost sources ------------------------------------------------------------
// panel(): once per panel (per-lane row data); column(): once per column
// (warp-uniform data); get(): the R cost entries of lane rows k at index idx,
// in the source's value type (value_t).
//
// C_ij = scale * ||x_i - y_j||^2 (squared-Euclidean kinds) or
// scale * ||x_i - y_j||_1 (L1 kinds) in FP32 from DIM-dimensional coordinates;
// nothing of C is read from memory.
template <int CK, int R, int RPL>
struct CostReader {
  static constexpr bool kL1 = is_l1_cost(CK);
  static constexpr int DIM = CK - (kL1 ? kCostL1Base : kCostSqBase);
  static_assert(is_point_cost(CK) && DIM >= 1 && DIM <= kMaxPointDim, "coordinate cost kinds only");
  using value_t = float;
  const float* __restrict__ xs;
  const float* __restrict__ ys;
  float scale;
  float xr[RPL][R][DIM];
  float yr[DIM];
  float yn[DIM];  // the next column's coordinates, loaded one unit ahead
  __device__ __forceinline__ CostReader(const CostSource& s, float scl) : xs(s.xs), ys(s.ys), scale(scl) {}
  __device__ __forceinline__ void panel(int64_t row0, int lane, int64_t m, const bool (&ok)[RPL]) {
#pragma unroll
    for (int k = 0; k < RPL; ++k)
#pragma unroll
      for (int e = 0; e < R; ++e) {
        const int64_t i = row0 + k * 32 * R + lane * R + e;
#pragma unroll
        for (int d = 0; d < DIM; ++d) xr[k][e][d] = (ok[k] && i < m) ? __ldg(xs + i * DIM + d) : 0.0f;
      }
  }
  __device__ __forceinline__ void column(int64_t j) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) yr[d] = __ldg(ys + j * DIM + d);
  }
  // prefetch(j) starts the loads of column j's coordinates; take() makes them
  // the current column. The batched staged pass prefetches its next unit's
  // column while it computes the current one, so the loads' latency is off the
  // unit's path (the batched solve measured 1.05 -> 0.95 s on B200; the single
  // instance's staged pass measured slower with it and loads in place).
  __device__ __forceinline__ void prefetch(int64_t j) {
#pragma unroll
    for (int d = 0; d < DIM; ++d) yn[d] = __ldg(ys + j * DIM + d);
  }
  __device__ __forceinline__ void take() {
#pragma unroll
    for (int d = 0; d < DIM; ++d) yr[d] = yn[d];
  }
  __device__ __forceinline__ void get(int64_t, int k, float (&c)[R]) const {
#pragma unroll
    for (int e = 0; e < R; ++e) {
      float acc = 0.0f;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const float t = xr[k][e][d] - yr[d];
        acc = kL1 ? acc + fabsf(t) : __fmaf_rn(t, t, acc);  // coordinate costs serve FP32 plans only
      }
      c[e] = acc * scale;
    }
  }
};

template <typename T, int R, int RPL>
struct StoredCost {
  using value_t = T;
  const T* __restrict__ C;
  __device__ __forceinline__ StoredCost(const CostSource& s, float) : C(static_cast<const T*>(s.C)) {}
  __device__ __forceinline__ void panel(int64_t, int, int64_t, const bool (&)[RPL]) {}
  __device__ __forceinline__ void column(int64_t) {}
  __device__ __forceinline__ void prefetch(int64_t) {}
  __device__ __forceinline__ void take() {}
  __device__ __forceinline__ void get(int64_t idx, int, T (&c)[R]) const { vldg<T, R>(C + idx, c); }
};
template <int R, int RPL>
struct CostReader<PDOT_COST_F64, R, RPL> : StoredCost<double, R, RPL> {
  using StoredCost<double, R, RPL>::StoredCost;
};
template <int R, int RPL>
struct CostReader<PDOT_COST_F32, R, RPL> : StoredCost<float, R, RPL> {
  using StoredCost<float, R, RPL>::StoredCost;
};
template <int R, int RPL>
struct CostReader<PDOT_COST_BF16, R, RPL> : StoredCost<__nv_bfloat16, R, RPL> {
  using StoredCost<__nv_bfloat16, R, RPL>::StoredCost;
};

// One entry of the primal pass (see the fused pass below).
//
// FP64 plan (the drop-in): the reference's statement order with explicit
// round-to-nearest FP64 operations, bit for bit as the oracle computes it.
//
// FP32 plan (mixed precision): the entry's arithmetic runs in FP32, the
// plan's own precision (the cost entry is FP32 or BF16 storage or computed in
// FP32; the duals and step weights are rounded to FP32 once), with fused
// multiply-adds where the drop-in rounds twice. The step d between the two
// stored values is formed exactly in FP64, so the FP64 row, column and
// squared-norm sums the caller accumulates add exactly what was stored.
__device__ __forceinline__ float jl_max0f(float x) { return x > 0.0f ? x : (x != x ? x : 0.0f); }

// The sum of squared steps: the FP64 plan rounds the product and the sum as
// the reference does; an FP32 plan's sum takes one fused multiply-add.
template <typename TX>
__device__ __forceinline__ void add_sq(double& sq, double d) {
  if constexpr (sizeof(TX) == 8)
    sq += d * d;
  else
    sq = __fma_rn(d, d, sq);
}

template <typename TX>
__device__ __forceinline__ void primal_entry(double c, double ui, double vj, double s, double nw, double aw,
                                             bool zero_g, bool first, TX& xs, TX& xas, double& d) {
  if constexpr (sizeof(TX) == 8) {
    const double x = xs;
    const double gg = zero_g ? 0.0 : __dsub_rn(__dsub_rn(c, ui), vj);
    const double t = jl_max0(__dsub_rn(x, __dmul_rn(s, gg)));
    d = __dsub_rn(t, x);
    const double xn = __dadd_rn(x, d);
    xs = xn;
    xas = first ? xn : __dmul_rn(__dadd_rn(xas, __dmul_rn(xn, nw)), aw);
  } else {
    const float x = xs;
    const float gg = zero_g ? 0.0f : __fsub_rn(__fsub_rn((float)c, (float)ui), (float)vj);
    const float t = jl_max0f(__fmaf_rn(-(float)s, gg, x));
    d = __dsub_rn((double)t, (double)x);
    xs = t;
    xas = first ? t : __fmul_rn(__fmaf_rn(t, (float)nw, xas), (float)aw);
  }
}

constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase `parity` of an mbarrier: at most `polls` polls and at
// most about kWaitLimitNs of device time (each try_wait may suspend the
// thread for a while, so the poll count alone does not bound the time).
constexpr unsigned long long kWaitLimitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, int polls = kSpinLimit) {
  unsigned long long t0 = 0;
  for (int it = 0; it < polls; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 1023) == 1023) {
      const unsigned long long t = globaltimer_ns();
      if (t0 == 0)
        t0 = t;
      else if (t - t0 > kWaitLimitNs)
        return false;
    }
  }
  return false;
}

// Programmatic dependent launch. The kernels of the iteration loop are
// launched with programmatic stream serialization (pdl_launch): the next
// kernel in the stream may be scheduled before this one ends, and its CTAs
// then block in griddepcontrol.wait until this grid has completed and its
// writes are visible. Every such kernel calls pdl_wait() before it touches
// global memory (reads of the previous kernel's results and writes of the
// buffers it reads alike), then pdl_trigger() so that the kernel after it may
// be scheduled while it runs. Both are no-ops in a kernel launched without
// the attribute. The time saved is the launch and ramp of each kernel, which
// is most of an iteration's time on small problems.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_enter() {
  pdl_wait();
  pdl_trigger();
}

// Build knob: PDOT_PDL 0 launches the loop's kernels without the attribute.
#ifndef PDOT_PDL
#define PDOT_PDL 1
#endif
template <typename... P, typename... A>
inline cudaError_t pdl_launch(void (*kfn)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              A&&... args) {
  cudaLaunchConfig_t c = {};
  c.gridDim = grid;
  c.blockDim = block;
  c.dynamicSmemBytes = smem;
  c.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  c.attrs = at;
  c.numAttrs = PDOT_PDL ? 1 : 0;
  return cudaLaunchKernelEx(&c, kfn, std::forward<A>(args)...);
}

// Grid-wide barrier of a persistent launch whose CTAs are all co-resident (a
// cooperative launch). Thread 0 of each CTA reads the generation, publishes
// its CTA's writes (fence) and arrives; the last arrival resets the count and
// releases the next generation, the others poll it with acquire loads, at most
// `polls` times, and stop early once `abort_flag` is non-zero (another CTA's
// poll ran out). Returns false to every thread of the CTA when its poll ran
// out or was aborted (the caller records the error and leaves), so after one
// timeout every CTA leaves within one more barrier.
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int* gen, unsigned int ctas,
                                             const int* abort_flag, int polls = kSpinLimit) {
  __shared__ int bar_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned int g0 = ld_acquire_gpu(gen);
    __threadfence();
    if (atomicAdd(count, 1u) == ctas - 1) {
      atomicExch(count, 0u);
      st_release_gpu(gen, g0 + 1u);
    } else {
      int it = 0;
      while (ld_acquire_gpu(gen) == g0) {
        if (++it >= polls || ld_acquire_gpu(reinterpret_cast<const unsigned int*>(abort_flag)) != 0u) {
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    bar_ok = ok;
  }
  __syncthreads();
  return bar_ok != 0;
}

// The units of warp w inside [q0, q1): column w, w+8, ... of each panel segment.
struct UnitCursor {
  int64_t p, j, je, q1, n;
  bool valid;
  __device__ __forceinline__ void init(int64_t q0, int64_t q1_, int64_t n_, int w) {
    q1 = q1_;
    n = n_;
    p = q0 / n;
    const int64_t jb = (q0 > p * n ? q0 : p * n) - p * n;
    je = (q1 < (p + 1) * n ? q1 : (p + 1) * n) - p * n;
    j = jb + w;
    valid = true;
    normalize(w);
  }
  __device__ __forceinline__ void normalize(int w) {
    while (j >= je) {
      ++p;
      if (p * n >= q1) {
        valid = false;
        return;
      }
      je = (q1 < (p + 1) * n ? q1 : (p + 1) * n) - p * n;
      j = w;
    }
  }
  __device__ __forceinline__ void advance(int w) {
    j += kWarps;
    normalize(w);
  }
};


// ---------------------------------------------------------------------------
// Adaptive step-size rule and the state update on acceptance,
// src/solver_gpu.jl:290-367 (take_step!) and :370-410 (constant step).
// The retried candidate of a rejected attempt is identical to the first one
// (the kernels use solver_state.step_size, not the shrunk local step), so the
// candidate computed once is the accepted one; a rejection only adds an
// attempt to the counters and one more application of the shrink rule.
// First-attempt powers of the step-size rule, computed by a spare warp while
// the finishing CTA's other warps reduce the partial sums: (k + 1)^e for the
// iteration count k that the first attempt sees.
struct StepPowers {
  double k1 = -1.0, reduction = 0.0, growth = 0.0;
};
__device__ __forceinline__ StepPowers step_powers(const DevState* st, const SolveConfig& cfg) {
  StepPowers p;
  p.k1 = (double)(st->total_iters + 2);
  p.reduction = powd(p.k1, cfg.reduction_exponent);
  p.growth = powd(p.k1, cfg.growth_exponent);
  return p;
}

__device__ void step_control(DevState* st, const SolveConfig& cfg, double dot_r, double dot_c, double dx2,
                             double dy2, const StepPowers& pre = StepPowers()) {
  const double omega = st->primal_weight;
  const double weight = st->step_size;
  const bool fresh = !(st->sum_weights > 0.0);
  bool accepted = true;
  if (cfg.adaptive) {
    const double interaction = fabs(dot_r + dot_c);
    const double ndp = sqrt(dx2), ndd = sqrt(dy2);
    const double movement = __dadd_rn(__dmul_rn(__dmul_rn(0.5, omega), __dmul_rn(ndp, ndp)),
                                      __dmul_rn(__ddiv_rn(0.5, omega), __dmul_rn(ndd, ndd)));
    double tau = st->step_size;
    accepted = false;
    for (int attempt = 0; attempt < 64; ++attempt) {
      st->total_iters += 1;
      st->kkt_passes += 1.0;
      double limit;
      if (interaction > 0.0) {
        limit = __ddiv_rn(movement, interaction);
        if (movement == 0.0) {
          st->numerical_error = 1;
          break;
        }
      } else {
        limit = INFINITY;
      }
      if (tau <= limit) accepted = true;
      const double k1 = (double)(st->total_iters + 1);
      const bool have = k1 == pre.k1;
      const double pr = have ? pre.reduction : powd(k1, cfg.reduction_exponent);
      const double pg = have ? pre.growth : powd(k1, cfg.growth_exponent);
      const double first_term = __dmul_rn(__dsub_rn(1.0, __ddiv_rn(1.0, pr)), limit);
      const double second_term = __dmul_rn(__dadd_rn(1.0, __ddiv_rn(1.0, pg)), tau);
      tau = jl_min(first_term, second_term);
      if (accepted) break;
      // the reference loops forever on a NaN limit; stop with a numerical error
      if (tau != tau) {
        st->numerical_error = 1;
        break;
      }
    }
    if (!accepted) st->numerical_error = 1;
    st->step_size = tau;
  } else {
    st->kkt_passes += 1.0;
  }
  if (accepted) {
    st->sum_weights = st->sum_weights + weight;
    st->avg_count += 1;
    st->g_is_zero = 0;
  }
  st->primal_passes += 1;
  st->fresh_passes += fresh ? 1 : 0;
  st->iteration += 1;
}

struct DualArgs {
  double tw, nw, aw;
  bool first;
};

// Dual step of one entry, src/solver_gpu.jl:172-173,191,272-279 and the
// vector averages src/saddle_point_gpu.jl:140-221.
__device__ __forceinline__ void dual_entry(double sum_delta, double dist, double* r, double* u, double* ravg,
                                           double* uavg, const DualArgs& A, double& dot, double& dy2) {
  const double rr = *r;
  const double rn = __dadd_rn(sum_delta, rr);
  const double dr = __dsub_rn(rn, rr);
  const double uu = *u;
  const double un = __dadd_rn(uu, __dmul_rn(A.tw, __dadd_rn(__dsub_rn(dist, __dmul_rn(2.0, rn)), rr)));
  const double du = __dsub_rn(un, uu);
  dot += dr * du;
  dy2 += du * du;
  *r = rn;
  *u = un;
  *ravg = A.first ? rn : __dmul_rn(__dadd_rn(*ravg, __dmul_rn(rn, A.nw)), A.aw);
  *uavg = A.first ? un : __dmul_rn(__dadd_rn(*uavg, __dmul_rn(un, A.nw)), A.aw);
}


enum { E_DOT = 0, E_SQX, E_MAXX, E_SQG, E_MAXG, E_AVG = 5 };
constexpr unsigned kEvalMaxMask = (1u << E_MAXX) | (1u << E_MAXG) | (1u << (E_AVG + E_MAXX)) |
                                  (1u << (E_AVG + E_MAXG));


// Evaluation, vector part: per point, ||dist - sums||^2, max|dist - sums|,
// <dist, dual>, ||dual||^2, max|dual| (src/utils_gpu.jl:26-27,54,94-95,115-116).
enum { V_SQRES = 0, V_MAXRES, V_DOT, V_SQDUAL, V_MAXDUAL, V_AVG = 5 };
constexpr unsigned kVecMaxMask = (1u << V_MAXRES) | (1u << V_MAXDUAL) | (1u << (V_AVG + V_MAXRES)) |
                                 (1u << (V_AVG + V_MAXDUAL));

struct PointSums {
  double pobj, sq_x, max_x, sq_g, max_g;
  double sq_src, max_src, dot_src, sq_u, max_u;
  double sq_tgt, max_tgt, dot_tgt, sq_v, max_v;
};

__device__ __forceinline__ PointSums point_sums(const double* E, const double* R, const double* Cc, int off) {
  PointSums P;
  P.pobj = E[off + E_DOT];
  P.sq_x = E[off + E_SQX];
  P.max_x = E[off + E_MAXX];
  P.sq_g = E[off + E_SQG];
  P.max_g = E[off + E_MAXG];
  P.sq_src = R[off + V_SQRES];
  P.max_src = R[off + V_MAXRES];
  P.dot_src = R[off + V_DOT];
  P.sq_u = R[off + V_SQDUAL];
  P.max_u = R[off + V_MAXDUAL];
  P.sq_tgt = Cc[off + V_SQRES];
  P.max_tgt = Cc[off + V_MAXRES];
  P.dot_tgt = Cc[off + V_DOT];
  P.sq_v = Cc[off + V_SQDUAL];
  P.max_v = Cc[off + V_MAXDUAL];
  return P;
}

// compute_weight_kkt_residual, src/saddle_point_gpu.jl:299-330
__device__ __forceinline__ double weighted_kkt(double l2_pres, double l2_dres, double gap, double omega) {
  return sqrt(omega * (l2_pres * l2_pres) + (1.0 / omega) * (l2_dres * l2_dres) + gap * gap);
}

// src/termination.jl:106-134
__device__ bool optimality_met(const SolveConfig& cfg, const DevState* st,
                               const pdot_convergence_information& ci) {
  const double abs_obj = fabs(ci.primal_objective) + fabs(ci.dual_objective);
  const double gap = fabs(ci.primal_objective - ci.dual_objective);
  double perr, pbase, derr, dbase;
  if (cfg.optimality_norm == PDOT_L_INF) {
    perr = ci.l_inf_primal_residual;
    pbase = st->linf_rhs;
    derr = ci.l_inf_dual_residual;
    dbase = st->linf_obj;
  } else {
    perr = ci.l2_primal_residual;
    pbase = st->l2_rhs;
    derr = ci.l2_dual_residual;
    dbase = st->l2_obj;
  }
  return derr < cfg.eps_abs + cfg.eps_rel * dbase && perr < cfg.eps_abs + cfg.eps_rel * pbase &&
         gap < cfg.eps_abs + cfg.eps_rel * abs_obj;
}

// A warm start's last-restart record. The reference's restart information
// starts at the initial point (create_last_restart_info,
// src/saddle_point_gpu.jl:371-393: copies of the initial plan, duals, sums and
// stored gradient), so a solve started from (X0, u0, v0) keeps that point:
// its l2 primal residual ||[a - X0 1; b - X0^T 1]||, its l2 dual residual
// ||min(C - u0 - v0, 0)|| (the stored gradient is C - u0 - v0 from the start),
// its gap and the norms ||X0||, ||[u0; v0]|| that the first restart measures
// the distance from (Q3). `P` holds the start point's evaluation sums.
__device__ __forceinline__ void record_start_point(DevState* st, const PointSums& P) {
  st->last_rp = sqrt(P.sq_src + P.sq_tgt);
  st->last_rd = sqrt(P.sq_g);
  st->last_gap = fabs(P.pobj - (P.dot_src + P.dot_tgt));
  st->last_xnorm = sqrt(P.sq_x);
  st->last_ynorm = sqrt(P.sq_u + P.sq_v);
}

// The evaluation block of optimize(), src/solver_gpu.jl:529-696, with
// compute_convergence_information (src/utils_gpu.jl:68-129),
// check_termination_criteria (src/termination.jl:140-166), run_restart_scheme
// (src/saddle_point_gpu.jl:539-696) and compute_new_primal_weight (:701-728).
__device__ void eval_control(DevState* st, const SolveConfig& cfg, const PointSums& cur, const PointSums& avg,
                             pdot_iteration_stats* ring, int ring_cap) {
  const long long it = st->iteration;
  st->kkt_passes += 2.0;
  const bool have_avg = st->avg_count > 0;
  const bool use_cur = st->numerical_error || !have_avg;
  const PointSums& P = use_cur ? cur : avg;
  const double eps_ratio = cfg.eps_abs / cfg.eps_rel;
  const unsigned long long now = globaltimer_ns();

  pdot_iteration_stats rec;
  memset(&rec, 0, sizeof(rec));
  pdot_convergence_information& ci = rec.convergence_information;
  ci.candidate_type = PDOT_POINT_TYPE_AVERAGE_ITERATE;
  ci.primal_objective = P.pobj;
  ci.l_inf_primal_residual = nanmax(P.max_src, P.max_tgt);
  ci.l2_primal_residual = sqrt(P.sq_src + P.sq_tgt);
  ci.relative_l_inf_primal_residual = ci.l_inf_primal_residual / (eps_ratio + st->linf_rhs);
  ci.relative_l2_primal_residual = ci.l2_primal_residual / (eps_ratio + st->l2_rhs);
  ci.l_inf_primal_variable = P.max_x;
  ci.l2_primal_variable = sqrt(P.sq_x);
  ci.dual_objective = P.dot_src + P.dot_tgt;
  ci.l_inf_dual_residual = P.max_g;
  ci.l2_dual_residual = sqrt(P.sq_g);
  ci.relative_l_inf_dual_residual = ci.l_inf_dual_residual / (eps_ratio + st->linf_obj);
  ci.relative_l2_dual_residual = ci.l2_dual_residual / (eps_ratio + st->l2_obj);
  // src/utils_gpu.jl:115-116 measure [u; u] (the source duals twice)
  ci.l_inf_dual_variable = P.max_u;
  ci.l2_dual_variable = sqrt(P.sq_u + P.sq_u);
  ci.corrected_dual_objective = ci.l_inf_dual_residual == 0.0 ? ci.dual_objective : -INFINITY;
  {
    const double gap = fabs(ci.primal_objective - ci.dual_objective);
    const double abs_obj = fabs(ci.primal_objective) + fabs(ci.dual_objective);
    ci.relative_optimality_gap = gap / (eps_ratio + abs_obj);
  }
  rec.iteration_number = (int32_t)it;
  rec.cumulative_kkt_matrix_passes = st->kkt_passes;
  rec.cumulative_rejected_steps = 0;
  rec.cumulative_time_sec = (double)(now - st->t_start_ns) * 1e-9;
  rec.restart_used = PDOT_RESTART_CHOICE_UNSPECIFIED;
  rec.step_size = st->step_size;
  rec.primal_weight = st->primal_weight;
  rec.time_spent_doing_basic_algorithm = rec.cumulative_time_sec - st->eval_time_sec;

  const double omega = st->primal_weight, tau = st->step_size;
  const double pnp = 1.0 / tau * omega, dnp = 1.0 / tau / omega;  // define_norms

  int term = 0;
  if (optimality_met(cfg, st, ci))
    term = PDOT_TERMINATION_REASON_OPTIMAL;
  else if (it >= cfg.iteration_limit)
    term = PDOT_TERMINATION_REASON_ITERATION_LIMIT;
  else if (rec.cumulative_kkt_matrix_passes >= cfg.kkt_matrix_pass_limit)
    term = PDOT_TERMINATION_REASON_KKT_MATRIX_PASS_LIMIT;
  else if (rec.cumulative_time_sec >= cfg.time_sec_limit)
    term = PDOT_TERMINATION_REASON_TIME_LIMIT;
  // Non-finite objectives can never meet the optimality test; the reference
  // would iterate to the iteration limit. Stop with a numerical error.
  if (!term && !(isfinite(ci.primal_objective) && isfinite(ci.dual_objective)))
    term = PDOT_TERMINATION_REASON_NUMERICAL_ERROR;
  if (st->numerical_error && !term) term = PDOT_TERMINATION_REASON_NUMERICAL_ERROR;

  if (!term) {
    int choice = PDOT_RESTART_CHOICE_NO_RESTART;
    if (have_avg) {
      const long long len = st->avg_count;
      bool do_restart = (double)len >= cfg.artificial_restart_threshold * (double)(it - 1);
      bool to_avg = false;
      double cand = 0.0;
      const double rp_c = sqrt(cur.sq_src + cur.sq_tgt), rd_c = sqrt(cur.sq_g);
      const double gap_c = fabs(cur.pobj - (cur.dot_src + cur.dot_tgt));
      const double rp_a = sqrt(avg.sq_src + avg.sq_tgt), rd_a = sqrt(avg.sq_g);
      const double gap_a = fabs(avg.pobj - (avg.dot_src + avg.dot_tgt));
      if (cfg.restart_scheme != PDOT_NO_RESTARTS) {
        const double kc = weighted_kkt(rp_c, rd_c, gap_c, omega);
        const double ka = weighted_kkt(rp_a, rd_a, gap_a, omega);
        to_avg = cfg.restart_to_current_metric == PDOT_KKT_GREEDY ? (kc >= ka) : true;
        cand = to_avg ? ka : kc;
      }
      if (!do_restart) {
        if (cfg.restart_scheme == PDOT_ADAPTIVE_KKT) {
          const double kl = weighted_kkt(st->last_rp, st->last_rd, st->last_gap, omega);
          const double ratio = cand / kl;
          if (ratio < cfg.necessary_reduction_for_restart) {
            if (ratio < cfg.sufficient_reduction_for_restart)
              do_restart = true;
            else if (ratio > st->ratio_last_trial)
              do_restart = true;
          }
          st->ratio_last_trial = ratio;
        } else if (cfg.restart_scheme == PDOT_FIXED_FREQUENCY && cfg.restart_frequency_if_fixed <= len) {
          do_restart = true;
        }
      }
      if (do_restart) {
        const PointSums& R = to_avg ? avg : cur;
        // update_last_restart_info! measures from the previous restart point
        // to the (already reset, zero) average: the norms of the previous point.
        st->pdist = (sqrt(pnp) * st->last_xnorm) / sqrt(omega);
        st->ddist = (sqrt(dnp) * st->last_ynorm) * sqrt(omega);
        st->last_xnorm = sqrt(R.sq_x);
        st->last_ynorm = sqrt(R.sq_u + R.sq_v);
        st->last_rp = to_avg ? rp_a : rp_c;
        st->last_rd = to_avg ? rd_a : rd_c;
        st->last_gap = to_avg ? gap_a : gap_c;
        st->last_restart_length = len;
        if (to_avg) st->buf ^= 1;
        st->sum_weights = 0.0;
        st->avg_count = 0;
        choice = to_avg ? PDOT_RESTART_CHOICE_RESTART_TO_AVERAGE : PDOT_RESTART_CHOICE_WEIGHTED_AVERAGE_RESET;
        if (st->pdist > DBL_EPSILON && st->ddist > DBL_EPSILON) {
          const double sm = cfg.primal_weight_update_smoothing;
          const double est = st->ddist / st->pdist;
          st->primal_weight = exp(sm * log(est) + (1.0 - sm) * log(omega));
        }
      }
    }
    rec.restart_used = choice;
    st->last_restart_choice = choice;
  } else {
    st->done = 1;
    st->termination_reason = term;
    st->out_current = have_avg ? 0 : 1;
  }
  if (cfg.record_iteration_stats || term) {
    ring[st->num_stats % ring_cap] = rec;
    st->num_stats += 1;
  }
  st->eval_time_sec += (double)(globaltimer_ns() - st->eval_t0_ns) * 1e-9;
}


}  // namespace
}  // namespace pdot
