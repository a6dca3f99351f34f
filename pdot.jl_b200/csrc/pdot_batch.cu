// pdot_batch.cu — many independent OT instances of uneven sizes solved at once.
//
// Every instance runs the reference's full loop (src/solver_gpu.jl:413-720)
// with its own step size, primal weight, averages, restart record and
// termination; the instances advance in lockstep (one global iteration runs
// one loop body of every active instance), so they share the evaluation
// schedule. Plans are FP32 (the mixed-precision arithmetic of pdot_kernels.cu),
// duals and control FP64; the cost is stored FP32 or computed from FP32
// coordinates (squared-Euclidean or L1).
//
// Work decomposition: the units (one column of one panel of 256 or 128 rows,
// the batch's tile shape) of all active instances are concatenated into one
// line and cut into contiguous CTA ranges of equal cost, a unit costing its
// rows plus a fixed per-unit overhead (the autotuner picks the tile and the
// overhead). The units of uneven instances carry from 1 to the panel's rows,
// so ranges of equal unit count would leave some CTAs with several times the
// bytes of others. kb_compact recomputes the ranges (cta_begin) whenever the
// active list changes. Row
// partials live in slot (cta + global panel), column partials at the global
// unit index, per-instance sums of squares and evaluation partials in slot
// (cta + active index): along the line the owning CTA, the global panel and
// the active index never decrease and one of them grows at every boundary, so
// each slot is written by one (CTA, segment) pair. After every evaluation a
// single CTA rebuilds the list of active instances and its prefix sums, so
// finished instances cost nothing and the captured CUDA graph stays valid.
//
// Each instance's plan is stored column-major with its row count padded to a
// multiple of 8 (32 bytes: every column starts on a DRAM sector, so no sector is
// read by the copies of two columns; with a multiple of 4 the reads were 1.13x
// the algorithmic bytes); padded rows hold zeros and are masked.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pdot_device.cuh"

namespace pdot {
namespace {

constexpr int kBR = 4;                       // FP32 rows per lane load
constexpr int kMaxBatch = 1 << 16;
constexpr int kJU = 2;  // columns per warp step of the batched primal pass

// Tile shapes of the matrix passes: a unit is one column of one panel of PR
// rows (256 or 128; the host picks one per batch, the autotuner between them).
// A lane loads kBR rows PR / 128 times per unit, so a 128-row tile holds half
// the per-row registers (row sums, row duals, source coordinates) and its
// primal passes are compiled for three resident CTAs per SM instead of two,
// with a ring of half the bytes in the staged form. The per-unit overhead of
// the CTA split stays counted in 256-row units (kUnitCostRows).
template <int PR>
struct Tile {
  static_assert(PR == 128 || PR == 256, "panels of 128 or 256 rows");
  static constexpr int RPL = PR / (32 * kBR);                    // loads per lane per unit
  static constexpr int kMinBlocks = PR == 256 ? 2 : 3;           // resident CTAs per SM of the primal passes
  static constexpr int kRingBudget = PR == 256 ? 96 * 1024 : 48 * 1024;  // staged ring bytes per CTA
};
constexpr int kUnitCostRows = 256;

struct BatchInstance {
  int64_t m, n, ld;  // rows, columns, padded leading dimension
  int64_t x_off;     // offset of the plan / stored cost (elements)
  int64_t row_off;   // offset of the row vectors (m entries)
  int64_t col_off;   // offset of the column vectors (n entries)
  int64_t pts_off;   // offset of the points (rows; times dim for elements)
  int64_t tpts_off;  // offset of the target points (rows)
  int64_t panels;    // ceil(m / panel rows)
  int64_t rblocks, cblocks;  // vector blocks over rows and columns
};

struct BatchActive {
  int count;
  int any_empty;          // some CTA range holds no unit (only in the tail of a solve)
  long long total_units;
  int error;              // a bounded wait gave up: every later launch returns at once
  unsigned int bar_count; // grid barrier of the persistent chunk: arrivals
  unsigned int bar_gen;   // and generation
  int pad_;
};

struct BatchBuffers {
  const BatchInstance* inst;
  int num;                 // instances
  int dim;                 // point dimension
  const float* C;          // stored FP32 costs (per instance at x_off, ld)
  const float* xs;         // source points (per instance at pts_off * dim)
  const float* ys;         // target points
  const double* a;         // marginals at row_off / col_off
  const double* b;
  float* X[2];
  double* u[2];
  double* v[2];
  double* r[2];
  double* c[2];
  double* rowpart;         // (grid + total panels) * panel rows
  double* colpart;         // total units
  double* sqpart;          // grid + num
  double* steppart;        // total vector blocks * kStepSums
  double* evpart;          // (grid + num) * kEvalSums
  double* vecpart;         // total vector blocks * kVecSums
  const int* warm;         // per instance: 1 when it starts from a warm start
  const double* warm_omega;// per instance: initial primal weight of a warm start (> 0), or null
  const int* race;         // per instance: race group (-1: none), or null
  int* winner;             // per group: lowest index of an optimal member (INT_MAX-like when none)
  DevState* st;            // per instance
  pdot_iteration_stats* rec;  // per instance: the latest evaluation record
  BatchActive* act;
  int* ids;                // active instance ids
  long long* unit_prefix;  // active prefix of units (count + 1)
  long long* panel_prefix; // active prefix of panels
  long long* vblock_prefix;// active prefix of vector blocks
  long long* cost_prefix;  // active prefix of the units' balancing cost (count + 1)
  long long* cta_begin;    // grid + 1: CTA c owns the active units [cta_begin[c], cta_begin[c + 1])
  int unit_cost;           // per-unit overhead of the balancing cost, in eighths of 256 rows
};

// The CTA that owns active unit q: the largest c with cta_begin[c] <= q (an
// empty range c has cta_begin[c] == cta_begin[c + 1], so the search passes it).
__device__ __forceinline__ long long bcta_of_unit(const long long* cta_begin, int grid, long long q) {
  int lo = 0, hi = grid - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cta_begin[mid] <= q)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}
// Loads of data that another CTA may have written earlier in the same launch
// (CO: the persistent chunk, where the dual step, the compaction and the
// primal pass are phases of one launch) go through L2 (ld.global.cg); the
// per-launch kernels read them through the read-only path.
template <bool CO, typename T>
__device__ __forceinline__ T ldro(const T* p) {
  if constexpr (CO)
    return __ldcg(p);
  else
    return __ldg(p);
}
template <bool CO, typename T, int R>
__device__ __forceinline__ void vldro(const T* p, T (&v)[R]) {
  if constexpr (CO)
    vldcg<T, R>(p, v);
  else
    vldg<T, R>(p, v);
}
// the plan, which the pass also writes: a plain load, or through L2
template <bool CO, typename T, int R>
__device__ __forceinline__ void vldx(const T* p, T (&v)[R]) {
  if constexpr (CO)
    vldcg<T, R>(p, v);
  else
    vld<T, R>(p, v);
}

// largest k in [0, count) with prefix[k] <= q
template <bool CO = false>
__device__ __forceinline__ int find_segment(const long long* prefix, int count, long long q) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (ldro<CO>(prefix + mid) <= q)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}


// A lane's per-load partial sums added in load order.
template <int N>
__device__ __forceinline__ double lane_sum(const double (&x)[N]) {
  double t = x[0];
#pragma unroll
  for (int kq = 1; kq < N; ++kq) t += x[kq];
  return t;
}

// Fixed-order sum of the non-empty CTA slots [lo, hi] (+ offset) of K values.
template <int K>
__device__ __forceinline__ void sum_cta_slots(const double* part, const long long* cta_begin, long long lo,
                                              long long hi, long long slot_off, unsigned maxmask,
                                              double (&out)[K]) {
  const int lane = threadIdx.x & 31;
  // all K values of a slot at once (independent loads); each value's
  // additions keep their order
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (long long c = lo + lane; c <= hi; c += 32) {
    if (cta_begin[c] == cta_begin[c + 1]) continue;  // empty CTA
    double v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = __ldcg(part + (c + slot_off) * K + k);
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = ((maxmask >> k) & 1u) ? nanmax(acc[k], v[k]) : acc[k] + v[k];
  }
#pragma unroll
  for (int k = 0; k < K; ++k) {
    const bool mx = (maxmask >> k) & 1u;
    double a = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_xor_sync(0xffffffffu, a, o);
      a = mx ? nanmax(a, y) : a + y;
    }
    out[k] = a;
  }
}

// ---------------------------------------------------------------------------
// Batched fused primal pass (FP32 plan): the per-entry step of pdot_kernels.cu.
// The body of CTA range `cta` (a kernel's CTA, or a virtual CTA of the
// persistent chunk).
template <int CK, int PR, bool CO>
__device__ __forceinline__ void kb_primal_body(const BatchBuffers& B, const long long cta) {
  constexpr int kBRPL = Tile<PR>::RPL;
  __shared__ double red[kWarps][PR];
  __shared__ double sqw[kWarps];
  const BatchActive act = *B.act;
  if (act.count == 0 || act.error) return;
  const long long q0 = B.cta_begin[cta], q1 = B.cta_begin[cta + 1];
  if (q0 >= q1) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int kk = find_segment<CO>(B.unit_prefix, act.count, q0);
  long long q = q0;
  while (q < q1) {
    const int k = B.ids[kk];
    const BatchInstance I = B.inst[k];
    const DevState* st = B.st + k;
    const long long base_u = B.unit_prefix[kk];
    const long long seg_end = min(q1, (long long)B.unit_prefix[kk + 1]);
    const int buf = st->buf;
    const double tau = st->step_size, omega = st->primal_weight, S = st->sum_weights;
    const bool zero_g = st->g_is_zero != 0;
    const bool first = !(S > 0.0);
    const double s = __ddiv_rn(tau, omega);
    const double nw = first ? 1.0 : __ddiv_rn(tau, S);
    const double aw = first ? 1.0 : __ddiv_rn(S, __dadd_rn(S, tau));
    float* __restrict__ X = B.X[buf] + I.x_off;
    float* __restrict__ Xa = B.X[buf ^ 1] + I.x_off;
    const double* __restrict__ u = B.u[buf] + I.row_off;
    const double* __restrict__ v = B.v[buf] + I.col_off;
    CostSource csrc;
    csrc.C = B.C ? B.C + I.x_off : nullptr;
    csrc.xs = B.xs ? B.xs + I.pts_off * B.dim : nullptr;
    csrc.ys = B.ys ? B.ys + I.tpts_off * B.dim : nullptr;
    csrc.dim = B.dim;
    CostReader<CK, kBR, kBRPL> cost(csrc, (float)st->cost_scale);
    // the sums of a lane's two row loads are kept apart (two shorter dependency
    // chains) and added at the end of the unit / segment
    double sqk[kBRPL];
#pragma unroll
    for (int kq = 0; kq < kBRPL; ++kq) sqk[kq] = 0.0;
    const long long ql0 = q - base_u, ql1 = seg_end - base_u;  // local unit range
    for (long long p = ql0 / I.n; p * I.n < ql1; ++p) {
      const long long jb = (ql0 > p * I.n ? ql0 : p * I.n) - p * I.n;
      const long long je = (ql1 < (p + 1) * I.n ? ql1 : (p + 1) * I.n) - p * I.n;
      const long long row0 = p * PR;
      double acc[kBRPL][kBR];
      float ur[kBRPL][kBR];  // the FP32 plan's entry arithmetic takes the duals in FP32
      bool ok[kBRPL];
#pragma unroll
      for (int kq = 0; kq < kBRPL; ++kq) {
        const long long i = row0 + kq * 32 * kBR + lane * kBR;
        ok[kq] = i < I.m;
#pragma unroll
        for (int e = 0; e < kBR; ++e) {
          acc[kq][e] = 0.0;
          ur[kq][e] = (ok[kq] && i + e < I.m && !zero_g) ? (float)ldro<CO>(u + i + e) : 0.0f;
        }
      }
      cost.panel(row0, lane, I.m, ok);
      // kJU columns per warp step: every load of the step is issued before any
      // entry is computed, so a warp keeps kJU units of plan and average in
      // flight (an FP32 plan with a coordinate cost has little else to load)
      for (long long j = jb + warp; j < je; j += kWarps * kJU) {
        typename CostReader<CK, kBR, kBRPL>::value_t cv[kJU][kBRPL][kBR];
        float xv[kJU][kBRPL][kBR], av[kJU][kBRPL][kBR];
        float vj[kJU];
#pragma unroll
        for (int ju = 0; ju < kJU; ++ju) {
          const long long jj = j + ju * kWarps;
          if (jj >= je) continue;
          vj[ju] = zero_g ? 0.0f : (float)ldro<CO>(v + jj);
          cost.column(jj);
          const long long col = jj * I.ld + row0 + lane * kBR;
#pragma unroll
          for (int kq = 0; kq < kBRPL; ++kq) {
            if (ok[kq]) {
              const long long idx = col + kq * 32 * kBR;
              cost.get(idx, kq, cv[ju][kq]);
              vldx<CO>(X + idx, xv[ju][kq]);
              if (!first) vldx<CO>(Xa + idx, av[ju][kq]);
            }
          }
        }
#pragma unroll
        for (int ju = 0; ju < kJU; ++ju) {
          const long long jj = j + ju * kWarps;
          if (jj >= je) continue;
          const long long col = jj * I.ld + row0 + lane * kBR;
          double csk[kBRPL];
#pragma unroll
          for (int kq = 0; kq < kBRPL; ++kq) csk[kq] = 0.0;
#pragma unroll
          for (int kq = 0; kq < kBRPL; ++kq) {
            if (ok[kq]) {
              const long long i = row0 + kq * 32 * kBR + lane * kBR;
#pragma unroll
              for (int e = 0; e < kBR; ++e) {
                if (i + e < I.m) {
                  double d;
                  primal_entry<float>(widen(cv[ju][kq][e]), ur[kq][e], vj[ju], s, nw, aw, zero_g, first,
                                      xv[ju][kq][e], av[ju][kq][e], d);
                  acc[kq][e] += d;
                  csk[kq] += d;
                  sqk[kq] = __fma_rn(d, d, sqk[kq]);
                } else {  // padded row
                  xv[ju][kq][e] = 0.0f;
                  av[ju][kq][e] = 0.0f;
                }
              }
              const long long idx = col + kq * 32 * kBR;
              vst<float, kBR>(X + idx, xv[ju][kq]);
              vst<float, kBR>(Xa + idx, av[ju][kq]);
            }
          }
          const double cs = warp_sum(lane_sum(csk));
          if (lane == 0) B.colpart[base_u + p * I.n + jj] = cs;
        }
      }
#pragma unroll
      for (int kq = 0; kq < kBRPL; ++kq)
#pragma unroll
        for (int e = 0; e < kBR; ++e) red[warp][kq * 32 * kBR + lane * kBR + e] = acc[kq][e];
      __syncthreads();
      const long long gp = B.panel_prefix[kk] + p;
      for (int t = threadIdx.x; t < PR; t += kThreads) {
        double s2 = red[0][t];
#pragma unroll
        for (int w = 1; w < kWarps; ++w) s2 += red[w][t];
        B.rowpart[(cta + gp) * PR + t] = s2;
      }
      __syncthreads();
    }
    const double sq = warp_sum(lane_sum(sqk));
    if (lane == 0) sqw[warp] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s2 = sqw[0];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) s2 += sqw[w];
      B.sqpart[cta + kk] = s2;
    }
    __syncthreads();
    q = seg_end;
    ++kk;
  }
}

template <int CK, int PR>
__global__ void __launch_bounds__(kThreads, Tile<PR>::kMinBlocks) kb_primal(BatchBuffers B) {
  pdl_enter();
  kb_primal_body<CK, PR, false>(B, blockIdx.x);
}

// ---------------------------------------------------------------------------
// The batched primal pass with bulk-copy staging (the single solver's staged
// pass, over the concatenated unit line). Each warp keeps an S-stage ring in
// shared memory; lane 0 issues cp.async.bulk copies of the plan, average and
// stored cost of the warp's next units, which may lie in the next panel or the
// next instance, so the bytes in flight do not depend on registers. A unit is
// copied with the padded leading dimension (rows up to ld, a multiple of 8),
// so every copy starts and ends on a 16-byte boundary; the padded rows are
// zero in the plan and in the stored cost. Every wait is bounded: on a timeout
// the kernel sets kernel_error of the instance at hand, drains (bounded) the
// copies in flight and leaves its remaining units alone.
template <int CK, int PR>
struct BatchStagedLayout {
  static constexpr bool kPts = is_point_cost(CK);
  static constexpr int kCBytes = kPts ? 0 : PR * 4;
  static constexpr int kXBytes = PR * 4;
  static constexpr int kStageBytes = kCBytes + 2 * kXBytes;
  static constexpr int S0 = Tile<PR>::kRingBudget / (kWarps * kStageBytes);
  static constexpr int S = S0 > 6 ? 6 : (S0 < 2 ? 2 : S0);
  static constexpr int kRingBytes = kWarps * S * kStageBytes;
  static constexpr int kSmem = kRingBytes + kWarps * S * 8;
};

// The units of warp w in a CTA's range [q0, q1) of the active unit line, in
// the order the pass consumes them: by instance, by panel, columns w, w+8, ...
struct BatchCursor {
  int kk, k, buf;
  bool first, valid;
  int n, p, j, je, ld, ql1;  // local to the current instance (units of one instance fit 32 bits)
  long long x_off;
  __device__ __forceinline__ void init(const BatchBuffers& B, int count, long long q0, long long q1, int w) {
    kk = find_segment(B.unit_prefix, count, q0);
    valid = true;
    enter(B, count, q0, q1, w, true);
  }
  // the instance of segment kk: its local range and first column of this warp
  __device__ __forceinline__ void enter(const BatchBuffers& B, int count, long long q0, long long q1, int w,
                                        bool first_segment) {
    for (;;) {
      if (kk >= count) {
        valid = false;
        return;
      }
      const long long base = B.unit_prefix[kk];
      if (base >= q1) {
        valid = false;
        return;
      }
      k = B.ids[kk];
      const BatchInstance& I = B.inst[k];
      n = (int)I.n;
      ld = (int)I.ld;
      x_off = I.x_off;
      buf = B.st[k].buf;
      first = !(B.st[k].sum_weights > 0.0);
      const long long ql0 = (first_segment ? q0 : base) - base;
      const long long end = B.unit_prefix[kk + 1];
      ql1 = (int)((q1 < end ? q1 : end) - base);
      p = (int)(ql0 / n);
      const int jb = (int)(ql0 - (long long)p * n);
      je = (ql1 < (p + 1) * n ? ql1 : (p + 1) * n) - p * n;
      j = jb + w;
      if (normalize_panels(w)) return;
      ++kk;
      first_segment = false;
    }
  }
  // true while (p, j) is a unit of the current instance
  __device__ __forceinline__ bool normalize_panels(int w) {
    while (j >= je) {
      ++p;
      if (p * n >= ql1) return false;
      je = (ql1 < (p + 1) * n ? ql1 : (p + 1) * n) - p * n;
      j = w;
    }
    return true;
  }
  __device__ __forceinline__ void advance(const BatchBuffers& B, int count, long long q0, long long q1, int w) {
    j += kWarps;
    if (normalize_panels(w)) return;
    ++kk;
    enter(B, count, q0, q1, w, false);
  }
};

template <int CK, int PR>
__global__ void __launch_bounds__(kThreads, Tile<PR>::kMinBlocks) kb_primal_staged(BatchBuffers B) {
  using L = BatchStagedLayout<CK, PR>;
  constexpr int kBRPL = Tile<PR>::RPL;
  // the rings, the row-sum tiles and the per-CTA reserve of the resident CTAs fit an SM's 228 KB
  static_assert((L::kSmem + 8 * kWarps * (PR + 1) + 1024) * Tile<PR>::kMinBlocks <= 228 * 1024,
                "the resident CTAs hold their rings");
  constexpr int S = L::S;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double red[kWarps][PR];
  __shared__ double sqw[kWarps];
  pdl_enter();
  const BatchActive act = *B.act;
  if (act.count == 0 || act.error) return;
  const long long cta = blockIdx.x;
  const long long q0 = B.cta_begin[cta], q1 = B.cta_begin[cta + 1];
  if (q0 >= q1) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned char* ring = smem + (size_t)warp * S * L::kStageBytes;
  const uint32_t bar0 = smem_u32(smem + L::kRingBytes) + (uint32_t)(warp * S * 8);
  if (lane == 0) {
    for (int t = 0; t < S; ++t) mbar_init(bar0 + 8 * t, 1);
    fence_mbar_init();
  }
  __syncwarp();

  // lane 0 fills stage t with the producer cursor's unit
  auto issue = [&](const BatchCursor& c, int t) {
    const long long row0 = (long long)c.p * PR;
    const long long rows = ((long long)c.ld - row0) < PR ? ((long long)c.ld - row0) : PR;
    const uint32_t xb = (uint32_t)(rows * 4);
    const uint32_t cb = L::kPts ? 0u : xb;
    const uint32_t bar = bar0 + 8 * t;
    unsigned char* stg = ring + (size_t)t * L::kStageBytes;
    const long long off = (long long)c.j * c.ld + row0;
    mbar_expect_tx(bar, cb + xb + (c.first ? 0u : xb));
    if (!L::kPts) bulk_g2s(smem_u32(stg), B.C + c.x_off + off, cb, bar);
    bulk_g2s(smem_u32(stg + L::kCBytes), B.X[c.buf] + c.x_off + off, xb, bar);
    if (!c.first) bulk_g2s(smem_u32(stg + L::kCBytes + L::kXBytes), B.X[c.buf ^ 1] + c.x_off + off, xb, bar);
  };

  // the producer walks the warp's units ahead of the consumer, which visits
  // them in the same order through the structured loops below
  BatchCursor prod;
  prod.init(B, act.count, q0, q1, warp);
  long long issued = 0, consumed = 0;
  int cstage = 0;           // consumed % S, kept incrementally (no 64-bit division per unit)
  uint32_t cphase = 0;      // (consumed / S) & 1
  for (int t = 0; t < S && prod.valid; ++t) {
    if (lane == 0) issue(prod, t);
    prod.advance(B, act.count, q0, q1, warp);
    ++issued;
  }
  bool failed = false;
  int kk = find_segment(B.unit_prefix, act.count, q0);
  long long q = q0;
  while (q < q1) {
    const int k = B.ids[kk];
    const BatchInstance I = B.inst[k];
    DevState* st = B.st + k;
    const long long base_u = B.unit_prefix[kk];
    const long long seg_end = min(q1, (long long)B.unit_prefix[kk + 1]);
    const int buf = st->buf;
    const double tau = st->step_size, omega = st->primal_weight, Ssum = st->sum_weights;
    const bool zero_g = st->g_is_zero != 0;
    const bool first = !(Ssum > 0.0);
    // the FP32 plan's entry arithmetic takes its step weights in FP32
    const float s = (float)__ddiv_rn(tau, omega);
    const float nw = first ? 1.0f : (float)__ddiv_rn(tau, Ssum);
    const float aw = first ? 1.0f : (float)__ddiv_rn(Ssum, __dadd_rn(Ssum, tau));
    float* __restrict__ X = B.X[buf] + I.x_off;
    float* __restrict__ Xa = B.X[buf ^ 1] + I.x_off;
    const double* __restrict__ u = B.u[buf] + I.row_off;
    const double* __restrict__ v = B.v[buf] + I.col_off;
    CostSource csrc;
    csrc.C = nullptr;
    csrc.xs = B.xs ? B.xs + I.pts_off * B.dim : nullptr;
    csrc.ys = B.ys ? B.ys + I.tpts_off * B.dim : nullptr;
    csrc.dim = B.dim;
    CostReader<CK, kBR, kBRPL> cost(csrc, (float)st->cost_scale);
    // the sums of a lane's two row loads are kept apart (two shorter dependency
    // chains) and added at the end of the unit / segment
    double sqk[kBRPL];
#pragma unroll
    for (int kq = 0; kq < kBRPL; ++kq) sqk[kq] = 0.0;
    const long long ql0 = q - base_u, ql1 = seg_end - base_u;
    for (long long p = ql0 / I.n; p * I.n < ql1; ++p) {
      const long long row0 = p * PR;
      double acc[kBRPL][kBR];
      float ur[kBRPL][kBR];
      bool ok[kBRPL];
      int nv[kBRPL];  // rows of this lane's load that exist (the rest are padding)
#pragma unroll
      for (int kq = 0; kq < kBRPL; ++kq) {
        const long long i = row0 + kq * 32 * kBR + lane * kBR;
        nv[kq] = (int)min(max(I.m - i, 0ll), (long long)kBR);
        ok[kq] = nv[kq] > 0;
#pragma unroll
        for (int e = 0; e < kBR; ++e) {
          acc[kq][e] = 0.0;
          ur[kq][e] = (e < nv[kq] && !zero_g) ? (float)__ldg(u + i + e) : 0.0f;
        }
      }
      cost.panel(row0, lane, I.m, ok);
      const long long jb = (ql0 > p * I.n ? ql0 : p * I.n) - p * I.n;
      const long long je = (ql1 < (p + 1) * I.n ? ql1 : (p + 1) * I.n) - p * I.n;
      // the column's dual and coordinates are loaded one unit ahead
      double vnext = 0.0;
      if (jb + warp < je) {
        if (!zero_g) vnext = __ldg(v + jb + warp);
        cost.prefetch(jb + warp);
      }
      for (long long j = jb + warp; !failed && j < je; j += kWarps) {
        const int stage = cstage;
        const uint32_t parity = cphase;
        if (!mbar_wait_bounded(bar0 + 8 * stage, parity)) {
          failed = true;
          if (lane == 0) {
            atomicExch(&st->kernel_error, 1);
            atomicExch(&B.act->error, 1);
          }
          break;
        }
        const unsigned char* stg = ring + (size_t)stage * L::kStageBytes;
        const float* sC = reinterpret_cast<const float*>(stg);
        const float* sX = reinterpret_cast<const float*>(stg + L::kCBytes);
        const float* sXa = reinterpret_cast<const float*>(stg + L::kCBytes + L::kXBytes);
        const float vj = (float)vnext;
        cost.take();
        if (j + kWarps < je) {
          if (!zero_g) vnext = __ldg(v + j + kWarps);
          cost.prefetch(j + kWarps);
        }
        const long long col = j * I.ld + row0 + lane * kBR;
        double csk[kBRPL];
#pragma unroll
        for (int kq = 0; kq < kBRPL; ++kq) csk[kq] = 0.0;
#pragma unroll
        for (int kq = 0; kq < kBRPL; ++kq) {
          if (ok[kq]) {
            const int r = kq * 32 * kBR + lane * kBR;
            typename CostReader<CK, kBR, kBRPL>::value_t cv[kBR];
            if constexpr (L::kPts)
              cost.get(0, kq, cv);
            else
              vld<float, kBR>(sC + r, cv);
            float xv[kBR], av[kBR];
            vld<float, kBR>(sX + r, xv);
            if (!first) vld<float, kBR>(sXa + r, av);
#pragma unroll
            for (int e = 0; e < kBR; ++e) {
              if (e < nv[kq]) {
                double d;
                primal_entry<float>(widen(cv[e]), ur[kq][e], vj, s, nw, aw, zero_g, first, xv[e], av[e], d);
                acc[kq][e] += d;
                csk[kq] += d;
                sqk[kq] = __fma_rn(d, d, sqk[kq]);
              } else {  // padded row
                xv[e] = 0.0f;
                av[e] = 0.0f;
              }
            }
            vst<float, kBR>(X + col + kq * 32 * kBR, xv);
            vst<float, kBR>(Xa + col + kq * 32 * kBR, av);
          }
        }
        const double cs = warp_sum(lane_sum(csk));
        if (lane == 0) B.colpart[base_u + p * I.n + j] = cs;
        __syncwarp();
        ++consumed;
        if (++cstage == S) {
          cstage = 0;
          cphase ^= 1u;
        }
        if (prod.valid) {
          if (lane == 0) issue(prod, stage);
          prod.advance(B, act.count, q0, q1, warp);
          ++issued;
        }
      }
#pragma unroll
      for (int kq = 0; kq < kBRPL; ++kq)
#pragma unroll
        for (int e = 0; e < kBR; ++e) red[warp][kq * 32 * kBR + lane * kBR + e] = acc[kq][e];
      __syncthreads();
      const long long gp = B.panel_prefix[kk] + p;
      for (int t = threadIdx.x; t < PR; t += kThreads) {
        double s2 = red[0][t];
#pragma unroll
        for (int w = 1; w < kWarps; ++w) s2 += red[w][t];
        B.rowpart[(cta + gp) * PR + t] = s2;
      }
      __syncthreads();
    }
    const double sq = warp_sum(lane_sum(sqk));
    if (lane == 0) sqw[warp] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
      double s2 = sqw[0];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) s2 += sqw[w];
      B.sqpart[cta + kk] = s2;
    }
    __syncthreads();
    q = seg_end;
    ++kk;
  }
  if (consumed < issued) {
    // only after a timeout: drain the copies still in flight (bounded) before
    // the shared memory goes away, and report
    if (!failed && lane == 0) {
      atomicExch(&B.st[B.ids[find_segment(B.unit_prefix, act.count, q0)]].kernel_error, 1);
      atomicExch(&B.act->error, 1);
    }
    for (long long c = consumed; c < issued; ++c)
      mbar_wait_bounded(bar0 + 8 * (int)(c % S), (uint32_t)((c / S) & 1));
  }
}

// Batched dual step + per-instance step control (last CTA of each instance).
template <int PR, bool CO>
__device__ __forceinline__ void kb_dual_body(const BatchBuffers& B, const SolveConfig& cfg, const int grid,
                                             const long long blk) {
  const BatchActive act = *B.act;
  if (act.count == 0 || act.error) return;
  if (blk >= B.vblock_prefix[act.count]) return;
  const int kk = find_segment<CO>(B.vblock_prefix, act.count, blk);
  const int k = B.ids[kk];
  const BatchInstance I = B.inst[k];
  DevState* st = B.st + k;
  const long long lb = blk - B.vblock_prefix[kk];  // block inside the instance
  const int buf = st->buf;
  const double tau = st->step_size, omega = st->primal_weight, S = st->sum_weights;
  DualArgs A;
  A.first = !(S > 0.0);
  A.tw = __dmul_rn(tau, omega);
  A.nw = A.first ? 1.0 : __ddiv_rn(tau, S);
  A.aw = A.first ? 1.0 : __ddiv_rn(S, __dadd_rn(S, tau));
  const long long ubase = B.unit_prefix[kk];
  double vals[kStepSums] = {0.0, 0.0};
  if (lb < I.rblocks) {
    const long long i = lb * kVecThreads + threadIdx.x;
    if (i < I.m) {
      const long long p = i / PR, t = i - p * PR;
      const long long gp = B.panel_prefix[kk] + p;
      const long long lo = bcta_of_unit(B.cta_begin, grid, ubase + p * I.n), hi = bcta_of_unit(B.cta_begin, grid, ubase + (p + 1) * I.n - 1);
      double sd = 0.0;
      if (!act.any_empty) {
        // every CTA owns a unit: the slots c + gp, c = lo..hi, all hold partials
        sd = sum_strided(B.rowpart + (lo + gp) * PR + t, hi - lo + 1, PR);
      } else {
        // some CTA ranges are empty (the tail of a solve): skip them, their
        // slots hold nothing of this panel
        for (long long c = lo; c <= hi; ++c) {
          if (B.cta_begin[c] == B.cta_begin[c + 1]) continue;
          sd += B.rowpart[(c + gp) * PR + t];
        }
      }
      const long long o = I.row_off + i;
      dual_entry(sd, B.a[o], B.r[buf] + o, B.u[buf] + o, B.r[buf ^ 1] + o, B.u[buf ^ 1] + o, A, vals[0], vals[1]);
    }
  } else {
    const long long j = (lb - I.rblocks) * kVecThreads + threadIdx.x;
    if (j < I.n) {
      const double sd = sum_strided(B.colpart + ubase + j, I.panels, I.n);
      const long long o = I.col_off + j;
      dual_entry(sd, B.b[o], B.c[buf] + o, B.v[buf] + o, B.c[buf ^ 1] + o, B.v[buf ^ 1] + o, A, vals[0], vals[1]);
    }
  }
  block_reduce<kStepSums>(vals, 0u, B.steppart + blk * kStepSums);
  if (!elect_last_of(&st->ticket_step, (unsigned)(I.rblocks + I.cblocks))) return;
  // warps 0-2 reduce the three partial sets side by side, warp 3 computes the
  // step rule's powers; thread 0 then runs the step control
  __shared__ double fin[2 * kStepSums + 1];
  __shared__ StepPowers pw;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w == 0) {
    double rs[kStepSums];
    warp_reduce_partials<kStepSums>(B.steppart, B.vblock_prefix[kk], I.rblocks, 0u, rs);
    if (lane == 0) fin[0] = rs[0], fin[1] = rs[1];
  } else if (w == 1) {
    double cs[kStepSums];
    warp_reduce_partials<kStepSums>(B.steppart, B.vblock_prefix[kk] + I.rblocks, I.cblocks, 0u, cs);
    if (lane == 0) fin[2] = cs[0], fin[3] = cs[1];
  } else if (w == 2) {
    double xs[1];
    const long long lo = bcta_of_unit(B.cta_begin, grid, ubase), hi = bcta_of_unit(B.cta_begin, grid, B.unit_prefix[kk + 1] - 1);
    sum_cta_slots<1>(B.sqpart, B.cta_begin, lo, hi, kk, 0u, xs);
    if (lane == 0) fin[4] = xs[0];
  } else if (w == 3 && lane == 0) {
    pw = step_powers(st, cfg);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    step_control(st, cfg, fin[0], fin[2], fin[4], fin[1] + fin[3], pw);
    st->ticket_step = 0;
  }
}
template <int PR>
__global__ void __launch_bounds__(kVecThreads) kb_dual(BatchBuffers B, SolveConfig cfg, int grid) {
  pdl_enter();
  kb_dual_body<PR, false>(B, cfg, grid, blockIdx.x);
}

// Batched evaluation, matrix part: per (CTA, instance) partials.
template <int CK, int PR, bool CO>
__device__ __forceinline__ void kb_eval_body(const BatchBuffers& B, const long long cta, const int grid) {
  constexpr int kBRPL = Tile<PR>::RPL;
  const BatchActive act = *B.act;
  if (act.count == 0 || act.error) return;
  const long long q0 = B.cta_begin[cta], q1 = B.cta_begin[cta + 1];
  if (q0 >= q1) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int kk = find_segment<CO>(B.unit_prefix, act.count, q0);
  long long q = q0;
  while (q < q1) {
    const int k = B.ids[kk];
    const BatchInstance I = B.inst[k];
    DevState* st = B.st + k;
    if (cta == bcta_of_unit(B.cta_begin, grid, B.unit_prefix[kk]) && threadIdx.x == 0) st->eval_t0_ns = globaltimer_ns();
    const long long base_u = B.unit_prefix[kk];
    const long long seg_end = min(q1, (long long)B.unit_prefix[kk + 1]);
    const int buf = st->buf;
    const bool have_avg = st->avg_count > 0;
    const bool zero_g = st->g_is_zero != 0;
    const float* __restrict__ X = B.X[buf] + I.x_off;
    const float* __restrict__ Xa = B.X[buf ^ 1] + I.x_off;
    const double* __restrict__ u = B.u[buf] + I.row_off;
    const double* __restrict__ v = B.v[buf] + I.col_off;
    const double* __restrict__ ua = B.u[buf ^ 1] + I.row_off;
    const double* __restrict__ va = B.v[buf ^ 1] + I.col_off;
    CostSource csrc;
    csrc.C = B.C ? B.C + I.x_off : nullptr;
    csrc.xs = B.xs ? B.xs + I.pts_off * B.dim : nullptr;
    csrc.ys = B.ys ? B.ys + I.tpts_off * B.dim : nullptr;
    csrc.dim = B.dim;
    CostReader<CK, kBR, kBRPL> cost(csrc, (float)st->cost_scale);
    double accv[kEvalSums];
#pragma unroll
    for (int e = 0; e < kEvalSums; ++e) accv[e] = 0.0;
    const long long ql0 = q - base_u, ql1 = seg_end - base_u;
    for (long long p = ql0 / I.n; p * I.n < ql1; ++p) {
      const long long jb = (ql0 > p * I.n ? ql0 : p * I.n) - p * I.n;
      const long long je = (ql1 < (p + 1) * I.n ? ql1 : (p + 1) * I.n) - p * I.n;
      const long long row0 = p * PR;
      double ur[kBRPL][kBR], uar[kBRPL][kBR];
      bool ok[kBRPL];
#pragma unroll
      for (int kq = 0; kq < kBRPL; ++kq) {
        const long long i = row0 + kq * 32 * kBR + lane * kBR;
        ok[kq] = i < I.m;
#pragma unroll
        for (int e = 0; e < kBR; ++e) {
          const bool in = ok[kq] && i + e < I.m;
          ur[kq][e] = in ? ldro<CO>(u + i + e) : 0.0;
          uar[kq][e] = (in && have_avg) ? ldro<CO>(ua + i + e) : 0.0;
        }
      }
      cost.panel(row0, lane, I.m, ok);
      for (long long j = jb + warp; j < je; j += kWarps) {
        const double vj = ldro<CO>(v + j);
        const double vaj = have_avg ? ldro<CO>(va + j) : 0.0;
        cost.column(j);
        const long long col = j * I.ld + row0 + lane * kBR;
#pragma unroll
        for (int kq = 0; kq < kBRPL; ++kq) {
          if (!ok[kq]) continue;
          const long long idx = col + kq * 32 * kBR;
          const long long i = row0 + kq * 32 * kBR + lane * kBR;
          typename CostReader<CK, kBR, kBRPL>::value_t cv[kBR];
          float xv[kBR], av[kBR];
          cost.get(idx, kq, cv);
          vldro<CO>(X + idx, xv);
          if (have_avg) vldro<CO>(Xa + idx, av);
#pragma unroll
          for (int e = 0; e < kBR; ++e) {
            if (i + e >= I.m) continue;
            const double c = widen(cv[e]), x = widen(xv[e]);
            const double gg = zero_g ? 0.0 : __dsub_rn(__dsub_rn(c, ur[kq][e]), vj);
            const double mg = neg_part(gg);
            accv[E_DOT] += c * x;
            accv[E_SQX] += x * x;
            accv[E_MAXX] = nanmax(accv[E_MAXX], fabs(x));
            accv[E_SQG] += mg * mg;
            accv[E_MAXG] = nanmax(accv[E_MAXG], mg);
            if (have_avg) {
              const double xa = widen(av[e]);
              const double ga = __dsub_rn(__dsub_rn(c, uar[kq][e]), vaj);
              const double mga = neg_part(ga);
              accv[E_AVG + E_DOT] += c * xa;
              accv[E_AVG + E_SQX] += xa * xa;
              accv[E_AVG + E_MAXX] = nanmax(accv[E_AVG + E_MAXX], fabs(xa));
              accv[E_AVG + E_SQG] += mga * mga;
              accv[E_AVG + E_MAXG] = nanmax(accv[E_AVG + E_MAXG], mga);
            }
          }
        }
      }
    }
    block_reduce<kEvalSums>(accv, kEvalMaxMask, B.evpart + (cta + kk) * kEvalSums);
    q = seg_end;
    ++kk;
  }
}
template <int CK, int PR>
__global__ void __launch_bounds__(kThreads, 2) kb_eval(BatchBuffers B) {
  pdl_enter();
  kb_eval_body<CK, PR, false>(B, blockIdx.x, (int)gridDim.x);
}

// Batched evaluation, vector part + per-instance evaluation control.
// start_only: the evaluation of the initial points, run once after
// kb_init_state when some instance starts warm; the warm instances record
// their start point as the last restart point (record_start_point) and no
// instance takes any other step of the evaluation block.
template <bool CO>
__device__ __forceinline__ void kb_eval_vec_body(const BatchBuffers& B, const SolveConfig& cfg, const int grid,
                                                 const int start_only, const long long blk) {
  const BatchActive act = *B.act;
  if (act.count == 0 || act.error) return;
  if (blk >= B.vblock_prefix[act.count]) return;
  const int kk = find_segment<CO>(B.vblock_prefix, act.count, blk);
  const int k = B.ids[kk];
  const BatchInstance I = B.inst[k];
  DevState* st = B.st + k;
  const long long lb = blk - B.vblock_prefix[kk];
  const int buf = st->buf;
  const bool have_avg = st->avg_count > 0;
  double acc[kVecSums];
#pragma unroll
  for (int e = 0; e < kVecSums; ++e) acc[e] = 0.0;
  const bool is_row = lb < I.rblocks;
  const long long idx = (is_row ? lb : lb - I.rblocks) * kVecThreads + threadIdx.x;
  if (idx < (is_row ? I.m : I.n)) {
    const long long o = (is_row ? I.row_off : I.col_off) + idx;
    const double dist = is_row ? B.a[o] : B.b[o];
    const double sc = (is_row ? B.r[buf] : B.c[buf])[o];
    const double dc = (is_row ? B.u[buf] : B.v[buf])[o];
    const double res = dist - sc;
    acc[V_SQRES] = res * res;
    acc[V_MAXRES] = fabs(res);
    acc[V_DOT] = dist * dc;
    acc[V_SQDUAL] = dc * dc;
    acc[V_MAXDUAL] = fabs(dc);
    if (have_avg) {
      const double sa = (is_row ? B.r[buf ^ 1] : B.c[buf ^ 1])[o];
      const double da = (is_row ? B.u[buf ^ 1] : B.v[buf ^ 1])[o];
      const double ra = dist - sa;
      acc[V_AVG + V_SQRES] = ra * ra;
      acc[V_AVG + V_MAXRES] = fabs(ra);
      acc[V_AVG + V_DOT] = dist * da;
      acc[V_AVG + V_SQDUAL] = da * da;
      acc[V_AVG + V_MAXDUAL] = fabs(da);
    }
  }
  block_reduce<kVecSums>(acc, kVecMaxMask, B.vecpart + blk * kVecSums);
  if (!elect_last_of(&st->ticket_eval, (unsigned)(I.rblocks + I.cblocks))) return;
  // warps 0-2 reduce the three partial sets side by side
  __shared__ double fin[kEvalSums + 2 * kVecSums];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w == 0) {
    const long long lo = bcta_of_unit(B.cta_begin, grid, B.unit_prefix[kk]);
    const long long hi = bcta_of_unit(B.cta_begin, grid, B.unit_prefix[kk + 1] - 1);
    double E[kEvalSums];
    sum_cta_slots<kEvalSums>(B.evpart, B.cta_begin, lo, hi, kk, kEvalMaxMask, E);
    if (lane == 0)
      for (int q = 0; q < kEvalSums; ++q) fin[q] = E[q];
  } else if (w == 1) {
    double R[kVecSums];
    warp_reduce_partials<kVecSums>(B.vecpart, B.vblock_prefix[kk], I.rblocks, kVecMaxMask, R);
    if (lane == 0)
      for (int q = 0; q < kVecSums; ++q) fin[kEvalSums + q] = R[q];
  } else if (w == 2) {
    double Cc[kVecSums];
    warp_reduce_partials<kVecSums>(B.vecpart, B.vblock_prefix[kk] + I.rblocks, I.cblocks, kVecMaxMask, Cc);
    if (lane == 0)
      for (int q = 0; q < kVecSums; ++q) fin[kEvalSums + kVecSums + q] = Cc[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double* E = fin;
    const double* R = fin + kEvalSums;
    const double* Cc = fin + kEvalSums + kVecSums;
    const PointSums cur = point_sums(E, R, Cc, 0);
    const PointSums avg = point_sums(E, R, Cc, E_AVG);
    if (!start_only)
      eval_control(st, cfg, cur, avg, B.rec + k, 1);
    else if (B.warm[k])
      record_start_point(st, cur);
    st->ticket_eval = 0;
  }
}
__global__ void __launch_bounds__(kVecThreads) kb_eval_vec(BatchBuffers B, SolveConfig cfg, int grid,
                                                            int start_only) {
  pdl_enter();
  kb_eval_vec_body<false>(B, cfg, grid, start_only, blockIdx.x);
}

// Rebuild the active list and its prefix sums (one CTA, instances in order),
// then the CTA ranges: CTA c starts at the first active unit whose cumulative
// cost reaches c / grid of the total, a unit costing 8 * rows + unit_cost * 256
// (integers, so the split is exact and repeatable). Within an instance the
// units run panel-major, n units of PR rows per full panel and n units of the
// remaining rows in the last panel, so the start of a range follows in closed
// form after a binary search over the instances' cost prefix.
// One CTA of blockDim.x <= 1024 threads runs it (the kernel: 1024; the
// persistent chunk: CTA 0 with its 256).
template <int PR>
__device__ __forceinline__ void kb_compact_body(const BatchBuffers& B, const int grid) {
  __shared__ int flags[1024];
  __shared__ int base;
  __shared__ long long total_cost;
  __shared__ int empty_flag;
  const int T = (int)blockDim.x;
  if (threadIdx.x == 0) {
    base = 0;
    empty_flag = 0;
  }
  if (B.race) {
    // racing instances: once a member of a group is optimal, the others stop
    for (int k = threadIdx.x; k < B.num; k += blockDim.x) {
      const int g = B.race[k];
      if (g >= 0 && B.st[k].done && B.st[k].termination_reason == PDOT_TERMINATION_REASON_OPTIMAL)
        atomicMin(B.winner + g, k);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < B.num; k += blockDim.x) {
      const int g = B.race[k];
      if (g < 0 || B.st[k].done) continue;
      const int w = __ldcg(B.winner + g);
      if (w < B.num && w != k) {
        B.st[k].done = 1;
        B.st[k].termination_reason = PDOT_TERMINATION_REASON_OTHER;
      }
    }
  }
  __syncthreads();
  long long units = 0, panels = 0, vblocks = 0, cost = 0;
  const long long wu = (long long)B.unit_cost * kUnitCostRows;
  for (int off = 0; off < B.num; off += T) {
    const int k = off + threadIdx.x;
    flags[threadIdx.x] = (k < B.num && !B.st[k].done) ? 1 : 0;
    __syncthreads();
    if (threadIdx.x == 0) {
      int c = base;
      for (int t = 0; t < T && off + t < B.num; ++t) {
        if (!flags[t]) continue;
        const int kk = off + t;
        const BatchInstance& I = B.inst[kk];
        B.ids[c] = kk;
        B.unit_prefix[c] = units;
        B.panel_prefix[c] = panels;
        B.vblock_prefix[c] = vblocks;
        B.cost_prefix[c] = cost;
        units += I.panels * I.n;
        panels += I.panels;
        vblocks += I.rblocks + I.cblocks;
        cost += I.n * (8 * I.m + wu * I.panels);
        ++c;
      }
      base = c;
      B.unit_prefix[c] = units;
      B.panel_prefix[c] = panels;
      B.vblock_prefix[c] = vblocks;
      B.cost_prefix[c] = cost;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    B.act->count = base;
    B.act->total_units = units;
    total_cost = cost;
  }
  __syncthreads();
  const int count = base;
  const long long W = total_cost;
  for (int c = threadIdx.x; c <= grid; c += blockDim.x) {
    long long q;
    if (count == 0 || c == 0) {
      q = 0;
    } else if (c == grid) {
      q = B.unit_prefix[count];
    } else {
      const long long T = (long long)c * W / grid;
      // the largest kk with cost_prefix[kk] <= T (plain loads: written above)
      int lo = 0, hi = count - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (B.cost_prefix[mid] <= T)
          lo = mid;
        else
          hi = mid - 1;
      }
      const BatchInstance& I = B.inst[B.ids[lo]];
      const long long e = T - B.cost_prefix[lo];
      const long long uf = 8 * PR + wu;                          // a unit of a full panel
      const long long ul = 8 * (I.m - PR * (I.panels - 1)) + wu;  // a unit of the last panel
      const long long F = I.n * uf;                                      // a full panel
      long long local;
      if (e < (I.panels - 1) * F) {
        const long long p = e / F;
        local = p * I.n + (e - p * F + uf - 1) / uf;
      } else {
        local = (I.panels - 1) * I.n + (e - (I.panels - 1) * F + ul - 1) / ul;
      }
      q = B.unit_prefix[lo] + local;
    }
    B.cta_begin[c] = q;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < grid; c += blockDim.x)
    if (B.cta_begin[c] == B.cta_begin[c + 1]) empty_flag = 1;
  __syncthreads();
  if (threadIdx.x == 0) B.act->any_empty = empty_flag;
}
template <int PR>
__global__ void kb_compact(BatchBuffers B, int grid) {
  pdl_enter();
  kb_compact_body<PR>(B, grid);
}

// ---------------------------------------------------------------------------
// Persistent chunk: one cooperative launch runs a regular chunk of loop bodies
// of the whole batch (the evaluation, the compaction, then `steps` iterations
// of primal pass and dual step) with grid barriers between the phases instead
// of kernel boundaries. Every phase runs the body of its kernel over the same
// virtual CTAs (physical CTA b takes the CTA ranges b, b + gridDim.x, ... of
// the `grid` ranges the kernels use) and the same vector blocks, with the same
// last-block elections, so the results are bit-identical to the CUDA graph's
// launches. It runs the direct primal pass: the staged pass's ring does not
// fit beside the other phases' shared memory. Data written earlier in the
// launch is loaded through L2 (CO = true), never through the read-only path.
// A barrier whose poll runs out sets the batch's error word and the CTA
// leaves; the other CTAs' polls see the word and leave too.
template <int CK, int PR>
__global__ void __launch_bounds__(kThreads, 1)
    kb_chunk(BatchBuffers B, SolveConfig cfg, int grid, int vblocks, int steps) {
  static_assert(kThreads == kVecThreads, "the chunk runs the vector passes' blocks on its CTAs");
  BatchActive* A = B.act;
  const unsigned P = gridDim.x;
  auto sync = [&]() -> bool {
    if (grid_barrier(&A->bar_count, &A->bar_gen, P, &A->error)) return true;
    if (threadIdx.x == 0) atomicExch(&A->error, 1);
    return false;
  };
  for (long long c = blockIdx.x; c < grid; c += P) {
    kb_eval_body<CK, PR, true>(B, c, grid);
    __syncthreads();
  }
  if (!sync()) return;
  for (long long b = blockIdx.x; b < vblocks; b += P) {
    kb_eval_vec_body<true>(B, cfg, grid, 0, b);
    __syncthreads();
  }
  if (!sync()) return;
  if (blockIdx.x == 0) kb_compact_body<PR>(B, grid);
  if (!sync()) return;
  for (int k = 0; k < steps; ++k) {
    // the same value in every CTA: read after the same barrier
    if (__ldcg(&A->count) == 0 || __ldcg(&A->error) != 0) return;
    for (long long c = blockIdx.x; c < grid; c += P) {
      kb_primal_body<CK, PR, true>(B, c);
      __syncthreads();
    }
    if (!sync()) return;
    for (long long b = blockIdx.x; b < vblocks; b += P) {
      kb_dual_body<PR, true>(B, cfg, grid, b);
      __syncthreads();
    }
    if (!sync()) return;
  }
}

// Per-instance cost norms (stage one, over the full unit line).
template <int CK, int PR>
__global__ void __launch_bounds__(kThreads, 2) kb_norms(BatchBuffers B) {
  constexpr int kBRPL = Tile<PR>::RPL;
  const BatchActive act = *B.act;
  const long long cta = blockIdx.x;
  const long long q0 = B.cta_begin[cta], q1 = B.cta_begin[cta + 1];
  if (q0 >= q1) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int kk = find_segment(B.unit_prefix, act.count, q0);
  long long q = q0;
  while (q < q1) {
    const int k = B.ids[kk];
    const BatchInstance I = B.inst[k];
    const long long base_u = B.unit_prefix[kk];
    const long long seg_end = min(q1, (long long)B.unit_prefix[kk + 1]);
    CostSource csrc;
    csrc.C = B.C ? B.C + I.x_off : nullptr;
    csrc.xs = B.xs ? B.xs + I.pts_off * B.dim : nullptr;
    csrc.ys = B.ys ? B.ys + I.tpts_off * B.dim : nullptr;
    csrc.dim = B.dim;
    CostReader<CK, kBR, kBRPL> cost(csrc, 1.0f);
    double accv[kNormSums] = {0.0, 0.0};
    const long long ql0 = q - base_u, ql1 = seg_end - base_u;
    for (long long p = ql0 / I.n; p * I.n < ql1; ++p) {
      const long long jb = (ql0 > p * I.n ? ql0 : p * I.n) - p * I.n;
      const long long je = (ql1 < (p + 1) * I.n ? ql1 : (p + 1) * I.n) - p * I.n;
      const long long row0 = p * PR;
      bool ok[kBRPL];
#pragma unroll
      for (int kq = 0; kq < kBRPL; ++kq) ok[kq] = row0 + kq * 32 * kBR + lane * kBR < I.m;
      cost.panel(row0, lane, I.m, ok);
      for (long long j = jb + warp; j < je; j += kWarps) {
        cost.column(j);
        const long long col = j * I.ld + row0 + lane * kBR;
#pragma unroll
        for (int kq = 0; kq < kBRPL; ++kq) {
          if (!ok[kq]) continue;
          const long long i = row0 + kq * 32 * kBR + lane * kBR;
          typename CostReader<CK, kBR, kBRPL>::value_t cv[kBR];
          cost.get(col + kq * 32 * kBR, kq, cv);
#pragma unroll
          for (int e = 0; e < kBR; ++e) {
            if (i + e >= I.m) continue;
            const double c = widen(cv[e]);
            accv[0] += c * c;
            accv[1] = nanmax(accv[1], fabs(c));
          }
        }
      }
    }
    block_reduce<kNormSums>(accv, 2u, B.evpart + (cta + kk) * kNormSums);
    q = seg_end;
    ++kk;
  }
}

// Per-instance initial state (one warp per instance), cf. k0_init.
__global__ void kb_init_state(BatchBuffers B, SolveConfig cfg, int grid) {
  const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const BatchActive act = *B.act;
  if (warp_global >= act.count) return;
  const int kk = warp_global;
  const int k = B.ids[kk];
  const BatchInstance I = B.inst[k];
  const long long lo = bcta_of_unit(B.cta_begin, grid, B.unit_prefix[kk]), hi = bcta_of_unit(B.cta_begin, grid, B.unit_prefix[kk + 1] - 1);
  double nc[kNormSums];
  sum_cta_slots<kNormSums>(B.evpart, B.cta_begin, lo, hi, kk, 2u, nc);
  double sqab = 0.0, mxab = 0.0;
  for (long long i = lane; i < I.m + I.n; i += 32) {
    const double x = i < I.m ? B.a[I.row_off + i] : B.b[I.col_off + i - I.m];
    sqab += x * x;
    mxab = nanmax(mxab, fabs(x));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sqab += __shfl_xor_sync(0xffffffffu, sqab, o);
    mxab = nanmax(mxab, __shfl_xor_sync(0xffffffffu, mxab, o));
  }
  if (lane != 0) return;
  DevState* st = B.st + k;
  double scale = 1.0;
  if (B.xs) {
    scale = cfg.cost_scale > 0.0 ? cfg.cost_scale : (nc[1] > 0.0 ? 1.0 / nc[1] : 1.0);
    nc[0] *= scale * scale;
    nc[1] *= scale;
  }
  memset(st, 0, sizeof(*st));
  st->cost_scale = scale;
  st->linf_obj = nc[1];
  st->l2_obj = sqrt(nc[0]);
  st->linf_rhs = mxab;
  st->l2_rhs = sqrt(sqab);
  st->step_size = cfg.adaptive ? 1.0 : (1.0 - 0.2) / sqrt((double)(I.m + I.n));
  if (cfg.scale_invariant_initial_primal_weight) {
    const double rhs = st->l2_rhs, obj = st->l2_obj;
    st->primal_weight = (obj > 0.0 && rhs > 0.0) ? cfg.primal_importance * (obj / rhs) : cfg.primal_importance;
  } else {
    st->primal_weight = cfg.primal_importance;
  }
  if (B.warm[k] && B.warm_omega && B.warm_omega[k] > 0.0) st->primal_weight = B.warm_omega[k];
  st->iteration = 1;
  st->last_rp = st->l2_rhs;
  st->ratio_last_trial = 1.0;
  st->last_restart_length = 1;
  st->g_is_zero = B.warm[k] ? 0 : 1;
  st->out_current = 1;
  if (!(isfinite(st->l2_obj) && isfinite(st->l2_rhs) && isfinite(st->linf_obj))) {
    st->done = 1;
    st->termination_reason = PDOT_TERMINATION_REASON_INVALID_PROBLEM;
  }
  st->t_start_ns = globaltimer_ns();
}

// Widen a padded FP32 plan of one instance into a dense FP64 column-major one.
__global__ void kb_widen(const float* __restrict__ X, int64_t m, int64_t n, int64_t ld, double* __restrict__ out) {
  const int64_t N = m * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / m, i = e - j * m;
    out[e] = (double)X[i + j * ld];
  }
}

__global__ void kb_convert_cost(const double* __restrict__ src, int64_t m, int64_t n, int64_t ld,
                                float* __restrict__ dst) {
  const int64_t N = ld * n;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < N; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / ld, i = e - j * ld;
    dst[e] = i < m ? __double2float_rn(src[i + j * m]) : 0.0f;
  }
}

#define PDOT_BATCH_KINDS(kind, KERNEL, PRV, LAUNCH)                                              \
  switch (kind) {                                                                                 \
    case PDOT_COST_F32: { auto kfn = KERNEL<PDOT_COST_F32, PRV>; LAUNCH; } break;                 \
    case pdot::kCostSqBase + 1: { auto kfn = KERNEL<pdot::kCostSqBase + 1, PRV>; LAUNCH; } break; \
    case pdot::kCostSqBase + 2: { auto kfn = KERNEL<pdot::kCostSqBase + 2, PRV>; LAUNCH; } break; \
    case pdot::kCostSqBase + 3: { auto kfn = KERNEL<pdot::kCostSqBase + 3, PRV>; LAUNCH; } break; \
    case pdot::kCostL1Base + 1: { auto kfn = KERNEL<pdot::kCostL1Base + 1, PRV>; LAUNCH; } break; \
    case pdot::kCostL1Base + 2: { auto kfn = KERNEL<pdot::kCostL1Base + 2, PRV>; LAUNCH; } break; \
    default: { auto kfn = KERNEL<pdot::kCostL1Base + 3, PRV>; LAUNCH; } break;                    \
  }
// a matrix-pass kernel for the cost kind and the tile's panel rows (128 or 256)
#define PDOT_BATCH_VARIANT(kind, pr, KERNEL, LAUNCH)        \
  do {                                                      \
    if ((pr) == 128) {                                      \
      PDOT_BATCH_KINDS(kind, KERNEL, 128, LAUNCH)           \
    } else {                                                \
      PDOT_BATCH_KINDS(kind, KERNEL, 256, LAUNCH)           \
    }                                                       \
  } while (0)

}  // namespace
}  // namespace pdot

// ============================================================================
// Host side
namespace {

struct BatchFailure {
  int code;
  std::string msg;
};

[[noreturn]] void bfail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw BatchFailure{code, buf};
}

void bck(cudaError_t e, const char* what, int line) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    bfail(e == cudaErrorMemoryAllocation ? PDOT_ERR_OUT_OF_MEMORY : PDOT_ERR_CUDA, "%s failed: %s (pdot_batch.cu:%d)",
          what, cudaGetErrorString(e), line);
  }
}
#define BCK(x) bck((x), #x, __LINE__)

class BatchSolver {
 public:
  BatchSolver(const pdot_batch_problem& P, const pdot_pdhg_parameters& prm, const pdot_solver_options* opt) {
    device_ = opt ? opt->device : 0;
    const int pub_kind = opt ? opt->cost_storage : PDOT_COST_F32;
    dim_ = (pub_kind == PDOT_COST_SQEUCLID_POINTS || pub_kind == PDOT_COST_L1_POINTS) ? opt->point_dim : 0;
    kind_ = pdot::internal_cost_kind(pub_kind, dim_);
    use_graph_ = opt ? opt->use_cuda_graph != 0 : true;
    pr_ = (opt && opt->batch_panel_rows) ? opt->batch_panel_rows : 256;
    if (pr_ != 128 && pr_ != 256) bfail(PDOT_ERR_INVALID_ARGUMENT, "batch_panel_rows must be 0, 128 or 256");
    const int B = (int)P.num_instances;
    num_ = B;
    BCK(cudaSetDevice(device_));
    BCK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    // instance layout
    inst_.resize(B);
    int64_t xo = 0, ro = 0, co = 0, po = 0, to = 0, units = 0, panels = 0, vblocks = 0;
    for (int k = 0; k < B; ++k) {
      pdot::BatchInstance& I = inst_[k];
      I.m = P.num_rows[k];
      I.n = P.num_cols[k];
      I.ld = (I.m + 7) / 8 * 8;
      I.x_off = xo;
      I.row_off = ro;
      I.col_off = co;
      I.pts_off = po;
      I.tpts_off = to;
      I.panels = (I.m + pr_ - 1) / pr_;
      I.rblocks = (I.m + pdot::kVecThreads - 1) / pdot::kVecThreads;
      I.cblocks = (I.n + pdot::kVecThreads - 1) / pdot::kVecThreads;
      xo += I.ld * I.n;
      ro += I.m;
      co += I.n;
      po += I.m;
      to += I.n;
      units += I.panels * I.n;
      panels += I.panels;
      vblocks += I.rblocks + I.cblocks;
    }
    total_x_ = xo;
    total_units_ = units;
    total_panels_ = panels;
    total_vblocks_ = vblocks;
    int sms = 148;
    BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
    // the primal pass: staged by bulk copies for the coordinate costs (whose
    // plan and average are all there is to load), direct 16-byte loads for the
    // stored FP32 cost; primal_pass overrides
    const int pass = opt ? opt->primal_pass : PDOT_PASS_AUTO;
    // persistent chunks (1) run the direct pass throughout; 0 (automatic) and
    // -1 keep the CUDA graph, which measured faster on B200
    persistent_ = opt && opt->persistent_chunks == 1;
    if (persistent_ && pass == PDOT_PASS_STAGED)
      bfail(PDOT_ERR_INVALID_ARGUMENT, "persistent chunks run the direct primal pass (primal_pass AUTO or DIRECT)");
    staged_ = !persistent_ && (pass == PDOT_PASS_STAGED || (pass == PDOT_PASS_AUTO && dim_ > 0));
    int occ = 1;
    if (staged_) {
      PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_primal_staged, {
        const int smem = staged_smem(kind_, pr_);
        if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, pdot::kThreads, smem) != cudaSuccess || occ < 1)
          occ = 1;
      });
    } else {
      PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_primal,
                         if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, pdot::kThreads, 0) !=
                                 cudaSuccess ||
                             occ < 1) occ = 1);
    }
    cudaGetLastError();
    grid_ = (int)std::min<int64_t>((int64_t)sms * occ, std::max<int64_t>(units, 1));
    if (opt && opt->ctas_per_sm > 0)
      grid_ = (int)std::min<int64_t>((int64_t)std::min(opt->ctas_per_sm, occ) * sms, std::max<int64_t>(units, 1));
    if (persistent_) {
      // as many co-resident CTAs as the chunk kernel allows, at most one per CTA range
      int coop = 0, cocc = 0;
      BCK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device_));
      PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_chunk, {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cocc, kfn, pdot::kThreads, 0) != cudaSuccess) cocc = 0;
      });
      cudaGetLastError();
      if (!coop || cocc < 1) bfail(PDOT_ERR_CUDA, "this device cannot run the persistent chunk kernel");
      chunk_ctas_ = std::min(sms * cocc, grid_);
    }
    // per-unit overhead of the CTA split, in eighths of a full unit (0..64)
    if (opt && opt->warm_restart_at_zero != 0 && opt->warm_restart_at_zero != 1)
      bfail(PDOT_ERR_INVALID_ARGUMENT, "warm_restart_at_zero must be 0 or 1");
    warm_zero_ = opt && opt->warm_restart_at_zero == 1;
    const double uc = opt ? opt->batch_unit_cost : 0.0;
    if (!(uc >= 0.0 && uc <= 8.0)) bfail(PDOT_ERR_INVALID_ARGUMENT, "batch_unit_cost must be in [0, 8]");
    D_.unit_cost = (int)std::lround(uc * 8.0);

    // device buffers
    D_.inst = upload(inst_.data(), B);
    D_.num = B;
    D_.dim = dim_;
    if (dim_ == 0) {
      float* C = alloc<float>(total_x_);
      double* tmp = nullptr;
      size_t tmp_cap = 0;
      for (int k = 0; k < B; ++k) {
        const size_t mn = (size_t)inst_[k].m * inst_[k].n;
        if (mn > tmp_cap) {
          if (tmp) BCK(cudaFree(tmp));
          BCK(cudaMalloc(&tmp, mn * sizeof(double)));
          tmp_cap = mn;
        }
        BCK(cudaMemcpyAsync(tmp, P.cost_matrices[k], mn * sizeof(double), cudaMemcpyHostToDevice, stream_));
        pdot::kb_convert_cost<<<256, 256, 0, stream_>>>(tmp, inst_[k].m, inst_[k].n, inst_[k].ld, C + inst_[k].x_off);
        BCK(cudaGetLastError());
        BCK(cudaStreamSynchronize(stream_));
      }
      if (tmp) BCK(cudaFree(tmp));
      D_.C = C;
      D_.xs = D_.ys = nullptr;
    } else {
      float* xs = alloc<float>((size_t)po * dim_);
      float* ys = alloc<float>((size_t)to * dim_);
      for (int k = 0; k < B; ++k) {
        BCK(cudaMemcpyAsync(xs + inst_[k].pts_off * dim_, P.source_points[k], (size_t)inst_[k].m * dim_ * sizeof(float),
                            cudaMemcpyHostToDevice, stream_));
        BCK(cudaMemcpyAsync(ys + inst_[k].tpts_off * dim_, P.target_points[k], (size_t)inst_[k].n * dim_ * sizeof(float),
                            cudaMemcpyHostToDevice, stream_));
      }
      D_.C = nullptr;
      D_.xs = xs;
      D_.ys = ys;
    }
    double* a = alloc<double>(ro);
    double* b = alloc<double>(co);
    for (int k = 0; k < B; ++k) {
      BCK(cudaMemcpyAsync(a + inst_[k].row_off, P.source_distributions[k], inst_[k].m * sizeof(double),
                          cudaMemcpyHostToDevice, stream_));
      BCK(cudaMemcpyAsync(b + inst_[k].col_off, P.target_distributions[k], inst_[k].n * sizeof(double),
                          cudaMemcpyHostToDevice, stream_));
    }
    D_.a = a;
    D_.b = b;
    for (int h = 0; h < 2; ++h) {
      D_.X[h] = alloc<float>(total_x_);
      D_.u[h] = alloc<double>(ro);
      D_.r[h] = alloc<double>(ro);
      D_.v[h] = alloc<double>(co);
      D_.c[h] = alloc<double>(co);
    }
    rows_ = ro;
    cols_ = co;
    // warm starts: duals, the plan narrowed to FP32 (padded columns) and its sums
    std::vector<int> warm(B, 0);
    for (int k = 0; k < B; ++k)
      if (P.warm_dual_sources && P.warm_dual_targets && P.warm_dual_sources[k] && P.warm_dual_targets[k])
        warm[k] = 1;
      else if (P.warm_primals && P.warm_primals[k])
        bfail(PDOT_ERR_INVALID_ARGUMENT, "instance %d: a warm-start plan needs the warm-start dual vectors", k);
    any_warm_ = false;
    for (int k = 0; k < B; ++k) any_warm_ = any_warm_ || warm[k];
    D_.warm = upload(warm.data(), B);
    if (P.warm_primal_weights) {
      std::vector<double> om(B, 0.0);
      for (int k = 0; k < B; ++k) {
        const double w = P.warm_primal_weights[k];
        if (!std::isfinite(w)) bfail(PDOT_ERR_INVALID_ARGUMENT, "instance %d: warm_primal_weight must be finite", k);
        om[k] = (warm[k] && w > 0.0) ? w : 0.0;
      }
      D_.warm_omega = upload(om.data(), B);
    }
    if (any_warm_) {
      std::vector<double> hu(ro, 0.0), hv(co, 0.0), hr(ro, 0.0), hc(co, 0.0);
      std::vector<float> hx;
      warm_x_ = alloc<float>(total_x_);
      BCK(cudaMemsetAsync(warm_x_, 0, total_x_ * sizeof(float), stream_));
      for (int k = 0; k < B; ++k) {
        if (!warm[k]) continue;
        const pdot::BatchInstance& I = inst_[k];
        memcpy(hu.data() + I.row_off, P.warm_dual_sources[k], I.m * sizeof(double));
        memcpy(hv.data() + I.col_off, P.warm_dual_targets[k], I.n * sizeof(double));
        if (!P.warm_primals || !P.warm_primals[k]) continue;
        const double* X0 = P.warm_primals[k];
        hx.assign((size_t)I.ld * I.n, 0.0f);
        for (int64_t j = 0; j < I.n; ++j) {
          double cs = 0.0;
          for (int64_t i = 0; i < I.m; ++i) {
            const float x = (float)X0[i + j * I.m];
            hx[i + j * I.ld] = x;
            cs += (double)x;
            hr[I.row_off + i] += (double)x;
          }
          hc[I.col_off + j] = cs;
        }
        BCK(cudaMemcpy(warm_x_ + I.x_off, hx.data(), hx.size() * sizeof(float), cudaMemcpyHostToDevice));
      }
      warm_u_ = alloc<double>(ro);
      warm_v_ = alloc<double>(co);
      warm_r_ = alloc<double>(ro);
      warm_c_ = alloc<double>(co);
      BCK(cudaMemcpy(warm_u_, hu.data(), ro * sizeof(double), cudaMemcpyHostToDevice));
      BCK(cudaMemcpy(warm_v_, hv.data(), co * sizeof(double), cudaMemcpyHostToDevice));
      BCK(cudaMemcpy(warm_r_, hr.data(), ro * sizeof(double), cudaMemcpyHostToDevice));
      BCK(cudaMemcpy(warm_c_, hc.data(), co * sizeof(double), cudaMemcpyHostToDevice));
    }
    // race groups: an instance stops (reason OTHER) once another member of
    // its group has ended optimal
    if (P.race_groups) {
      std::vector<int> rg(B);
      for (int k = 0; k < B; ++k) {
        rg[k] = P.race_groups[k];
        if (rg[k] < -1 || rg[k] >= B)
          bfail(PDOT_ERR_INVALID_ARGUMENT, "instance %d: race group %d is not in -1..num_instances-1", k, rg[k]);
      }
      D_.race = upload(rg.data(), B);
      D_.winner = alloc<int>(B);
    }
    // plans recovered from the warm duals of the instances given no warm plan
    const double peps = opt ? opt->warm_plan_epsilon : 0.0;
    if (opt && (!(peps >= 0.0) || !std::isfinite(peps) || opt->warm_plan_iterations < 0 ||
                opt->warm_plan_iterations > 100000))
      bfail(PDOT_ERR_INVALID_ARGUMENT, "warm_plan_epsilon must be finite and >= 0, warm_plan_iterations 0..100000");
    if (peps > 0.0 && any_warm_) {
      std::vector<pdot::PlanInstance> pi(B);
      std::vector<long long> rp(B + 1, 0), cp(B + 1, 0);
      for (int k = 0; k < B; ++k) {
        const pdot::BatchInstance& I = inst_[k];
        pi[k] = pdot::PlanInstance{I.m, I.n, I.ld, I.x_off, I.row_off, I.col_off,
                                   (warm[k] && !(P.warm_primals && P.warm_primals[k])) ? 1 : 0, 0};
        rp[k + 1] = rp[k] + I.m;
        cp[k + 1] = cp[k] + I.n;
      }
      plan_iters_ = opt->warm_plan_iterations;
      wp_.inst = upload(pi.data(), B);
      wp_.num = B;
      wp_.row_prefix = upload(rp.data(), B + 1);
      wp_.col_prefix = upload(cp.data(), B + 1);
      wp_.total_rows = ro;
      wp_.total_cols = co;
      wp_.kind = kind_;
      wp_.dim = dim_;
      wp_.C = D_.C;
      wp_.xs = D_.xs;
      wp_.ys = D_.ys;
      wp_.a = D_.a;
      wp_.b = D_.b;
      wp_.u0 = warm_u_;
      wp_.v0 = warm_v_;
      wp_.f = alloc<double>(ro);
      wp_.g = alloc<double>(co);
      wp_.X = D_.X[0];
      wp_.plan_f32 = 1;
      wp_.r = D_.r[0];
      wp_.c = D_.c[0];
      wp_.eps = peps;
      recover_plans_ = true;
    }
    D_.rowpart = alloc<double>(((size_t)grid_ + total_panels_) * pr_);
    D_.colpart = alloc<double>(total_units_);
    D_.sqpart = alloc<double>((size_t)grid_ + B);
    D_.steppart = alloc<double>((size_t)total_vblocks_ * pdot::kStepSums);
    D_.evpart = alloc<double>(((size_t)grid_ + B) * pdot::kEvalSums);
    D_.vecpart = alloc<double>((size_t)total_vblocks_ * pdot::kVecSums);
    D_.st = alloc<pdot::DevState>(B);
    D_.rec = alloc<pdot_iteration_stats>(B);
    D_.act = alloc<pdot::BatchActive>(1);
    BCK(cudaMemset(D_.act, 0, sizeof(pdot::BatchActive)));
    D_.ids = alloc<int>(B);
    D_.unit_prefix = alloc<long long>(B + 1);
    D_.panel_prefix = alloc<long long>(B + 1);
    D_.cost_prefix = alloc<long long>(B + 1);
    D_.cta_begin = alloc<long long>(grid_ + 1);
    D_.vblock_prefix = alloc<long long>(B + 1);
    cfg_ = pdot::SolveConfig{};
    fill_config(prm);
    freq_ = prm.termination_evaluation_frequency;
    limit_ = prm.termination_criteria.iteration_limit;
    void* hp = nullptr;
    BCK(cudaMallocHost(&hp, sizeof(pdot::BatchActive) * 2));
    host_act_ = static_cast<pdot::BatchActive*>(hp);
    for (int k = 0; k < 2; ++k) BCK(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming));
    if (use_graph_ && !persistent_) capture();
  }

  ~BatchSolver() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (graph_) cudaGraphExecDestroy(graph_);
    for (int k = 0; k < 2; ++k)
      if (ev_[k]) cudaEventDestroy(ev_[k]);
    if (host_act_) cudaFreeHost(host_act_);
    for (void* p : allocs_) cudaFree(p);
    if (stream_) cudaStreamDestroy(stream_);
  }

  void run(pdot_batch_output* outs, double* seconds) {
    cudaEvent_t t0, t1;
    BCK(cudaEventCreate(&t0));
    BCK(cudaEventCreate(&t1));
    BCK(cudaEventRecord(t0, stream_));
    init();
    long long it = 1;
    int issued = 0, completed = 0;
    for (;;) {
      while (issued - completed < 2) {
        enqueue_chunk(it);
        BCK(cudaMemcpyAsync(&host_act_[issued % 2], D_.act, sizeof(pdot::BatchActive), cudaMemcpyDeviceToHost, stream_));
        BCK(cudaEventRecord(ev_[issued % 2], stream_));
        ++issued;
      }
      BCK(cudaEventSynchronize(ev_[completed % 2]));
      const pdot::BatchActive a = host_act_[completed % 2];
      ++completed;
      if (a.error) {
        BCK(cudaStreamSynchronize(stream_));
        bfail(PDOT_ERR_CUDA, "a bounded wait timed out (the staged primal pass's copies or a persistent chunk barrier)");
      }
      if (a.count == 0) break;
      if (it > (long long)limit_ + 2 * freq_ + 16)
        bfail(PDOT_ERR_CUDA, "batched solve did not finish by the iteration limit");
    }
    BCK(cudaEventRecord(t1, stream_));
    BCK(cudaStreamSynchronize(stream_));
    float ms = 0.0f;
    BCK(cudaEventElapsedTime(&ms, t0, t1));
    if (seconds) *seconds = ms / 1000.0;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    collect(outs);
  }

 private:
  template <typename T>
  T* alloc(size_t count) {
    void* p = nullptr;
    BCK(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    allocs_.push_back(p);
    return static_cast<T*>(p);
  }
  template <typename T>
  const T* upload(const T* src, size_t count) {
    T* d = alloc<T>(count);
    BCK(cudaMemcpy(d, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return d;
  }

  void fill_config(const pdot_pdhg_parameters& p) {
    pdot::SolveConfig& c = cfg_;
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
    // every evaluation overwrites the instance's one record, so an instance
    // stopped by its race group keeps its last evaluation
    c.record_iteration_stats = 1;
    c.scale_invariant_initial_primal_weight = p.scale_invariant_initial_primal_weight != 0;
    c.primal_importance = p.primal_importance;
    c.cost_scale = 0.0;
    c.warm_start = 0;
  }

  // zero (or warm) starts, cost norms, initial states, the first active list
  void init() {
    BCK(cudaMemsetAsync(D_.X[1], 0, total_x_ * sizeof(float), stream_));
    if (any_warm_) {
      BCK(cudaMemcpyAsync(D_.X[0], warm_x_, total_x_ * sizeof(float), cudaMemcpyDeviceToDevice, stream_));
      BCK(cudaMemcpyAsync(D_.u[0], warm_u_, rows_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      BCK(cudaMemcpyAsync(D_.r[0], warm_r_, rows_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      BCK(cudaMemcpyAsync(D_.v[0], warm_v_, cols_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      BCK(cudaMemcpyAsync(D_.c[0], warm_c_, cols_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    } else {
      BCK(cudaMemsetAsync(D_.X[0], 0, total_x_ * sizeof(float), stream_));
      BCK(cudaMemsetAsync(D_.u[0], 0, rows_ * sizeof(double), stream_));
      BCK(cudaMemsetAsync(D_.r[0], 0, rows_ * sizeof(double), stream_));
      BCK(cudaMemsetAsync(D_.v[0], 0, cols_ * sizeof(double), stream_));
      BCK(cudaMemsetAsync(D_.c[0], 0, cols_ * sizeof(double), stream_));
    }
    BCK(cudaMemsetAsync(D_.st, 0, num_ * sizeof(pdot::DevState), stream_));
    if (D_.winner) BCK(cudaMemsetAsync(D_.winner, 0x7F, num_ * sizeof(int), stream_));  // no winner yet
    BCK(cudaMemsetAsync(D_.rec, 0, num_ * sizeof(pdot_iteration_stats), stream_));
    launch_compact();
    BCK(cudaGetLastError());
    PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_norms, (kfn<<<grid_, pdot::kThreads, 0, stream_>>>(D_)));
    BCK(cudaGetLastError());
    pdot::kb_init_state<<<(num_ * 32 + 255) / 256, 256, 0, stream_>>>(D_, cfg_, grid_);
    BCK(cudaGetLastError());
    if (recover_plans_) {
      wp_.st = D_.st;  // allocated after the recovery arguments were set up
      BCK(pdot::launch_warm_plan(wp_, plan_iters_, stream_));
    }
    launch_compact();  // drops invalid problems
    BCK(cudaGetLastError());
    // warm instances start their restart information at the warm point, as
    // the reference starts it at its initial point (unless asked to start at
    // zero, kb_init_state's record)
    if (any_warm_ && !warm_zero_) {
      PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_eval, (kfn<<<grid_, pdot::kThreads, 0, stream_>>>(D_)));
      pdot::kb_eval_vec<<<(unsigned)total_vblocks_, pdot::kVecThreads, 0, stream_>>>(D_, cfg_, grid_, 1);
      BCK(cudaGetLastError());
    }
  }

  bool is_eval(long long it) const { return (it - 1) % freq_ == 0 || it == limit_ + 1 || it <= 10; }

  // the loop's kernels are launched with programmatic dependent launch (pdot::pdl_launch)
  void launch_compact() {
    BCK(pdot::pdl_launch(pr_ == 128 ? pdot::kb_compact<128> : pdot::kb_compact<256>, dim3(1), dim3(1024), 0, stream_,
                         D_, grid_));
  }
  void launch_eval() {
    PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_eval,
                       BCK(pdot::pdl_launch(kfn, dim3(grid_), dim3(pdot::kThreads), 0, stream_, D_)));
    BCK(pdot::pdl_launch(pdot::kb_eval_vec, dim3((unsigned)total_vblocks_), dim3(pdot::kVecThreads), 0, stream_, D_,
                         cfg_, grid_, 0));
    launch_compact();
  }
  static int staged_smem(int kind, int pr) {
    // the stored FP32 cost adds a plane to every stage; the coordinate costs do not
    if (pr == 128)
      return kind == PDOT_COST_F32 ? pdot::BatchStagedLayout<PDOT_COST_F32, 128>::kSmem
                                   : pdot::BatchStagedLayout<pdot::kCostSqBase + 1, 128>::kSmem;
    return kind == PDOT_COST_F32 ? pdot::BatchStagedLayout<PDOT_COST_F32, 256>::kSmem
                                 : pdot::BatchStagedLayout<pdot::kCostSqBase + 1, 256>::kSmem;
  }

  void launch_step() {
    if (staged_) {
      const int smem = staged_smem(kind_, pr_);
      PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_primal_staged,
                         BCK(pdot::pdl_launch(kfn, dim3(grid_), dim3(pdot::kThreads), smem, stream_, D_)));
    } else {
      PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_primal,
                         BCK(pdot::pdl_launch(kfn, dim3(grid_), dim3(pdot::kThreads), 0, stream_, D_)));
    }
    BCK(pdot::pdl_launch(pr_ == 128 ? pdot::kb_dual<128> : pdot::kb_dual<256>, dim3((unsigned)total_vblocks_),
                         dim3(pdot::kVecThreads), 0, stream_, D_, cfg_, grid_));
  }

  bool regular_start(long long it) const {
    if (!(graph_ || persistent_) || it <= 10 || (it - 1) % freq_ != 0) return false;
    for (long long k = it + 1; k < it + freq_; ++k)
      if (is_eval(k)) return false;
    return true;
  }

  void enqueue_chunk(long long& it) {
    if (regular_start(it)) {
      if (persistent_)
        launch_persistent_chunk();
      else
        BCK(cudaGraphLaunch(graph_, stream_));
      it += freq_;
      return;
    }
    long long k = 0;
    do {
      if (is_eval(it)) launch_eval();
      launch_step();
      ++it;
      ++k;
    } while (k < freq_ && !regular_start(it));
  }

  // the regular chunk as one cooperative launch of kb_chunk (bit-identical to the graph)
  void launch_persistent_chunk() {
    int grid = grid_, vblocks = (int)total_vblocks_, steps = (int)freq_;
    void* args[] = {&D_, &cfg_, &grid, &vblocks, &steps};
    PDOT_BATCH_VARIANT(kind_, pr_, pdot::kb_chunk,
                       BCK(cudaLaunchCooperativeKernel((const void*)kfn, dim3(chunk_ctas_), dim3(pdot::kThreads),
                                                       args, 0, stream_)));
  }

  void capture() {
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    launch_eval();
    for (long long k = 0; k < freq_; ++k) launch_step();
    BCK(cudaStreamEndCapture(stream_, &g));
    const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    BCK(e);
  }

  void collect(pdot_batch_output* outs) {
    std::vector<pdot::DevState> st(num_);
    std::vector<pdot_iteration_stats> rec(num_);
    BCK(cudaMemcpy(st.data(), D_.st, num_ * sizeof(pdot::DevState), cudaMemcpyDeviceToHost));
    BCK(cudaMemcpy(rec.data(), D_.rec, num_ * sizeof(pdot_iteration_stats), cudaMemcpyDeviceToHost));
    for (int k = 0; k < num_; ++k)
      if (st[k].kernel_error)
        bfail(PDOT_ERR_CUDA, "instance %d: the staged primal pass gave up waiting for its copies", k);
    double* tmp = nullptr;
    size_t cap = 0;
    for (int k = 0; k < num_; ++k) {
      const pdot::BatchInstance& I = inst_[k];
      pdot_batch_output& o = outs[k];
      o.termination_reason = st[k].termination_reason;
      o.iteration_count = (int32_t)(st[k].iteration - 1);
      o.final_stats = rec[k];
      const int xb = st[k].out_current ? st[k].buf : (st[k].buf ^ 1);
      const size_t mn = (size_t)I.m * I.n;
      if (o.primal_solution) {
        if (mn > cap) {
          if (tmp) BCK(cudaFree(tmp));
          BCK(cudaMalloc(&tmp, mn * sizeof(double)));
          cap = mn;
        }
        pdot::kb_widen<<<256, 256, 0, stream_>>>(D_.X[xb] + I.x_off, I.m, I.n, I.ld, tmp);
        BCK(cudaGetLastError());
        BCK(cudaMemcpyAsync(o.primal_solution, tmp, mn * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        BCK(cudaStreamSynchronize(stream_));
      }
      if (o.dual_source_solution)
        BCK(cudaMemcpy(o.dual_source_solution, D_.u[xb] + I.row_off, I.m * sizeof(double), cudaMemcpyDeviceToHost));
      if (o.dual_target_solution)
        BCK(cudaMemcpy(o.dual_target_solution, D_.v[xb] + I.col_off, I.n * sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (tmp) BCK(cudaFree(tmp));
  }

  int device_ = 0, num_ = 0, dim_ = 0, kind_ = 0, grid_ = 1, pr_ = 256, chunk_ctas_ = 0;
  bool persistent_ = false;  // regular chunks run as one persistent cooperative launch
  bool warm_zero_ = false;
  bool use_graph_ = true, any_warm_ = false, recover_plans_ = false, staged_ = false;
  int plan_iters_ = 0;
  pdot::WarmPlanArgs wp_{};
  float* warm_x_ = nullptr;
  double *warm_u_ = nullptr, *warm_v_ = nullptr, *warm_r_ = nullptr, *warm_c_ = nullptr;
  int64_t total_x_ = 0, total_units_ = 0, total_panels_ = 0, total_vblocks_ = 0, rows_ = 0, cols_ = 0;
  long long freq_ = 128, limit_ = 0;
  std::vector<pdot::BatchInstance> inst_;
  std::vector<void*> allocs_;
  pdot::BatchBuffers D_{};
  pdot::SolveConfig cfg_{};
  cudaStream_t stream_ = nullptr;
  cudaGraphExec_t graph_ = nullptr;
  cudaEvent_t ev_[2] = {};
  pdot::BatchActive* host_act_ = nullptr;
};

}  // namespace

extern "C" int pdot_optimize_batched(const pdot_batch_problem* problem, const pdot_pdhg_parameters* params,
                                     const pdot_solver_options* options, pdot_batch_output* outputs,
                                     double* solve_seconds) {
  pdot::set_last_error("");
  try {
    if (!problem || !params || !outputs) bfail(PDOT_ERR_INVALID_ARGUMENT, "null argument");
    if (problem->num_instances < 1 || problem->num_instances > pdot::kMaxBatch)
      bfail(PDOT_ERR_INVALID_ARGUMENT, "num_instances must be 1..%d", pdot::kMaxBatch);
    if (!problem->num_rows || !problem->num_cols || !problem->source_distributions || !problem->target_distributions)
      bfail(PDOT_ERR_INVALID_ARGUMENT, "null instance arrays");
    const int kind = options ? options->cost_storage : PDOT_COST_F32;
    const bool points = kind == PDOT_COST_SQEUCLID_POINTS || kind == PDOT_COST_L1_POINTS;
    if (!(kind == PDOT_COST_F32 || points))
      bfail(PDOT_ERR_INVALID_ARGUMENT, "the batched solver takes an FP32-stored or a coordinate cost");
    if (options && options->plan_precision != PDOT_PRECISION_F32)
      bfail(PDOT_ERR_INVALID_ARGUMENT, "the batched solver keeps FP32 plans (plan_precision must be F32)");
    if (points && (options->point_dim < 1 || options->point_dim > 3))
      bfail(PDOT_ERR_INVALID_ARGUMENT, "point_dim must be 1..3 for the batched solver");
    if (points && (!problem->source_points || !problem->target_points))
      bfail(PDOT_ERR_INVALID_ARGUMENT, "null point arrays");
    if (!points && !problem->cost_matrices) bfail(PDOT_ERR_INVALID_ARGUMENT, "null cost matrices");
    if (params->termination_evaluation_frequency < 1 || !(params->primal_importance > 0))
      bfail(PDOT_ERR_INVALID_ARGUMENT, "invalid parameters");
    if (options && options->batch_panel_rows != 0 && options->batch_panel_rows != 128 &&
        options->batch_panel_rows != 256)
      bfail(PDOT_ERR_INVALID_ARGUMENT, "batch_panel_rows must be 0, 128 or 256");
    if (options && (options->persistent_chunks < -1 || options->persistent_chunks > 1))
      bfail(PDOT_ERR_INVALID_ARGUMENT, "persistent_chunks must be -1, 0 or 1");
    for (int64_t k = 0; k < problem->num_instances; ++k) {
      if (problem->num_rows[k] < 1 || problem->num_cols[k] < 1) bfail(PDOT_ERR_INVALID_ARGUMENT, "empty instance %lld", (long long)k);
      // the staged pass's producer cursor keeps positions inside an instance in 32 bits
      if ((problem->num_rows[k] + 7) / 8 * 8 * problem->num_cols[k] >= (int64_t(1) << 31))
        bfail(PDOT_ERR_INVALID_ARGUMENT, "instance %lld: a batched instance holds fewer than 2^31 plan entries",
              (long long)k);
    }
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
      cudaGetLastError();
      bfail(PDOT_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    BatchSolver solver(*problem, *params, options);
    solver.run(outputs, solve_seconds);
    return PDOT_OK;
  } catch (const BatchFailure& f) {
    pdot::set_last_error(f.msg.c_str());
    return f.code;
  } catch (...) {
    pdot::set_last_error("unexpected C++ exception");
    return PDOT_ERR_CUDA;
  }
}
