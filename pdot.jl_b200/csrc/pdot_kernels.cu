// pdot_kernels.cu — sm_100a kernels of the FP64 PDHG-for-OT drop-in.
//
// Per PDHG iteration two launches run (both captured in a CUDA graph):
//   k1_primal  the fused matrix pass: reads C, X, Xavg once, writes X, Xavg,
//              emits per-(panel, column) column sums of the step, per-(CTA,
//              panel) row sums and per-CTA sum of squares. 40 B/entry in FP64.
//   k2_dual    finishes the two-stage sums in a fixed order, takes the dual
//              step and the vector averages, and its last CTA runs the
//              adaptive step-size rule (accept / retry bookkeeping).
// Every evaluation (iterations 1..10, then every termination_evaluation_
// frequency iterations) adds two more:
//   k3_eval    matrix reductions for the KKT statistics of the current and
//              average points (24 B/entry)
//   k4_eval    vector reductions; its last CTA computes the statistics, checks
//              termination, runs the restart scheme and the primal-weight
//              update, and writes one iteration-stats record.
//
// Elementwise arithmetic uses explicit round-to-nearest intrinsics in the
// reference's operation order (no fused multiply-add), so the projected step,
// the plan update and the averages round exactly as the reference's Julia code
// does; only the order of the sums differs.
//
// The matrix kernels are templates over the plan element (double for the FP64
// drop-in, float for mixed precision), the cost source (FP64 / FP32 / BF16
// storage, or the squared-Euclidean cost computed from FP32 coordinates) and
// the rows each lane loads at once (16 bytes of plan, or 1 on the scalar path
// for odd sizes and unaligned buffers). The FP64 plan's per-entry arithmetic is
// FP64; an FP32 plan's is FP32, its own precision (primal_entry). In both, the
// step entering the FP64 row/column sums is taken exactly between the stored
// values, so the sums track the stored plan exactly.
#include <cfloat>
#include <cmath>

#include "pdot_device.cuh"

namespace pdot {
namespace {

// ---------------------------------------------------------------------------
// The fused primal pass. Per entry (src/solver_gpu.jl:139-141,242,249-250;
// src/saddle_point_gpu.jl:129-130):
//   g  = (C - u_i) - v_j ;  t = max(X - s*g, 0) ;  d = t - X ;  X' = X + d
//   Xavg' = (Xavg + X'*nw)*aw      (Xavg' = X' after a reset of the average)
//
// XS: the next loop body evaluates, so the pass also accumulates that
// evaluation's plan sums of the updated current and average plans (the
// E_DOT, E_SQX, E_MAXX fields of k3_eval's partials, current and average) into
// `evpart`. Each thread visits the same entries in the same order as k3_eval
// and the block reduction is the same, so the sums are bit-identical to the
// ones k3_eval would compute from memory; k3_eval then reads only the cost.
constexpr int kXSums = 6;
__device__ __forceinline__ void xsums_add(double (&xa)[kXSums], double c, double x, double xav) {
  xa[0] += c * x;
  xa[1] += x * x;
  xa[2] = nanmax(xa[2], fabs(x));
  xa[3] += c * xav;
  xa[4] += xav * xav;
  xa[5] = nanmax(xa[5], fabs(xav));
}
__device__ __forceinline__ void xsums_store(double (&xa)[kXSums], double* evpart_cta) {
  __shared__ double xs_out[kXSums];
  block_reduce<kXSums>(xa, (1u << 2) | (1u << 5), xs_out);
  if (threadIdx.x == 0) {
    evpart_cta[E_DOT] = xs_out[0];
    evpart_cta[E_SQX] = xs_out[1];
    evpart_cta[E_MAXX] = xs_out[2];
    evpart_cta[E_AVG + E_DOT] = xs_out[3];
    evpart_cta[E_AVG + E_SQX] = xs_out[4];
    evpart_cta[E_AVG + E_MAXX] = xs_out[5];
  }
}

template <typename TX, int CK, int R, bool XS = false>
__device__ __forceinline__ void primal_pass_body(const CostSource& csrc, float scale, TX* __restrict__ X,
                                                 TX* __restrict__ Xa, const double* __restrict__ u,
                                                 const double* __restrict__ v, const double s,
                                                 const double nw, const double aw, const bool zero_g,
                                                 const bool first, double* __restrict__ colpart,
                                                 double* __restrict__ rowpart, double* __restrict__ sqpart,
                                                 const Geometry g, const int64_t cta,
                                                 double* __restrict__ evpart = nullptr) {
  constexpr int RPL = kPanelRows / (32 * R);
  __shared__ double red[kWarps][kPanelRows];
  __shared__ double sqw[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t m = g.m, n = g.n;
  const int64_t q0 = unit_begin(g, cta), q1 = unit_begin(g, cta + 1);
  CostReader<CK, R, RPL> cost(csrc, scale);
  double sq = 0.0;
  double xa[kXSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t p = q0 / n; p * n < q1; ++p) {
    const int64_t jb = (q0 > p * n ? q0 : p * n) - p * n;
    const int64_t je = (q1 < (p + 1) * n ? q1 : (p + 1) * n) - p * n;
    const int64_t row0 = p * kPanelRows;
    double acc[RPL][R];
    TX ur[RPL][R];  // an FP32 plan's entry arithmetic takes u_i in FP32: rounded once per panel
    bool ok[RPL];
#pragma unroll
    for (int k = 0; k < RPL; ++k) {
      const int64_t i = row0 + k * 32 * R + lane * R;
      ok[k] = i < m;
#pragma unroll
      for (int e = 0; e < R; ++e) {
        acc[k][e] = 0.0;
        ur[k][e] = (ok[k] && !zero_g) ? (TX)__ldcg(u + i + e) : (TX)0;
      }
    }
    cost.panel(row0, lane, m, ok);
    for (int64_t j = jb + warp; j < je; j += kWarps) {
      const double vj = zero_g ? 0.0 : __ldcg(v + j);
      cost.column(j);
      const int64_t base = j * m + row0 + lane * R;
      typename CostReader<CK, R, RPL>::value_t cv[RPL][R];
      TX xv[RPL][R], av[RPL][R];
#pragma unroll
      for (int k = 0; k < RPL; ++k) {
        if (ok[k]) {
          const int64_t idx = base + k * 32 * R;
          cost.get(idx, k, cv[k]);
          vld<TX, R>(X + idx, xv[k]);
          if (!first) vld<TX, R>(Xa + idx, av[k]);
        }
      }
      double cs = 0.0;
#pragma unroll
      for (int k = 0; k < RPL; ++k) {
        if (ok[k]) {
#pragma unroll
          for (int e = 0; e < R; ++e) {
            double d;
            primal_entry<TX>(widen(cv[k][e]), ur[k][e], vj, s, nw, aw, zero_g, first, xv[k][e], av[k][e], d);
            acc[k][e] += d;
            cs += d;
            add_sq<TX>(sq, d);
            if constexpr (XS) xsums_add(xa, widen(cv[k][e]), widen(xv[k][e]), widen(av[k][e]));
          }
          const int64_t idx = base + k * 32 * R;
          vst<TX, R>(X + idx, xv[k]);
          vst<TX, R>(Xa + idx, av[k]);
        }
      }
      cs = warp_sum(cs);
      if (lane == 0) colpart[p * n + j] = cs;
    }
    // this panel's row sums: combine the warps in a fixed order
#pragma unroll
    for (int k = 0; k < RPL; ++k)
#pragma unroll
      for (int e = 0; e < R; ++e) red[warp][k * 32 * R + lane * R + e] = acc[k][e];
    __syncthreads();
    for (int t = threadIdx.x; t < kPanelRows; t += kThreads) {
      double s2 = red[0][t];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) s2 += red[w][t];
      rowpart[row_slot(cta, p) * kPanelRows + t] = s2;
    }
    __syncthreads();
  }
  sq = warp_sum(sq);
  if (lane == 0) sqw[warp] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s2 = sqw[0];
#pragma unroll
    for (int w = 1; w < kWarps; ++w) s2 += sqw[w];
    sqpart[cta] = s2;
  }
  if constexpr (XS) xsums_store(xa, evpart + cta * kEvalSums);
}

// The duals are read through L2 (__ldcg): in the persistent chunk kernel the
// dual step of the same launch wrote them.
template <typename TX, int CK, int R, bool XS>
__device__ __forceinline__ void k1_primal_impl(const Buffers& B, const Geometry& g, const int64_t cta) {
  DevState* st = B.st;
  if (st->done | st->numerical_error | st->kernel_error) return;
  const int buf = st->buf;
  const double tau = st->step_size, omega = st->primal_weight, S = st->sum_weights;
  const bool zero_g = st->g_is_zero != 0;
  const bool first = !(S > 0.0);
  // compute_next_primal_solution! uses solver_state.step_size; the averaging
  // weight is the same solver_state.step_size (src/solver_gpu.jl:252).
  const double s = __ddiv_rn(tau, omega);
  const double nw = first ? 1.0 : __ddiv_rn(tau, S);
  const double aw = first ? 1.0 : __ddiv_rn(S, __dadd_rn(S, tau));
  primal_pass_body<TX, CK, R, XS>(B.cost, (float)st->cost_scale, static_cast<TX*>(B.X[buf]),
                                  static_cast<TX*>(B.X[buf ^ 1]), B.u[buf], B.v[buf], s, nw, aw, zero_g, first,
                                  B.colpart, B.rowpart, B.sqpart, g, cta, B.evpart);
  if (XS && cta == 0 && threadIdx.x == 0) st->xsums_iter = st->iteration;
}

template <typename TX, int CK, int R>
__global__ void __launch_bounds__(kThreads, 2) k1_primal(Buffers B, Geometry g) {
  pdl_enter();
  k1_primal_impl<TX, CK, R, false>(B, g, blockIdx.x);
}
// the same pass before an evaluation: it also leaves the evaluation's plan sums
template <typename TX, int CK, int R>
__global__ void __launch_bounds__(kThreads, 2) k1_primal_xs(Buffers B, Geometry g) {
  pdl_enter();
  k1_primal_impl<TX, CK, R, true>(B, g, blockIdx.x);
}

template <int R>
__global__ void __launch_bounds__(kThreads, 2)
    k1_primal_args(const double* C, double* X, double* Xa, const double* u, const double* v, double s,
                   double nw, double aw, int flags, double* colpart, double* rowpart, double* sqpart,
                   Geometry g) {
  CostSource cs;
  cs.C = C;
  cs.xs = cs.ys = nullptr;
  cs.dim = 0;
  primal_pass_body<double, PDOT_COST_F64, R>(cs, 1.0f, X, Xa, u, v, s, nw, aw,
                                             (flags & PDOT_PASS_ZERO_GRADIENT) != 0,
                                             (flags & PDOT_PASS_FIRST_AVERAGE) != 0, colpart, rowpart, sqpart, g,
                                             blockIdx.x);
}

// ---------------------------------------------------------------------------
// The fused primal pass with bulk-copy staging. Each warp keeps an S-stage
// ring in shared memory; lane 0 issues cp.async.bulk copies of the cost, plan
// and average segments of its next units (one mbarrier per stage, completed by
// the copies' byte count), so the bytes in flight no longer depend on the
// registers a lane can hold. Results are written straight to global memory.
// Every wait is bounded: on a timeout the kernel records kernel_error, waits
// (bounded) for the copies it still has in flight and returns.
template <typename TX, int CK>
struct StagedLayout {
  static constexpr bool kSq = is_point_cost(CK);
  using TC = typename CostReader<CK, 16 / sizeof(TX), kPanelRows / (32 * (16 / sizeof(TX)))>::value_t;
  static constexpr int kCBytes = kSq ? 0 : kPanelRows * (int)sizeof(TC);
  static constexpr int kXBytes = kPanelRows * (int)sizeof(TX);
  static constexpr int kStageBytes = kCBytes + 2 * kXBytes;
  // stages per warp: two CTAs (16 warps) per SM fit in shared memory
  static constexpr int S0 = (96 * 1024) / (kWarps * kStageBytes);
  static constexpr int S = S0 > 6 ? 6 : (S0 < 2 ? 2 : S0);
  static constexpr int kRingBytes = kWarps * S * kStageBytes;
  static constexpr int kSmem = kRingBytes + kWarps * S * 8;  // plus the mbarriers
};

template <typename TX, int CK>
__device__ __forceinline__ void k1_primal_staged_impl(const Buffers& B, const Geometry& g) {
  using L = StagedLayout<TX, CK>;
  constexpr int R = 16 / sizeof(TX);
  constexpr int RPL = kPanelRows / (32 * R);
  constexpr int S = L::S;
  using TC = typename L::TC;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ double red[kWarps][kPanelRows];
  __shared__ double sqw[kWarps];
  DevState* st = B.st;
  if (st->done | st->numerical_error | st->kernel_error) return;
  const int buf = st->buf;
  const double tau = st->step_size, omega = st->primal_weight, Ssum = st->sum_weights;
  const bool zero_g = st->g_is_zero != 0;
  const bool first = !(Ssum > 0.0);
  const double s = __ddiv_rn(tau, omega);
  const double nw = first ? 1.0 : __ddiv_rn(tau, Ssum);
  const double aw = first ? 1.0 : __ddiv_rn(Ssum, __dadd_rn(Ssum, tau));
  TX* __restrict__ X = static_cast<TX*>(B.X[buf]);
  TX* __restrict__ Xa = static_cast<TX*>(B.X[buf ^ 1]);
  const double* __restrict__ u = B.u[buf];
  const double* __restrict__ v = B.v[buf];
  const TC* __restrict__ Cg = static_cast<const TC*>(B.cost.C);
  CostReader<CK, R, RPL> cost(B.cost, (float)st->cost_scale);

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t m = g.m, n = g.n;
  const int64_t cta = blockIdx.x;
  const int64_t q0 = unit_begin(g, cta), q1 = unit_begin(g, cta + 1);
  unsigned char* ring = smem + (size_t)warp * S * L::kStageBytes;
  const uint32_t bar0 = smem_u32(smem + L::kRingBytes) + (uint32_t)(warp * S * 8);
  if (lane == 0) {
    for (int k = 0; k < S; ++k) mbar_init(bar0 + 8 * k, 1);
    fence_mbar_init();
  }
  __syncwarp();

  // lane 0 fills stage k with unit (p, j)
  auto issue = [&](int64_t p, int64_t j, int k) {
    const int64_t row0 = p * kPanelRows;
    const int64_t rows = (m - row0) < kPanelRows ? (m - row0) : kPanelRows;
    const uint32_t xb = (uint32_t)(rows * sizeof(TX));
    const uint32_t cb = L::kSq ? 0u : (uint32_t)(rows * sizeof(TC));
    const uint32_t bar = bar0 + 8 * k;
    unsigned char* stg = ring + (size_t)k * L::kStageBytes;
    const int64_t off = j * m + row0;
    mbar_expect_tx(bar, cb + xb + (first ? 0u : xb));
    if (!L::kSq) bulk_g2s(smem_u32(stg), Cg + off, cb, bar);
    bulk_g2s(smem_u32(stg + L::kCBytes), X + off, xb, bar);
    if (!first) bulk_g2s(smem_u32(stg + L::kCBytes + L::kXBytes), Xa + off, xb, bar);
  };

  UnitCursor prod, cons;
  prod.init(q0, q1, n, warp);
  cons.init(q0, q1, n, warp);
  long long issued = 0, consumed = 0;
  int cstage = 0;           // consumed % S, kept incrementally (no 64-bit division per unit)
  uint32_t cphase = 0;      // (consumed / S) & 1
  for (int k = 0; k < S && prod.valid; ++k) {
    if (lane == 0) issue(prod.p, prod.j, k);
    prod.advance(warp);
    ++issued;
  }
  bool failed = false;
  // consumer waits poll up to kSpinLimit times (none under the fail_waits test
  // hook); the drain after a failure always polls up to kSpinLimit times
  const int polls = g.fail_waits ? 0 : kSpinLimit;
  // a lane's two row loads keep their column and square sums apart (two
  // shorter dependency chains), added in load order
  double sqk[RPL];
#pragma unroll
  for (int k = 0; k < RPL; ++k) sqk[k] = 0.0;
  for (int64_t p = q0 / n; p * n < q1; ++p) {
    const int64_t row0 = p * kPanelRows;
    double acc[RPL][R];
    TX ur[RPL][R];  // an FP32 plan's entry arithmetic takes u_i in FP32: rounded once per panel
    bool ok[RPL];
#pragma unroll
    for (int k = 0; k < RPL; ++k) {
      const int64_t i = row0 + k * 32 * R + lane * R;
      ok[k] = i < m;
#pragma unroll
      for (int e = 0; e < R; ++e) {
        acc[k][e] = 0.0;
        ur[k][e] = (ok[k] && !zero_g) ? (TX)__ldg(u + i + e) : (TX)0;
      }
    }
    cost.panel(row0, lane, m, ok);
    while (!failed && cons.valid && cons.p == p) {
      const int64_t j = cons.j;
      const int stage = cstage;
      const uint32_t parity = cphase;
      if (!mbar_wait_bounded(bar0 + 8 * stage, parity, polls)) {
        failed = true;
        break;
      }
      const unsigned char* stg = ring + (size_t)stage * L::kStageBytes;
      const TC* sC = reinterpret_cast<const TC*>(stg);
      const TX* sX = reinterpret_cast<const TX*>(stg + L::kCBytes);
      const TX* sXa = reinterpret_cast<const TX*>(stg + L::kCBytes + L::kXBytes);
      const double vj = zero_g ? 0.0 : __ldg(v + j);
      cost.column(j);
      const int64_t base = j * m + row0 + lane * R;
      double csk[RPL];
#pragma unroll
      for (int k = 0; k < RPL; ++k) csk[k] = 0.0;
#pragma unroll
      for (int k = 0; k < RPL; ++k) {
        if (ok[k]) {
          const int r = k * 32 * R + lane * R;
          typename CostReader<CK, R, RPL>::value_t cv[R];
          if constexpr (L::kSq)
            cost.get(0, k, cv);
          else
            vld<TC, R>(sC + r, cv);
          TX xv[R], av[R];
          vld<TX, R>(sX + r, xv);
          if (!first) vld<TX, R>(sXa + r, av);
#pragma unroll
          for (int e = 0; e < R; ++e) {
            double d;
            primal_entry<TX>(widen(cv[e]), ur[k][e], vj, s, nw, aw, zero_g, first, xv[e], av[e], d);
            acc[k][e] += d;
            csk[k] += d;
            add_sq<TX>(sqk[k], d);
          }
          vst<TX, R>(X + base + k * 32 * R, xv);
          vst<TX, R>(Xa + base + k * 32 * R, av);
        }
      }
      double cs = csk[0];
#pragma unroll
      for (int k = 1; k < RPL; ++k) cs += csk[k];
      cs = warp_sum(cs);
      if (lane == 0) B.colpart[p * n + j] = cs;
      __syncwarp();
      ++consumed;
      if (++cstage == S) {
        cstage = 0;
        cphase ^= 1u;
      }
      cons.advance(warp);
      if (prod.valid) {
        if (lane == 0) issue(prod.p, prod.j, stage);
        prod.advance(warp);
        ++issued;
      }
    }
#pragma unroll
    for (int k = 0; k < RPL; ++k)
#pragma unroll
      for (int e = 0; e < R; ++e) red[warp][k * 32 * R + lane * R + e] = acc[k][e];
    __syncthreads();
    for (int t = threadIdx.x; t < kPanelRows; t += kThreads) {
      double s2 = red[0][t];
#pragma unroll
      for (int w = 1; w < kWarps; ++w) s2 += red[w][t];
      B.rowpart[row_slot(cta, p) * kPanelRows + t] = s2;
    }
    __syncthreads();
  }
  if (failed) {
    // drain the copies still in flight (bounded) before the shared memory goes away
    if (lane == 0) atomicExch(&st->kernel_error, 1);
    for (long long c = consumed; c < issued; ++c)
      mbar_wait_bounded(bar0 + 8 * (int)(c % S), (uint32_t)((c / S) & 1));
  }
  double sq = sqk[0];
#pragma unroll
  for (int k = 1; k < RPL; ++k) sq += sqk[k];
  sq = warp_sum(sq);
  if (lane == 0) sqw[warp] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s2 = sqw[0];
#pragma unroll
    for (int w = 1; w < kWarps; ++w) s2 += sqw[w];
    B.sqpart[cta] = s2;
  }
}

// The staged pass never carries the evaluation's plan sums: their six FP64
// accumulators push it past the registers of two CTAs per SM, and the spilling
// variant measured 1.8x slower on B200 than the plain pass, more than the plan
// reads it would save the evaluation (8 B per entry with an FP32 plan).
template <typename TX, int CK>
__global__ void __launch_bounds__(kThreads, 2) k1_primal_staged(Buffers B, Geometry g) {
  pdl_enter();
  k1_primal_staged_impl<TX, CK>(B, g);
}

// Second stage of the row sum of row i / column sum of column j: the partial
// slots added in a fixed order (sum_strided).
__device__ __forceinline__ double finish_row_sum(const Geometry& g, const double* rowpart, int64_t i) {
  const int64_t p = i / kPanelRows, t = i - p * kPanelRows;
  const int64_t lo = cta_of_unit(g, p * g.n), hi = cta_of_unit(g, (p + 1) * g.n - 1);
  // slots row_slot(c, p) = c + p for c = lo..hi are consecutive
  return sum_strided(rowpart + row_slot(lo, p) * kPanelRows + t, hi - lo + 1, kPanelRows);
}
__device__ __forceinline__ double finish_col_sum(const Geometry& g, const double* colpart, int64_t j) {
  return sum_strided(colpart + j, g.panels, g.n);
}

// Stand-alone stage two for pdot_primal_pass_f64: delta row/column sums and
// the sum of squares (one extra CTA).
__global__ void __launch_bounds__(kVecThreads) k_pass_sums(Geometry g, const double* rowpart,
                                                           const double* colpart, const double* sqpart,
                                                           double* drow, double* dcol, double* dsq) {
  const int bid = blockIdx.x;
  if (bid < g.row_blocks) {
    const int64_t i = (int64_t)bid * kVecThreads + threadIdx.x;
    if (i < g.m) drow[i] = finish_row_sum(g, rowpart, i);
  } else if (bid < g.row_blocks + g.col_blocks) {
    const int64_t j = (int64_t)(bid - g.row_blocks) * kVecThreads + threadIdx.x;
    if (j < g.n) dcol[j] = finish_col_sum(g, colpart, j);
  } else if (threadIdx.x < 32) {
    double out[1];
    warp_reduce_partials<1>(sqpart, 0, g.grid, 0u, out);
    if (threadIdx.x == 0) *dsq = out[0];
  }
}

// Block `bid` of the `nblocks` = dual_row_blocks + col_blocks blocks of the
// dual step; the last to finish runs the step control.
__device__ __forceinline__ void k2_dual_body(const Buffers& B, const Geometry& g, const SolveConfig& cfg,
                                             const int bid, const unsigned nblocks) {
  DevState* st = B.st;
  if (st->done | st->numerical_error | st->kernel_error) return;
  const int buf = st->buf;
  const double tau = st->step_size, omega = st->primal_weight, S = st->sum_weights;
  DualArgs A;
  A.first = !(S > 0.0);
  A.tw = __dmul_rn(tau, omega);
  A.nw = A.first ? 1.0 : __ddiv_rn(tau, S);
  A.aw = A.first ? 1.0 : __ddiv_rn(S, __dadd_rn(S, tau));
  double vals[kStepSums] = {0.0, 0.0};
  const int rb = g.dual_row_blocks;
  if (bid < rb && rb == g.row_blocks) {
    const int64_t i = (int64_t)bid * kVecThreads + threadIdx.x;
    if (i < g.m)
      dual_entry(finish_row_sum(g, B.rowpart, i), B.a[i], B.r[buf] + i, B.u[buf] + i, B.r[buf ^ 1] + i,
                 B.u[buf ^ 1] + i, A, vals[0], vals[1]);
  } else if (bid < rb) {
    // a warp per row: lane l adds slots l, l + 32, ... in order, then a fixed
    // shuffle tree; the row's many slots are read in parallel, not in a chain
    const int64_t i = (int64_t)bid * kWarps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i < g.m) {
      const int64_t p = i / kPanelRows, t = i - p * kPanelRows;
      const int64_t lo = cta_of_unit(g, p * g.n), hi = cta_of_unit(g, (p + 1) * g.n - 1);
      const double* q = B.rowpart + row_slot(lo, p) * kPanelRows + t;
      double sd = 0.0;
      for (int64_t c = lane; c <= hi - lo; c += 32) sd += q[c * kPanelRows];
      sd = warp_sum(sd);
      if (lane == 0)
        dual_entry(sd, B.a[i], B.r[buf] + i, B.u[buf] + i, B.r[buf ^ 1] + i, B.u[buf ^ 1] + i, A, vals[0],
                   vals[1]);
    }
  } else {
    const int64_t j = (int64_t)(bid - rb) * kVecThreads + threadIdx.x;
    if (j < g.n)
      dual_entry(finish_col_sum(g, B.colpart, j), B.b[j], B.c[buf] + j, B.v[buf] + j, B.c[buf ^ 1] + j,
                 B.v[buf ^ 1] + j, A, vals[0], vals[1]);
  }
  block_reduce<kStepSums>(vals, 0u, B.steppart + (int64_t)bid * kStepSums);
  if (!elect_last_of(&st->ticket_step, nblocks)) return;
  // warps 0-2 reduce the three partial sets side by side, warp 3 computes the
  // step rule's powers; thread 0 then runs the step control
  __shared__ double fin[2 * kStepSums + 1];
  __shared__ StepPowers pw;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w == 0) {
    double rs[kStepSums];
    warp_reduce_partials<kStepSums>(B.steppart, 0, rb, 0u, rs);
    if (lane == 0) fin[0] = rs[0], fin[1] = rs[1];
  } else if (w == 1) {
    double cs[kStepSums];
    warp_reduce_partials<kStepSums>(B.steppart, rb, g.col_blocks, 0u, cs);
    if (lane == 0) fin[2] = cs[0], fin[3] = cs[1];
  } else if (w == 2) {
    double xs[1];
    warp_reduce_partials<1>(B.sqpart, 0, g.grid, 0u, xs);
    if (lane == 0) fin[4] = xs[0];
  } else if (w == 3 && lane == 0) {
    pw = step_powers(st, cfg);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // interaction = dot(dr, du) + dot(dc, dv); ||[du; dv]||^2
    step_control(st, cfg, fin[0], fin[2], fin[4], fin[1] + fin[3], pw);
    st->ticket_step = 0;
  }
}

__global__ void __launch_bounds__(kVecThreads) k2_dual(Buffers B, Geometry g, SolveConfig cfg) {
  pdl_enter();
  k2_dual_body(B, g, cfg, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Evaluation, matrix part: for the current point (X, G = C - u - v^T, or G = 0
// before the first accepted step) and, when an average exists, the average
// point, the sums <C,X>, ||X||^2, max|X|, ||min(G,0)||^2, max|min(G,0)|
// (src/utils_gpu.jl:84,102-103,39,52,108; src/saddle_point_gpu.jl:313,325).
//
// When the primal pass of the previous loop body already left the plan sums
// (k1_primal_xs: xsums_iter is the previous loop body), only the cost is read
// and only the reduced-cost sums are written; otherwise every sum is computed
// here (the first evaluation, a warm start's initial point, an evaluation
// after a numerical error stopped the step kernels).
//
// The plan and the duals are read through L2 (vldcg, __ldcg): in the
// persistent chunk kernel other CTAs of the same launch wrote them.
template <typename TX, int CK, int R>
__device__ __forceinline__ void k3_eval_body(const Buffers& B, const Geometry& g, const int64_t cta) {
  DevState* st = B.st;
  if (st->done | st->kernel_error) return;
  if (cta == 0 && threadIdx.x == 0) st->eval_t0_ns = globaltimer_ns();
  constexpr int RPL = kPanelRows / (32 * R);
  const int buf = st->buf;
  const bool have_avg = st->avg_count > 0;
  const bool zero_g = st->g_is_zero != 0;
  const bool need_x = st->xsums_iter != st->iteration - 1;
  CostReader<CK, R, RPL> cost(B.cost, (float)st->cost_scale);
  const TX* __restrict__ X = static_cast<const TX*>(B.X[buf]);
  const TX* __restrict__ Xa = static_cast<const TX*>(B.X[buf ^ 1]);
  const double* __restrict__ u = B.u[buf];
  const double* __restrict__ v = B.v[buf];
  const double* __restrict__ ua = B.u[buf ^ 1];
  const double* __restrict__ va = B.v[buf ^ 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t m = g.m, n = g.n;
  const int64_t q0 = unit_begin(g, cta), q1 = unit_begin(g, cta + 1);
  double acc[kEvalSums];
#pragma unroll
  for (int k = 0; k < kEvalSums; ++k) acc[k] = 0.0;
  for (int64_t p = q0 / n; p * n < q1; ++p) {
    const int64_t jb = (q0 > p * n ? q0 : p * n) - p * n;
    const int64_t je = (q1 < (p + 1) * n ? q1 : (p + 1) * n) - p * n;
    const int64_t row0 = p * kPanelRows;
    double ur[RPL][R], uar[RPL][R];
    bool ok[RPL];
#pragma unroll
    for (int k = 0; k < RPL; ++k) {
      const int64_t i = row0 + k * 32 * R + lane * R;
      ok[k] = i < m;
#pragma unroll
      for (int e = 0; e < R; ++e) {
        ur[k][e] = ok[k] ? __ldcg(u + i + e) : 0.0;
        uar[k][e] = (ok[k] && have_avg) ? __ldcg(ua + i + e) : 0.0;
      }
    }
    cost.panel(row0, lane, m, ok);
    for (int64_t j = jb + warp; j < je; j += kWarps) {
      const double vj = __ldcg(v + j);
      const double vaj = have_avg ? __ldcg(va + j) : 0.0;
      cost.column(j);
      const int64_t base = j * m + row0 + lane * R;
      typename CostReader<CK, R, RPL>::value_t cv[RPL][R];
      TX xv[RPL][R], av[RPL][R];
#pragma unroll
      for (int k = 0; k < RPL; ++k) {
        if (ok[k]) {
          const int64_t idx = base + k * 32 * R;
          cost.get(idx, k, cv[k]);
          if (need_x) {
            vldcg<TX, R>(X + idx, xv[k]);
            if (have_avg) vldcg<TX, R>(Xa + idx, av[k]);
          }
        }
      }
#pragma unroll
      for (int k = 0; k < RPL; ++k) {
        if (ok[k]) {
#pragma unroll
          for (int e = 0; e < R; ++e) {
            const double c = widen(cv[k][e]);
            const double gg = zero_g ? 0.0 : __dsub_rn(__dsub_rn(c, ur[k][e]), vj);
            const double mg = neg_part(gg);
            if (need_x) {
              const double x = widen(xv[k][e]);
              acc[E_DOT] += c * x;
              acc[E_SQX] += x * x;
              acc[E_MAXX] = nanmax(acc[E_MAXX], fabs(x));
            }
            acc[E_SQG] += mg * mg;
            acc[E_MAXG] = nanmax(acc[E_MAXG], mg);
            if (have_avg) {
              const double ga = __dsub_rn(__dsub_rn(c, uar[k][e]), vaj);
              const double mga = neg_part(ga);
              if (need_x) {
                const double xa = widen(av[k][e]);
                acc[E_AVG + E_DOT] += c * xa;
                acc[E_AVG + E_SQX] += xa * xa;
                acc[E_AVG + E_MAXX] = nanmax(acc[E_AVG + E_MAXX], fabs(xa));
              }
              acc[E_AVG + E_SQG] += mga * mga;
              acc[E_AVG + E_MAXG] = nanmax(acc[E_AVG + E_MAXG], mga);
            }
          }
        }
      }
    }
  }
  if (need_x) {
    block_reduce<kEvalSums>(acc, kEvalMaxMask, B.evpart + cta * kEvalSums);
  } else {
    // the plan sums are already in place; the same reduction of the rest
    __shared__ double gout[4];
    double gacc[4] = {acc[E_SQG], acc[E_MAXG], acc[E_AVG + E_SQG], acc[E_AVG + E_MAXG]};
    block_reduce<4>(gacc, (1u << 1) | (1u << 3), gout);
    if (threadIdx.x == 0) {
      double* out = B.evpart + cta * kEvalSums;
      out[E_SQG] = gout[0];
      out[E_MAXG] = gout[1];
      out[E_AVG + E_SQG] = gout[2];
      out[E_AVG + E_MAXG] = gout[3];
    }
  }
}

template <typename TX, int CK, int R>
__global__ void __launch_bounds__(kThreads, 2) k3_eval(Buffers B, Geometry g) {
  pdl_enter();
  k3_eval_body<TX, CK, R>(B, g, blockIdx.x);
}

// start_only: the evaluation of a warm start's initial point, run once after
// k0_init; its last CTA records the point as the last restart point
// (record_start_point) and takes no other step of the evaluation block.
// Block `bid` of the `nblocks` = row_blocks + col_blocks blocks.
__device__ __forceinline__ void k4_eval_body(const Buffers& B, const Geometry& g, const SolveConfig& cfg,
                                             const int start_only, const int bid, const unsigned nblocks) {
  DevState* st = B.st;
  if (st->done | st->kernel_error) return;
  const int buf = st->buf;
  const bool have_avg = st->avg_count > 0;
  double acc[kVecSums];
#pragma unroll
  for (int k = 0; k < kVecSums; ++k) acc[k] = 0.0;
  const bool is_row = bid < g.row_blocks;
  const int64_t idx = (int64_t)(is_row ? bid : bid - g.row_blocks) * kVecThreads + threadIdx.x;
  const int64_t len = is_row ? g.m : g.n;
  if (idx < len) {
    const double dist = is_row ? B.a[idx] : B.b[idx];
    const double sc = (is_row ? B.r[buf] : B.c[buf])[idx];
    const double dc = (is_row ? B.u[buf] : B.v[buf])[idx];
    const double res = dist - sc;
    acc[V_SQRES] = res * res;
    acc[V_MAXRES] = fabs(res);
    acc[V_DOT] = dist * dc;
    acc[V_SQDUAL] = dc * dc;
    acc[V_MAXDUAL] = fabs(dc);
    if (have_avg) {
      const double sa = (is_row ? B.r[buf ^ 1] : B.c[buf ^ 1])[idx];
      const double da = (is_row ? B.u[buf ^ 1] : B.v[buf ^ 1])[idx];
      const double ra = dist - sa;
      acc[V_AVG + V_SQRES] = ra * ra;
      acc[V_AVG + V_MAXRES] = fabs(ra);
      acc[V_AVG + V_DOT] = dist * da;
      acc[V_AVG + V_SQDUAL] = da * da;
      acc[V_AVG + V_MAXDUAL] = fabs(da);
    }
  }
  block_reduce<kVecSums>(acc, kVecMaxMask, B.vecpart + (int64_t)bid * kVecSums);
  if (!elect_last_of(&st->ticket_eval, nblocks)) return;
  // warps 0-2 reduce the three partial sets side by side
  __shared__ double fin[kEvalSums + 2 * kVecSums];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w == 0) {
    double E[kEvalSums];
    warp_reduce_partials<kEvalSums>(B.evpart, 0, g.grid, kEvalMaxMask, E);
    if (lane == 0)
      for (int k = 0; k < kEvalSums; ++k) fin[k] = E[k];
  } else if (w == 1) {
    double R[kVecSums];
    warp_reduce_partials<kVecSums>(B.vecpart, 0, g.row_blocks, kVecMaxMask, R);
    if (lane == 0)
      for (int k = 0; k < kVecSums; ++k) fin[kEvalSums + k] = R[k];
  } else if (w == 2) {
    double Cc[kVecSums];
    warp_reduce_partials<kVecSums>(B.vecpart, g.row_blocks, g.col_blocks, kVecMaxMask, Cc);
    if (lane == 0)
      for (int k = 0; k < kVecSums; ++k) fin[kEvalSums + kVecSums + k] = Cc[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double* E = fin;
    const double* R = fin + kEvalSums;
    const double* Cc = fin + kEvalSums + kVecSums;
    const PointSums cur = point_sums(E, R, Cc, 0);
    const PointSums avg = point_sums(E, R, Cc, E_AVG);
    if (start_only)
      record_start_point(st, cur);
    else
      eval_control(st, cfg, cur, avg, B.ring, B.ring_cap);
    st->ticket_eval = 0;
  }
}

__global__ void __launch_bounds__(kVecThreads) k4_eval(Buffers B, Geometry g, SolveConfig cfg, int start_only) {
  pdl_enter();
  k4_eval_body(B, g, cfg, start_only, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------
// Persistent chunk: one cooperative launch runs a regular chunk of loop bodies
// (the evaluation, then `steps` iterations of primal pass and dual step) with
// grid barriers between the phases instead of kernel boundaries: for small
// problems the launches, the kernel tails and the dual step's chains of L2
// round trips, not the bytes, set the time of an iteration.
//
// Every phase runs the body of its own kernel over the same CTA ranges of the
// matrix passes (physical CTA b takes ranges b, b + gridDim.x, ...) and the same
// blocks of the vector passes, with the same last-block elections, so the
// results are bit-identical to the launches the chunk replaces. Each CTA reads
// the solver state after the same barrier, so all of them leave together once
// the solve is done. A barrier whose poll runs out records kernel_error and the
// CTA leaves; the others' polls see the error and leave too.
static_assert(kThreads == kVecThreads, "the chunk kernel runs the vector passes' blocks on its CTAs");
// Build knobs of the chunk kernel: resident CTAs per SM it is compiled for, and
// whether the phases are inlined (1) or calls (0). The default, 1 CTA per SM
// with inlined phases, measured fastest of the four on B200 (no spills; each
// CTA runs two of the matrix passes' CTA ranges).
#ifndef PDOT_CHUNK_MIN_BLOCKS
#define PDOT_CHUNK_MIN_BLOCKS 1
#endif
#ifndef PDOT_CHUNK_INLINE
#define PDOT_CHUNK_INLINE 1
#endif
#if PDOT_CHUNK_INLINE
#define PDOT_CHUNK_PHASE __device__ __forceinline__
#else
#define PDOT_CHUNK_PHASE __device__ __noinline__
#endif
template <typename TX, int CK, int R, bool XS>
PDOT_CHUNK_PHASE void chunk_primal(const Buffers& B, const Geometry& g, int64_t cta) {
  k1_primal_impl<TX, CK, R, XS>(B, g, cta);
}
template <typename TX, int CK, int R>
PDOT_CHUNK_PHASE void chunk_eval_matrix(const Buffers& B, const Geometry& g, int64_t cta) {
  k3_eval_body<TX, CK, R>(B, g, cta);
}
PDOT_CHUNK_PHASE void chunk_eval_vector(const Buffers& B, const Geometry& g, const SolveConfig& cfg, int bid,
                                               unsigned nblocks) {
  k4_eval_body(B, g, cfg, 0, bid, nblocks);
}
PDOT_CHUNK_PHASE void chunk_dual(const Buffers& B, const Geometry& g, const SolveConfig& cfg, int bid,
                                        unsigned nblocks) {
  k2_dual_body(B, g, cfg, bid, nblocks);
}

template <typename TX, int CK, int R>
__global__ void __launch_bounds__(kThreads, PDOT_CHUNK_MIN_BLOCKS)
    k_chunk(Buffers B, Geometry g, SolveConfig cfg, int steps) {
  DevState* st = B.st;
  const unsigned P = gridDim.x;
  auto sync = [&]() -> bool {
    if (grid_barrier(&st->bar_count, &st->bar_gen, P, &st->kernel_error)) return true;
    if (threadIdx.x == 0) atomicExch(&st->kernel_error, 1);
    return false;
  };
  const unsigned vb = (unsigned)(g.row_blocks + g.col_blocks);
  const unsigned db = (unsigned)(g.dual_row_blocks + g.col_blocks);
  for (int64_t c = blockIdx.x; c < g.grid; c += P) {
    chunk_eval_matrix<TX, CK, R>(B, g, c);
    __syncthreads();
  }
  if (!sync()) return;
  for (unsigned b = blockIdx.x; b < vb; b += P) {
    chunk_eval_vector(B, g, cfg, (int)b, vb);
    __syncthreads();
  }
  if (!sync()) return;
  for (int k = 0; k < steps; ++k) {
    if (st->done | st->numerical_error) return;  // the same value in every CTA
    const bool xs = k == steps - 1;               // the next chunk starts with an evaluation
    for (int64_t c = blockIdx.x; c < g.grid; c += P) {
      if (xs)
        chunk_primal<TX, CK, R, true>(B, g, c);
      else
        chunk_primal<TX, CK, R, false>(B, g, c);
      __syncthreads();
    }
    if (!sync()) return;
    for (unsigned b = blockIdx.x; b < db; b += P) {
      chunk_dual(B, g, cfg, (int)b, db);
      __syncthreads();
    }
    if (!sync()) return;
  }
}

// ---------------------------------------------------------------------------
// Start of a solve: cached_ot_info (src/termination.jl:94-101) on the device,
// the initial step size and primal weight (src/solver_gpu.jl:476-496,
// src/saddle_point_gpu.jl:848-866) and the initial last-restart record (the
// zero point, src/saddle_point_gpu.jl:371-393; after a warm start the host
// replaces it with the start point's, see record_start_point).
template <typename TX, int CK, int R>
__global__ void __launch_bounds__(kThreads, 2) k0_init(Buffers B, Geometry g, SolveConfig cfg) {
  constexpr int RPL = kPanelRows / (32 * R);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t m = g.m, n = g.n;
  const int64_t cta = blockIdx.x;
  const int64_t q0 = unit_begin(g, cta), q1 = unit_begin(g, cta + 1);
  // the coordinate cost is reduced unscaled; the scale is known only at the end
  CostReader<CK, R, RPL> cost(B.cost, 1.0f);
  double acc[kNormSums] = {0.0, 0.0};  // sum C^2, max |C|
  for (int64_t p = q0 / n; p * n < q1; ++p) {
    const int64_t jb = (q0 > p * n ? q0 : p * n) - p * n;
    const int64_t je = (q1 < (p + 1) * n ? q1 : (p + 1) * n) - p * n;
    const int64_t row0 = p * kPanelRows;
    bool ok[RPL];
#pragma unroll
    for (int k = 0; k < RPL; ++k) ok[k] = row0 + k * 32 * R + lane * R < m;
    cost.panel(row0, lane, m, ok);
    for (int64_t j = jb + warp; j < je; j += kWarps) {
      cost.column(j);
      const int64_t base = j * m + row0 + lane * R;
#pragma unroll
      for (int k = 0; k < RPL; ++k) {
        if (ok[k]) {
          typename CostReader<CK, R, RPL>::value_t cv[R];
          cost.get(base + k * 32 * R, k, cv);
#pragma unroll
          for (int e = 0; e < R; ++e) {
            const double c = widen(cv[e]);
            acc[0] += c * c;
            acc[1] = nanmax(acc[1], fabs(c));
          }
        }
      }
    }
  }
  block_reduce<kNormSums>(acc, 2u, B.evpart + cta * kNormSums);
  DevState* st = B.st;
  if (!elect_last_cta(&st->ticket_init)) return;
  // the marginals' norms, by the whole CTA in a fixed order
  double vacc[2] = {0.0, 0.0};
  for (int64_t i = threadIdx.x; i < m + n; i += kThreads) {
    const double x = i < m ? B.a[i] : B.b[i - m];
    vacc[0] += x * x;
    vacc[1] = nanmax(vacc[1], fabs(x));
  }
  __shared__ double vsum[2];
  block_reduce<2>(vacc, 2u, vsum);
  if (threadIdx.x < 32) {
    double nc[kNormSums];
    warp_reduce_partials<kNormSums>(B.evpart, 0, g.grid, 2u, nc);
    if (threadIdx.x == 0) {
      double scale = 1.0;
      if (is_point_cost(CK)) {
        scale = cfg.cost_scale > 0.0 ? cfg.cost_scale : (nc[1] > 0.0 ? 1.0 / nc[1] : 1.0);
        nc[0] *= scale * scale;
        nc[1] *= scale;
      }
      st->cost_scale = scale;
      st->linf_obj = nc[1];
      st->l2_obj = sqrt(nc[0]);
      st->linf_rhs = vsum[1];
      st->l2_rhs = sqrt(vsum[0]);
      st->step_size = cfg.adaptive ? 1.0 : (1.0 - 0.2) / sqrt((double)(m + n));
      if (cfg.scale_invariant_initial_primal_weight) {
        const double rhs = sqrt(1.0) * st->l2_rhs, obj = sqrt(1.0) * st->l2_obj;
        st->primal_weight = (obj > 0.0 && rhs > 0.0) ? cfg.primal_importance * (obj / rhs) : cfg.primal_importance;
      } else {
        st->primal_weight = cfg.primal_importance;
      }
      if (cfg.warm_start && cfg.warm_primal_weight > 0.0) st->primal_weight = cfg.warm_primal_weight;
      st->kkt_passes = 0.0;
      st->sum_weights = 0.0;
      st->avg_count = 0;
      st->total_iters = 0;
      st->iteration = 1;
      st->last_rp = st->l2_rhs;  // ||[a - 0; b - 0]||
      st->last_rd = 0.0;
      st->last_gap = 0.0;
      st->last_xnorm = 0.0;
      st->last_ynorm = 0.0;
      st->ratio_last_trial = 1.0;
      st->last_restart_length = 1;
      st->pdist = st->ddist = 0.0;
      st->numerical_error = 0;
      // the stored gradient starts at 0 (src/solver_gpu.jl:434); after a warm
      // start it is C - u - v from the first step on
      st->g_is_zero = cfg.warm_start ? 0 : 1;
      st->buf = 0;
      st->out_current = 1;
      st->num_stats = 0;
      st->primal_passes = 0;
      st->fresh_passes = 0;
      st->xsums_iter = -1;
      st->eval_time_sec = 0.0;
      st->done = 0;
      st->termination_reason = 0;
      // Non-finite data cannot be solved; the reference would iterate on NaNs.
      if (!(isfinite(st->l2_obj) && isfinite(st->l2_rhs) && isfinite(st->linf_obj))) {
        st->done = 1;
        st->termination_reason = PDOT_TERMINATION_REASON_INVALID_PROBLEM;
      }
      st->t_start_ns = globaltimer_ns();
      st->ticket_init = 0;
    }
  }
}

template <typename K>
int blocks_per_sm(K kernel) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, kThreads, 0) != cudaSuccess || nb < 1) nb = 1;
  return nb;
}

// FP32 storage of an FP64 cost, and an FP32 plan widened for the caller.
__global__ void k_convert_cost(const double* __restrict__ src, void* __restrict__ dst, int kind, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    if (kind == PDOT_COST_F32)
      static_cast<float*>(dst)[i] = __double2float_rn(src[i]);
    else
      static_cast<__nv_bfloat16*>(dst)[i] = __double2bfloat16(src[i]);
  }
}
__global__ void k_widen(const float* __restrict__ src, double* __restrict__ dst, size_t count) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

}  // namespace

// Expands to the kernel variant of geometry `g`:
//   plan FP64 + cost FP64, or plan FP32 + cost FP32 / BF16 / coordinates,
//   each with the 16-byte load path (R = 16 / sizeof(plan)) or R = 1.
#define PDOT_VARIANT(g, KERNEL, LAUNCH)                                                   \
  do {                                                                                     \
    if (!(g).plan_f32) {                                                                   \
      if ((g).vec > 1) { auto kfn = KERNEL<double, PDOT_COST_F64, 2>; LAUNCH; }            \
      else { auto kfn = KERNEL<double, PDOT_COST_F64, 1>; LAUNCH; }                        \
    } else if ((g).cost_kind == PDOT_COST_F32) {                                           \
      if ((g).vec > 1) { auto kfn = KERNEL<float, PDOT_COST_F32, 4>; LAUNCH; }             \
      else { auto kfn = KERNEL<float, PDOT_COST_F32, 1>; LAUNCH; }                         \
    } else if ((g).cost_kind == PDOT_COST_BF16) {                                          \
      if ((g).vec > 1) { auto kfn = KERNEL<float, PDOT_COST_BF16, 4>; LAUNCH; }            \
      else { auto kfn = KERNEL<float, PDOT_COST_BF16, 1>; LAUNCH; }                        \
    } else if ((g).cost_kind == kCostSqBase + 1) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostSqBase + 1, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostSqBase + 1, 1>; LAUNCH; }                       \
    } else if ((g).cost_kind == kCostSqBase + 2) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostSqBase + 2, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostSqBase + 2, 1>; LAUNCH; }                       \
    } else if ((g).cost_kind == kCostSqBase + 3) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostSqBase + 3, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostSqBase + 3, 1>; LAUNCH; }                       \
    } else if ((g).cost_kind == kCostSqBase + 4) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostSqBase + 4, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostSqBase + 4, 1>; LAUNCH; }                       \
    } else if ((g).cost_kind == kCostL1Base + 1) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostL1Base + 1, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostL1Base + 1, 1>; LAUNCH; }                       \
    } else if ((g).cost_kind == kCostL1Base + 2) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostL1Base + 2, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostL1Base + 2, 1>; LAUNCH; }                       \
    } else if ((g).cost_kind == kCostL1Base + 3) {                                         \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostL1Base + 3, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostL1Base + 3, 1>; LAUNCH; }                       \
    } else {                                                                               \
      if ((g).vec > 1) { auto kfn = KERNEL<float, kCostL1Base + 4, 4>; LAUNCH; }           \
      else { auto kfn = KERNEL<float, kCostL1Base + 4, 1>; LAUNCH; }                       \
    }                                                                                      \
  } while (0)

// The 16-byte variants only (g.vec > 1): the persistent chunk kernel.
#define PDOT_VEC_VARIANT(g, KERNEL, LAUNCH)  \
  do {  \
    if (!(g).plan_f32) { auto kfn = KERNEL<double, PDOT_COST_F64, 2>; LAUNCH; }  \
    else if ((g).cost_kind == PDOT_COST_F32) { auto kfn = KERNEL<float, PDOT_COST_F32, 4>; LAUNCH; }  \
    else if ((g).cost_kind == PDOT_COST_BF16) { auto kfn = KERNEL<float, PDOT_COST_BF16, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostSqBase + 1) { auto kfn = KERNEL<float, kCostSqBase + 1, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostSqBase + 2) { auto kfn = KERNEL<float, kCostSqBase + 2, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostSqBase + 3) { auto kfn = KERNEL<float, kCostSqBase + 3, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostSqBase + 4) { auto kfn = KERNEL<float, kCostSqBase + 4, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostL1Base + 1) { auto kfn = KERNEL<float, kCostL1Base + 1, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostL1Base + 2) { auto kfn = KERNEL<float, kCostL1Base + 2, 4>; LAUNCH; }  \
    else if ((g).cost_kind == kCostL1Base + 3) { auto kfn = KERNEL<float, kCostL1Base + 3, 4>; LAUNCH; }  \
    else { auto kfn = KERNEL<float, kCostL1Base + 4, 4>; LAUNCH; }  \
  } while (0)

// The staged fused pass exists for the 16-byte path of every variant
// (KERNEL: k1_primal_staged or k1_primal_staged_xs).
#define PDOT_STAGED_VARIANT(g, KERNEL, LAUNCH)                                                      \
  do {                                                                                            \
    if (!(g).plan_f32) { auto kfn = KERNEL<double, PDOT_COST_F64>;                               \
      constexpr int smem = StagedLayout<double, PDOT_COST_F64>::kSmem; LAUNCH; }                 \
    else if ((g).cost_kind == PDOT_COST_F32) { auto kfn = KERNEL<float, PDOT_COST_F32>;           \
      constexpr int smem = StagedLayout<float, PDOT_COST_F32>::kSmem; LAUNCH; }                  \
    else if ((g).cost_kind == PDOT_COST_BF16) { auto kfn = KERNEL<float, PDOT_COST_BF16>;         \
      constexpr int smem = StagedLayout<float, PDOT_COST_BF16>::kSmem; LAUNCH; }                 \
    else if ((g).cost_kind == kCostSqBase + 1) { auto kfn = KERNEL<float, kCostSqBase + 1>;       \
      constexpr int smem = StagedLayout<float, kCostSqBase + 1>::kSmem; LAUNCH; }                \
    else if ((g).cost_kind == kCostSqBase + 2) { auto kfn = KERNEL<float, kCostSqBase + 2>;       \
      constexpr int smem = StagedLayout<float, kCostSqBase + 2>::kSmem; LAUNCH; }                \
    else if ((g).cost_kind == kCostSqBase + 3) { auto kfn = KERNEL<float, kCostSqBase + 3>;       \
      constexpr int smem = StagedLayout<float, kCostSqBase + 3>::kSmem; LAUNCH; }                \
    else if ((g).cost_kind == kCostSqBase + 4) { auto kfn = KERNEL<float, kCostSqBase + 4>;       \
      constexpr int smem = StagedLayout<float, kCostSqBase + 4>::kSmem; LAUNCH; }                \
    else if ((g).cost_kind == kCostL1Base + 1) { auto kfn = KERNEL<float, kCostL1Base + 1>;       \
      constexpr int smem = StagedLayout<float, kCostL1Base + 1>::kSmem; LAUNCH; }                \
    else if ((g).cost_kind == kCostL1Base + 2) { auto kfn = KERNEL<float, kCostL1Base + 2>;       \
      constexpr int smem = StagedLayout<float, kCostL1Base + 2>::kSmem; LAUNCH; }                \
    else if ((g).cost_kind == kCostL1Base + 3) { auto kfn = KERNEL<float, kCostL1Base + 3>;       \
      constexpr int smem = StagedLayout<float, kCostL1Base + 3>::kSmem; LAUNCH; }                \
    else { auto kfn = KERNEL<float, kCostL1Base + 4>;                                             \
      constexpr int smem = StagedLayout<float, kCostL1Base + 4>::kSmem; LAUNCH; }                \
  } while (0)

Geometry make_geometry(int64_t m, int64_t n, int vec_ok, int device, int plan_f32, int cost_kind, int staged_ok) {
  Geometry g;
  g.m = m;
  g.n = n;
  g.plan_f32 = plan_f32 ? 1 : 0;
  g.cost_kind = cost_kind;
  g.panels = (m + kPanelRows - 1) / kPanelRows;
  g.units = g.panels * n;
  const int R = g.plan_f32 ? 4 : 2;
  g.vec = (vec_ok && (m % R == 0)) ? R : 1;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  // The staged pass needs 16-byte aligned segments: the vector path, and for a
  // BF16 cost m divisible by 8 (8 two-byte entries per 16 bytes). staged_ok:
  // 0 never, 1 always, 2 where it measured faster on B200 (BF16 and coordinate
  // costs, whose direct loads keep too few bytes in flight per warp).
  const bool want = staged_ok == 1 || (staged_ok == 2 && (cost_kind == PDOT_COST_BF16 || is_point_cost(cost_kind)));
  g.tma = (want && g.vec > 1 && !(cost_kind == PDOT_COST_BF16 && m % 8 != 0)) ? 1 : 0;
  g.tma_smem = 0;
  g.fail_waits = 0;
  int occ = 1;
  if (g.tma) {
    PDOT_STAGED_VARIANT(g, k1_primal_staged, {
      g.tma_smem = smem;
      if (cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kThreads, smem) != cudaSuccess || occ < 1) {
        cudaGetLastError();
        g.tma = 0;
        occ = 1;
      }
    });
  }
  if (!g.tma) PDOT_VARIANT(g, k1_primal, occ = blocks_per_sm(kfn));
  int64_t grid = (int64_t)sms * occ;
  if (grid > g.units) grid = g.units;
  g.grid = (int32_t)grid;
  // the persistent chunk kernel: the direct 16-byte passes only, as many CTAs
  // as stay co-resident (at most one per CTA range)
  g.chunk_ctas = 0;
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!g.tma && g.vec > 1 && coop) {
    int cocc = 0;
    PDOT_VEC_VARIANT(g, k_chunk, {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cocc, kfn, kThreads, 0) != cudaSuccess) cocc = 0;
    });
    cudaGetLastError();
    const int64_t c = (int64_t)sms * cocc;
    g.chunk_ctas = (int32_t)(c < g.grid ? c : g.grid);
  }
  g.row_blocks = (int32_t)((m + kVecThreads - 1) / kVecThreads);
  g.col_blocks = (int32_t)((n + kVecThreads - 1) / kVecThreads);
  // the most CTA slots one panel's row partials can lie in
  const int64_t slots = (g.grid + g.panels - 1) / g.panels + 1;
  g.dual_row_blocks = slots >= kDualWarpSlots ? (int32_t)((m + kWarps - 1) / kWarps) : g.row_blocks;
  return g;
}

size_t workspace_doubles(const Geometry& g) {
  const size_t vb = (size_t)g.row_blocks + g.col_blocks;
  const size_t db = (size_t)g.dual_row_blocks + g.col_blocks;
  return ((size_t)g.grid + g.panels) * kPanelRows  // rowpart
         + (size_t)g.panels * g.n                   // colpart
         + (size_t)g.grid                           // sqpart
         + db * kStepSums                           // steppart
         + (size_t)g.grid * kEvalSums               // evpart
         + vb * kVecSums;                           // vecpart
}

cudaError_t launch_init(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s) {
  PDOT_VARIANT(g, k0_init, (kfn<<<g.grid, kThreads, 0, s>>>(B, g, cfg)));
  return cudaGetLastError();
}

// The loop's kernels are launched with programmatic dependent launch (pdl_launch).
cudaError_t launch_primal(const Buffers& B, const Geometry& g, cudaStream_t s, int xsums) {
  cudaError_t e = cudaSuccess;
  if (g.tma)
    PDOT_STAGED_VARIANT(g, k1_primal_staged, (e = pdl_launch(kfn, dim3((unsigned)g.grid), dim3(kThreads), smem, s, B, g)));
  else if (xsums)
    PDOT_VARIANT(g, k1_primal_xs, (e = pdl_launch(kfn, dim3((unsigned)g.grid), dim3(kThreads), 0, s, B, g)));
  else
    PDOT_VARIANT(g, k1_primal, (e = pdl_launch(kfn, dim3((unsigned)g.grid), dim3(kThreads), 0, s, B, g)));
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_dual(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s) {
  const cudaError_t e =
      pdl_launch(k2_dual, dim3((unsigned)(g.dual_row_blocks + g.col_blocks)), dim3(kVecThreads), 0, s, B, g, cfg);
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_step(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s, int xsums) {
  cudaError_t e = launch_primal(B, g, s, xsums);
  if (e != cudaSuccess) return e;
  return launch_dual(B, g, cfg, s);
}

cudaError_t launch_chunk(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s,
                         int steps) {
  if (g.chunk_ctas < 1) return cudaErrorNotSupported;
  Buffers b = B;
  Geometry gg = g;
  SolveConfig c = cfg;
  void* args[] = {&b, &gg, &c, &steps};
  cudaError_t e = cudaSuccess;
  PDOT_VEC_VARIANT(g, k_chunk,
                   (e = cudaLaunchCooperativeKernel((const void*)kfn, dim3(g.chunk_ctas), dim3(kThreads), args, 0, s)));
  return e;
}

cudaError_t launch_eval(const Buffers& B, const Geometry& g, const SolveConfig& cfg, cudaStream_t s,
                        int start_only) {
  cudaError_t e = cudaSuccess;
  PDOT_VARIANT(g, k3_eval, (e = pdl_launch(kfn, dim3((unsigned)g.grid), dim3(kThreads), 0, s, B, g)));
  if (e != cudaSuccess) return e;
  e = pdl_launch(k4_eval, dim3((unsigned)(g.row_blocks + g.col_blocks)), dim3(kVecThreads), 0, s, B, g, cfg,
                 start_only);
  return e != cudaSuccess ? e : cudaGetLastError();
}

cudaError_t launch_primal_pass(const Geometry& g, const double* C, double* X, double* Xa, const double* u,
                               const double* v, double step_over_weight, double avg_new_weight,
                               double avg_scale, int flags, double* drow, double* dcol, double* dsq,
                               double* work, cudaStream_t s) {
  double* rowpart = work;
  double* colpart = rowpart + ((size_t)g.grid + g.panels) * kPanelRows;
  double* sqpart = colpart + (size_t)g.panels * g.n;
  if (g.vec > 1)
    k1_primal_args<2><<<g.grid, kThreads, 0, s>>>(C, X, Xa, u, v, step_over_weight, avg_new_weight, avg_scale,
                                                  flags, colpart, rowpart, sqpart, g);
  else
    k1_primal_args<1><<<g.grid, kThreads, 0, s>>>(C, X, Xa, u, v, step_over_weight, avg_new_weight, avg_scale,
                                                  flags, colpart, rowpart, sqpart, g);
  k_pass_sums<<<g.row_blocks + g.col_blocks + 1, kVecThreads, 0, s>>>(g, rowpart, colpart, sqpart, drow, dcol,
                                                                      dsq);
  return cudaGetLastError();
}

cudaError_t launch_convert_cost(const double* src, void* dst, int cost_kind, size_t count, cudaStream_t s) {
  k_convert_cost<<<4 * 148, 256, 0, s>>>(src, dst, cost_kind, count);
  return cudaGetLastError();
}

cudaError_t launch_widen(const float* src, double* dst, size_t count, cudaStream_t s) {
  k_widen<<<4 * 148, 256, 0, s>>>(src, dst, count);
  return cudaGetLastError();
}

}  // namespace pdot
