// pdot_noalloc.cu — the fused primal pass for callers that cannot allocate.
//
// pdot_primal_pass_f64 needs scratch for its two-stage reductions and takes it
// from a workspace the caller allocates. Some callers cannot provide one and
// cannot let a library call cudaMalloc either: a host framework that owns the
// whole device-memory budget and serves every buffer from its own pool, or a
// latency-critical loop where cudaMalloc's implicit device synchronisation, and
// its chance of failing under fragmentation in the middle of a run, are not
// acceptable. pdot_primal_pass_f64_noalloc serves them: its scratch is a fixed
// array compiled into this library, so a call allocates nothing.
//
// The array (kScratchBytes = 16 MiB) is part of the library's device image:
// every GPU that loads it holds the 16 MiB until the process exits. Host code
// cannot hand the array's name to a kernel (on the host it only names a
// stand-in, not device memory), so every call looks up the array's device
// address on the current device with cudaGetSymbolAddress (cheap once the
// module is loaded, and never stale, even after a cudaDeviceReset reloads
// it). The first call on a device loads the module there: make that first
// call before any stream capture. All calls on a device share the array and it
// keeps the last call's contents; nothing needs clearing, because the second
// stage reads only partial slots the first stage of the same call wrote. Calls
// that overlap on the GPU (different streams, or another host thread) race on
// the array and must be serialised by the caller.
#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "pdot_common.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(16) << 20;
constexpr size_t kScratchDoubles = kScratchBytes / sizeof(double);

static __device__ __align__(256) double g_pass_scratch[kScratchDoubles];

// Device address of g_pass_scratch on the current device.
cudaError_t scratch_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_pass_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<double*>(p);
  return cudaSuccess;
}

int report(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int report(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  pdot::set_last_error(buf);
  return code;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

extern "C" int pdot_primal_pass_f64_noalloc(int64_t m, int64_t n, const double* cost, double* primal,
                                            double* primal_avg, const double* dual_source,
                                            const double* dual_target, double step_over_weight,
                                            double avg_new_weight, double avg_scale, int32_t flags,
                                            double* delta_row_sum, double* delta_col_sum,
                                            double* delta_sq_norm, void* stream) {
  pdot::set_last_error("");
  if (m < 1 || n < 1) return report(PDOT_ERR_INVALID_ARGUMENT, "empty matrix");
  if (!cost || !primal || !primal_avg || !dual_source || !dual_target || !delta_row_sum || !delta_col_sum ||
      !delta_sq_norm)
    return report(PDOT_ERR_INVALID_ARGUMENT, "null pointer argument");
  if (primal == primal_avg) return report(PDOT_ERR_INVALID_ARGUMENT, "primal and primal_avg must not alias");
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return report(PDOT_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  const int vec_ok = aligned16(cost) && aligned16(primal) && aligned16(primal_avg);
  const pdot::Geometry g = pdot::make_geometry(m, n, vec_ok, device);
  const size_t need = pdot::pass_scratch_doubles(g);
  if (need > kScratchDoubles)
    return report(PDOT_ERR_TOO_LARGE,
                  "a %lld x %lld pass needs %zu bytes of scratch; the fixed scratch holds %zu bytes "
                  "(use pdot_primal_pass_f64 with a workspace)",
                  (long long)m, (long long)n, need * sizeof(double), kScratchBytes);
  double* scratch = nullptr;
  e = scratch_address(&scratch);
  if (e != cudaSuccess) return report(PDOT_ERR_CUDA, "cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
  e = pdot::launch_primal_pass(g, cost, primal, primal_avg, dual_source, dual_target, step_over_weight,
                               avg_new_weight, avg_scale, flags, delta_row_sum, delta_col_sum, delta_sq_norm,
                               scratch, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return report(PDOT_ERR_CUDA, "launch failed: %s", cudaGetErrorString(e));
  return PDOT_OK;
}
