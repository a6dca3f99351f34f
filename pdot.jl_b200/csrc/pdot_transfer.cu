// pdot_transfer.cu — large copies between the caller's host arrays and the
// device (the cost matrix in, the plan out; src/io.jl:18-53 in the reference).
//
// Page-locked host memory (cudaMallocHost, cudaHostRegister, a pinned torch
// tensor) is copied by one DMA. Pageable memory — a Julia Array, a numpy array —
// would make the driver stage the copy itself, single-threaded; here it goes
// through two page-locked staging buffers instead: while the GPU moves chunk
// k + 1, host threads move chunk k between its staging buffer and the caller's
// memory in parallel, so the copy runs at the bus rate rather than at one
// core's memcpy rate (and the first-touch page faults of a fresh output array
// are spread over the threads).
//
// The two 64 MiB staging buffers are allocated once per process on first use
// and kept; a mutex serialises the staged copies of concurrent solves.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "pdot_common.cuh"

namespace pdot {
namespace {

constexpr size_t kStageBytes = kTransferChunk * sizeof(double);
constexpr size_t kDirectBelow = size_t(16) << 20;  // smaller copies go by one cudaMemcpy
std::mutex g_stage_mutex;
void* g_stage[2] = {nullptr, nullptr};

int copy_workers() {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  return (int)std::min(8u, std::max(1u, hw / 2));
}

// memcpy of `bytes` split over `workers` threads (the caller is one of them),
// in slices aligned to 4 KiB pages.
void parallel_memcpy(void* dst, const void* src, size_t bytes, int workers) {
  const size_t page = 4096;
  size_t per = (bytes + workers - 1) / workers;
  per = (per + page - 1) / page * page;
  std::vector<std::thread> threads;
  for (int w = 1; w < workers; ++w) {
    const size_t lo = (size_t)w * per;
    if (lo >= bytes) break;
    const size_t len = std::min(per, bytes - lo);
    threads.emplace_back([=] { memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, len); });
  }
  memcpy(dst, src, std::min(per, bytes));
  for (std::thread& t : threads) t.join();
}

cudaError_t ensure_stage() {
  for (int k = 0; k < 2; ++k) {
    if (g_stage[k]) continue;
    const cudaError_t e = cudaMallocHost(&g_stage[k], kStageBytes);
    if (e != cudaSuccess) {
      g_stage[k] = nullptr;
      return e;
    }
  }
  return cudaSuccess;
}

struct Events {
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaError_t create() {
    for (cudaEvent_t& e : ev) {
      const cudaError_t r = cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
      if (r != cudaSuccess) return r;
    }
    return cudaSuccess;
  }
  ~Events() {
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

#define PDOT_TRY(x)                         \
  do {                                      \
    const cudaError_t e_ = (x);             \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

}  // namespace

bool host_is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

cudaError_t copy_to_device(void* dst, const void* src, size_t bytes, cudaStream_t s) {
  if (host_is_pinned(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  if (bytes < kDirectBelow) {
    PDOT_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return cudaStreamSynchronize(s);
  }
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  PDOT_TRY(ensure_stage());
  Events E;
  PDOT_TRY(E.create());
  const int workers = copy_workers();
  const size_t chunks = (bytes + kStageBytes - 1) / kStageBytes;
  for (size_t k = 0; k < chunks; ++k) {
    const int slot = (int)(k & 1);
    const size_t off = k * kStageBytes, len = std::min(kStageBytes, bytes - off);
    // the DMA of chunk k - 2 has left this staging buffer
    if (k >= 2) PDOT_TRY(cudaEventSynchronize(E.ev[slot]));
    parallel_memcpy(g_stage[slot], static_cast<const char*>(src) + off, len, workers);
    PDOT_TRY(cudaMemcpyAsync(static_cast<char*>(dst) + off, g_stage[slot], len, cudaMemcpyHostToDevice, s));
    PDOT_TRY(cudaEventRecord(E.ev[slot], s));
  }
  return cudaStreamSynchronize(s);
}

cudaError_t copy_to_host(double* dst, size_t count, const ChunkSource& source, cudaStream_t s) {
  const size_t chunk = kStageBytes / sizeof(double);
  const size_t chunks = (count + chunk - 1) / chunk;
  if (count * sizeof(double) < kDirectBelow || host_is_pinned(dst)) {
    for (size_t k = 0; k < chunks; ++k) {
      const size_t off = k * chunk, len = std::min(chunk, count - off);
      const double* p = source(off, len, (int)(k & 1), s);
      PDOT_TRY(cudaGetLastError());
      PDOT_TRY(cudaMemcpyAsync(dst + off, p, len * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    return cudaStreamSynchronize(s);
  }
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  PDOT_TRY(ensure_stage());
  Events E;
  PDOT_TRY(E.create());
  const int workers = copy_workers();
  auto issue = [&](size_t k) -> cudaError_t {
    const int slot = (int)(k & 1);
    const size_t off = k * chunk, len = std::min(chunk, count - off);
    const double* p = source(off, len, slot, s);
    PDOT_TRY(cudaGetLastError());
    PDOT_TRY(cudaMemcpyAsync(g_stage[slot], p, len * sizeof(double), cudaMemcpyDeviceToHost, s));
    return cudaEventRecord(E.ev[slot], s);
  };
  PDOT_TRY(issue(0));
  if (chunks > 1) PDOT_TRY(issue(1));
  for (size_t k = 0; k < chunks; ++k) {
    const int slot = (int)(k & 1);
    const size_t off = k * chunk, len = std::min(chunk, count - off);
    PDOT_TRY(cudaEventSynchronize(E.ev[slot]));
    // the GPU moves chunk k + 1 meanwhile
    parallel_memcpy(dst + off, g_stage[slot], len * sizeof(double), workers);
    if (k + 2 < chunks) PDOT_TRY(issue(k + 2));
  }
  return cudaSuccess;
}

}  // namespace pdot
