// Device -> pageable host copies through pinned staging memory.
#include <algorithm>
#include <cstring>
#include <thread>

#include "lbm_internal.h"

namespace lbm {

PinnedStage::~PinnedStage() {
  for (int i = 0; i < 2; i++) {
    if (buf[i]) cudaFreeHost(buf[i]);
    if (ev[i]) cudaEventDestroy(ev[i]);
  }
}

namespace {

// Host copy out of the staging buffer split over a few threads: one thread
// writes fresh pageable memory at well under the DMA's rate.
void copy_parallel(char* dst, const char* src, size_t bytes) {
  constexpr int kThreads = 4;
  constexpr size_t kMinSplit = size_t(1) << 20;
  if (bytes < kThreads * kMinSplit) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t part = (bytes / kThreads + 63) & ~size_t(63);
  std::thread workers[kThreads - 1];
  for (int t = 1; t < kThreads; t++) {
    const size_t off = std::min(bytes, t * part), len = std::min(bytes, (t + 1) * part) - off;
    workers[t - 1] = std::thread([=] { std::memcpy(dst + off, src + off, len); });
  }
  std::memcpy(dst, src, std::min(bytes, part));
  for (auto& w : workers) w.join();
}

}  // namespace

// Chunks of kChunk bytes alternate between two pinned buffers: the DMA of
// chunk i runs while the host copies chunk i-1 out of the other buffer, so
// the transfer takes about the longer of the two instead of a pageable copy
// (which the driver stages through a small bounce buffer, chunk by chunk,
// without overlap).
cudaError_t d2h_staged(PinnedStage& s, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return cudaSuccess;
  if (!s.buf[0]) {
    for (int i = 0; i < 2; i++) {
      cudaError_t e = cudaMallocHost(&s.buf[i], PinnedStage::kChunk);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.ev[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
  }
  const size_t n = (bytes + PinnedStage::kChunk - 1) / PinnedStage::kChunk;
  auto len = [&](size_t i) { return i + 1 < n ? PinnedStage::kChunk : bytes - i * PinnedStage::kChunk; };
  const char* s8 = static_cast<const char*>(src);
  char* d8 = static_cast<char*>(dst);
  for (size_t i = 0; i <= n; i++) {
    if (i < n) {
      // buffer i&1 was emptied by the host copy of chunk i-2 (previous iteration)
      cudaError_t e = cudaMemcpyAsync(s.buf[i & 1], s8 + i * PinnedStage::kChunk, len(i), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaEventRecord(s.ev[i & 1], st);
      if (e != cudaSuccess) return e;
    }
    if (i >= 1) {
      const size_t j = i - 1;
      cudaError_t e = cudaEventSynchronize(s.ev[j & 1]);
      if (e != cudaSuccess) return e;
      copy_parallel(d8 + j * PinnedStage::kChunk, static_cast<const char*>(s.buf[j & 1]), len(j));
    }
  }
  return cudaSuccess;
}

}  // namespace lbm
