// Device -> pageable host copies through pinned staging memory.
#include <cstring>

#include "lbm_internal.h"

namespace lbm {

PinnedStage::~PinnedStage() {
  for (int i = 0; i < 2; i++) {
    if (buf[i]) cudaFreeHost(buf[i]);
    if (ev[i]) cudaEventDestroy(ev[i]);
  }
}

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
      std::memcpy(d8 + j * PinnedStage::kChunk, s.buf[j & 1], len(j));
    }
  }
  return cudaSuccess;
}

}  // namespace lbm
