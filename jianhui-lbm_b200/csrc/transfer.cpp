// Device -> pageable host copies through pinned staging memory.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#ifdef __linux__
#include <sys/mman.h>
#endif

#include "host_copy.h"
#include "lbm_internal.h"

namespace lbm {

PinnedStage::~PinnedStage() {
  for (int i = 0; i < 2; i++) {
    if (buf[i]) cudaFreeHost(buf[i]);
    if (ev[i]) cudaEventDestroy(ev[i]);
  }
}

namespace {

// Process-wide free lists of staging buffers, one per device (the events
// belong to the device they were made on).  A copy borrows a stage and gives
// it back, so pinning host memory (milliseconds for 32 MiB) happens once per
// process and device rather than once per handle; concurrent copies from
// several threads take several stages.  The stages live until the process
// ends: freeing pinned memory from static destructors would run after the
// CUDA runtime is gone.
std::mutex g_stage_mu;
std::map<int, std::vector<PinnedStage*>>& free_stages() {
  static auto* m = new std::map<int, std::vector<PinnedStage*>>();
  return *m;
}

cudaError_t fill_stage(PinnedStage& s) {
  // whatever an earlier, failed attempt left missing
  for (int i = 0; i < 2; i++) {
    cudaError_t e = cudaSuccess;
    if (!s.buf[i]) e = cudaMallocHost(&s.buf[i], PinnedStage::kChunk);
    if (e == cudaSuccess && !s.ev[i]) e = cudaEventCreateWithFlags(&s.ev[i], cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

PinnedStage* borrow_stage(int dev) {
  std::lock_guard<std::mutex> lk(g_stage_mu);
  auto& v = free_stages()[dev];
  if (v.empty()) return new PinnedStage();
  PinnedStage* s = v.back();
  v.pop_back();
  return s;
}

void return_stage(int dev, PinnedStage* s) {
  std::lock_guard<std::mutex> lk(g_stage_mu);
  free_stages()[dev].push_back(s);
}

// Asks for transparent huge pages on the 2 MiB-aligned interior of a large
// destination: where the kernel backs anonymous memory with huge pages only
// on request (THP "madvise" mode), a fresh 188 MB field array otherwise
// takes 48 K page faults during the copy (a host test: 8 threads 21 -> 16
// ms, 4 threads 33 -> 16 ms for 188 MB).  The contents are unchanged; the
// advice only affects how the caller's pages are backed.
void advise_huge(void* dst, size_t bytes) {
#ifdef __linux__
  constexpr uintptr_t kHuge = uintptr_t(2) << 20;
  if (bytes < 2 * kHuge) return;
  const uintptr_t b = (reinterpret_cast<uintptr_t>(dst) + kHuge - 1) & ~(kHuge - 1);
  const uintptr_t e = (reinterpret_cast<uintptr_t>(dst) + bytes) & ~(kHuge - 1);
  if (e > b) madvise(reinterpret_cast<void*>(b), e - b, MADV_HUGEPAGE);  // advisory: failure is harmless
#else
  (void)dst;
  (void)bytes;
#endif
}

}  // namespace

cudaError_t stage_pool_prime() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lk(g_stage_mu);
    if (!free_stages()[dev].empty()) return cudaSuccess;
  }
  PinnedStage* s = new PinnedStage();
  e = fill_stage(*s);
  return_stage(dev, s);  // kept even when incomplete: the next copy retries
  return e;
}

// Chunks of kChunk bytes alternate between two pinned buffers: the DMA of
// chunk i runs while the host copies chunk i-1 out of the other buffer, so
// the transfer takes about the longer of the two instead of a pageable copy
// (which the driver stages through a small bounce buffer, chunk by chunk,
// without overlap).
cudaError_t d2h_staged(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  if (bytes == 0) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  advise_huge(dst, bytes);
  PinnedStage* sp = borrow_stage(dev);
  PinnedStage& s = *sp;
  e = fill_stage(s);
  const size_t n = (bytes + PinnedStage::kChunk - 1) / PinnedStage::kChunk;
  auto len = [&](size_t i) { return i + 1 < n ? PinnedStage::kChunk : bytes - i * PinnedStage::kChunk; };
  const char* s8 = static_cast<const char*>(src);
  char* d8 = static_cast<char*>(dst);
  for (size_t i = 0; i <= n && e == cudaSuccess; i++) {
    if (i < n) {
      // buffer i&1 was emptied by the host copy of chunk i-2 (previous iteration)
      e = cudaMemcpyAsync(s.buf[i & 1], s8 + i * PinnedStage::kChunk, len(i), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaEventRecord(s.ev[i & 1], st);
      if (e != cudaSuccess) break;
    }
    if (i >= 1) {
      const size_t j = i - 1;
      e = cudaEventSynchronize(s.ev[j & 1]);
      if (e != cudaSuccess) break;
      host_copy::copy_parallel(d8 + j * PinnedStage::kChunk, static_cast<const char*>(s.buf[j & 1]), len(j));
    }
  }
  // no DMA into the stage may be in flight when another copy borrows it
  if (e != cudaSuccess) cudaStreamSynchronize(st);
  return_stage(dev, sp);
  return e;
}

namespace {
std::mutex g_pool_mu;
std::map<int, bool> g_pool_ready;  // device -> release threshold raised
}  // namespace

cudaError_t dev_alloc(void** p, size_t bytes) {
  *p = nullptr;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool_ready[dev]) {
      cudaMemPool_t pool;
      e = cudaDeviceGetDefaultMemPool(&pool, dev);
      if (e != cudaSuccess) return e;
      unsigned long long keep = ~0ull;  // never return freed memory to the driver while the process runs
      e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
      g_pool_ready[dev] = true;
    }
  }
  e = cudaMallocAsync(p, bytes, 0);
  // usable on every stream once the allocation on the legacy stream is done
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  return e;
}

void dev_free(void* p) {
  if (!p) return;
  cudaDeviceSynchronize();
  cudaFreeAsync(p, 0);
}

cudaError_t dev_pool_trim() {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  int cur = 0;
  cudaError_t e = cudaGetDevice(&cur);
  if (e != cudaSuccess) return e;
  for (const auto& kv : g_pool_ready) {
    if (!kv.second) continue;
    cudaMemPool_t pool;
    if ((e = cudaSetDevice(kv.first)) != cudaSuccess) break;
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) break;
    if ((e = cudaDeviceGetDefaultMemPool(&pool, kv.first)) != cudaSuccess) break;
    if ((e = cudaMemPoolTrimTo(pool, 0)) != cudaSuccess) break;
  }
  const cudaError_t e2 = cudaSetDevice(cur);
  return e != cudaSuccess ? e : e2;
}

}  // namespace lbm
