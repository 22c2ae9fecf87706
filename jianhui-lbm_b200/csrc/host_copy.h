// Multi-threaded host memcpy for the copies out of pinned staging
// (transfer.cpp).  Header-only and free of CUDA so that a host test can
// build it alone.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>

namespace lbm {
namespace host_copy {

// Host threads for the copies out of staging, started once per process: a
// 188 MB field read is 12 chunks, and starting 15 threads per chunk cost
// about 0.3 ms each time.  One job at a time; the caller works on its parts
// too, so a job finishes even where the workers are gone (a forked child).
// The pool is never destroyed (its threads wait on the condition variable
// until the process ends).
class CopyWorkers {
 public:
  explicit CopyWorkers(int n) {
    for (int i = 0; i < n; i++) std::thread([this] { loop(); }).detach();
  }
  // fn(p) for every p in [0, parts); returns when all have run
  void run(int parts, const std::function<void(int)>& fn) {
    std::lock_guard<std::mutex> job(job_mu_);
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      parts_ = parts;
      next_ = 0;
      left_ = parts;
      gen_++;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return left_ == 0; });
    fn_ = nullptr;
  }

 private:
  void work() {
    for (;;) {
      int p;
      const std::function<void(int)>* f;
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (!fn_ || next_ >= parts_) return;
        p = next_++;
        f = fn_;
      }
      (*f)(p);
      std::lock_guard<std::mutex> lk(mu_);
      if (--left_ == 0) done_.notify_all();
    }
  }
  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
      }
      work();
    }
  }
  std::mutex job_mu_, mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* fn_ = nullptr;
  int parts_ = 0, next_ = 0, left_ = 0;
  unsigned long long gen_ = 0;
};

inline int copy_threads() {
  static const int n = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  return n;
}

inline CopyWorkers& copy_workers() {
  static CopyWorkers* w = new CopyWorkers(copy_threads() - 1);
  return *w;
}

// Host copy out of the staging buffer split over up to 16 threads: one
// thread writes fresh pageable memory (page faults, the kernel zeroing each
// page) at well under the DMA's rate.
inline void copy_parallel(char* dst, const char* src, size_t bytes) {
  constexpr size_t kMinSplit = size_t(1) << 20;
  const int nt = (int)std::min<size_t>((size_t)copy_threads(), std::max<size_t>(1, bytes / kMinSplit));
  if (nt == 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  // ceil(bytes / nt) rounded up to 64 bytes: the parts cover every byte
  const size_t part = ((bytes + nt - 1) / nt + 63) & ~size_t(63);
  copy_workers().run(nt, [=](int t) {
    const size_t off = std::min(bytes, t * part), len = std::min(bytes, (t + 1) * part) - off;
    if (len) std::memcpy(dst + off, src + off, len);
  });
}

}  // namespace host_copy
}  // namespace lbm
