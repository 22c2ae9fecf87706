// Host test of jianhui-lbm_b200/csrc/host_copy.h: copies of many sizes (every
// remainder modulo the thread count and the 64-byte rounding) from several
// caller threads at once must reproduce the source byte for byte.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "host_copy.h"

int main() {
  const size_t n = size_t(5) << 20;
  std::vector<char> src(n + 4096);
  for (size_t i = 0; i < src.size(); i++) src[i] = (char)(i * 131 + 7);
  int bad = 0;
  std::mutex m;
  std::vector<std::thread> callers;
  for (int c = 0; c < 4; c++)
    callers.emplace_back([&, c] {
      for (int r = 0; r < 64; r++) {
        const size_t bytes = n + (size_t)(c * 64 + r) * 17;  // odd and even remainders
        std::vector<char> dst(bytes + 64, 0);
        lbm::host_copy::copy_parallel(dst.data(), src.data(), bytes);
        const bool ok = std::memcmp(dst.data(), src.data(), bytes) == 0 && dst[bytes] == 0;
        if (!ok) {
          std::lock_guard<std::mutex> lk(m);
          bad++;
        }
      }
    });
  for (auto& t : callers) t.join();
  std::printf("threads %d, mismatched copies %d\n", lbm::host_copy::copy_threads(), bad);
  return bad == 0 ? 0 : 1;
}
