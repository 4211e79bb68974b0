// Host copies of large result arrays on several threads. One thread copies into freshly allocated
// memory at a few GB/s (the first touch of every page costs a fault), far below the host's memory
// bandwidth; result sets of millions of configurations are copied twice per call (device staging ->
// run, run -> caller), so both copies are split across threads.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstring>
#include <system_error>
#include <thread>
#include <vector>

namespace sqsg {

// Helper threads of all copies in flight share one budget (half the host's hardware threads, at most
// 8), so that concurrent callers (a server's finalizers) do not oversubscribe the host and starve the
// threads that feed the GPU.
inline std::atomic<int>& copy_threads_in_use() {
  static std::atomic<int> n{0};
  return n;
}

inline void parallel_copy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kMinPerThread = 4u << 20;
  const int budget = static_cast<int>(std::min<size_t>(8, std::max<size_t>(1, std::thread::hardware_concurrency() / 2)));
  size_t want = std::min<size_t>(static_cast<size_t>(budget), bytes / kMinPerThread);
  int helpers = 0;  // helper threads reserved from the budget (the caller copies one share itself)
  if (want > 1) {
    int used = copy_threads_in_use().load();
    for (;;) {
      helpers = std::min<int>(static_cast<int>(want) - 1, budget - used);
      if (helpers <= 0) {
        helpers = 0;
        break;
      }
      if (copy_threads_in_use().compare_exchange_weak(used, used + helpers)) break;
    }
  }
  const size_t n = static_cast<size_t>(helpers) + 1;
  if (n <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t per = (bytes / n + 4095) & ~static_cast<size_t>(4095);
  std::vector<std::thread> th;
  th.reserve(n - 1);
  size_t done = per;  // the calling thread copies the first share
  try {
    for (size_t off = per; off < bytes; off += per) {
      const size_t len = std::min(per, bytes - off);
      th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len); });
      done = off + len;
    }
  } catch (std::system_error const&) {  // no thread available: copy the rest here
  }
  std::memcpy(dst, src, std::min(per, bytes));
  if (done < bytes) std::memcpy(static_cast<char*>(dst) + done, static_cast<const char*>(src) + done, bytes - done);
  for (auto& t : th) t.join();
  copy_threads_in_use().fetch_sub(helpers);
}

}  // namespace sqsg
