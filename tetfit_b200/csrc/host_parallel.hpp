// Host-side parallel loops for the set-up.  Work is split into contiguous
// index ranges, one per thread, and every caller writes only its own
// positions, so results are the same for any thread count.
#pragma once
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace tf {

// threads <= 0: all hardware threads
inline int host_threads(int threads) {
  if (threads > 0) return threads;
  const unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// f(begin, end) over [0, n) in up to `threads` contiguous ranges
template <typename F>
void parallel_for(int64_t n, int threads, F&& f) {
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(host_threads(threads), n / 4096 + 1));
  if (nt <= 1) {
    if (n > 0) f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for (int64_t k = 1; k < nt; k++) pool.emplace_back([&, k] { f(n * k / nt, n * (k + 1) / nt); });
  f((int64_t)0, n / nt);
  for (auto& t : pool) t.join();
}

}  // namespace tf
