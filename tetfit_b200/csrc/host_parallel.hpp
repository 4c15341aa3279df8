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

// Stable sort of [first, last) by cmp: contiguous runs sorted in parallel,
// then merged pairwise (stable merges), so the result is exactly that of
// std::stable_sort for any thread count.
template <typename It, typename Cmp>
void parallel_stable_sort(It first, It last, int threads, Cmp cmp) {
  const int64_t n = last - first;
  int64_t runs = std::max<int64_t>(1, std::min<int64_t>(host_threads(threads), n / 65536 + 1));
  if (runs <= 1) {
    std::stable_sort(first, last, cmp);
    return;
  }
  std::vector<int64_t> cut(runs + 1);
  for (int64_t k = 0; k <= runs; k++) cut[k] = n * k / runs;
  {
    std::vector<std::thread> pool;
    for (int64_t k = 1; k < runs; k++)
      pool.emplace_back([&, k] { std::stable_sort(first + cut[k], first + cut[k + 1], cmp); });
    std::stable_sort(first + cut[0], first + cut[1], cmp);
    for (auto& t : pool) t.join();
  }
  while (cut.size() > 2) {
    std::vector<int64_t> next;
    std::vector<std::thread> pool;
    for (size_t k = 0; k + 2 < cut.size(); k += 2) {
      const int64_t a = cut[k], m = cut[k + 1], b = cut[k + 2];
      pool.emplace_back([=, &cmp] { std::inplace_merge(first + a, first + m, first + b, cmp); });
      next.push_back(a);
    }
    if ((cut.size() - 1) % 2) next.push_back(cut[cut.size() - 2]);
    next.push_back(cut.back());
    for (auto& t : pool) t.join();
    cut.swap(next);
  }
}

}  // namespace tf
