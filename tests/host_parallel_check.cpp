// Checks of the set-up's host threading (tetfit_b200/csrc/host_parallel.hpp),
// built and run by tests/test_host_parallel.py:
//   1. parallel_for covers every index exactly once, over many short jobs of
//      random sizes and grains (the persistent pool's job hand-off);
//   2. two host threads calling parallel_for at once (one finds the pool busy
//      and starts its own threads) both get exact coverage;
//   3. parallel_stable_sort gives exactly std::stable_sort's order, ties
//      included, for any thread count.
// Prints "ok" and exits 0, or names the failed check and exits 1.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <thread>
#include <utility>
#include <vector>

#include "../tetfit_b200/csrc/host_parallel.hpp"

static bool cover(std::mt19937& g, int jobs) {
  for (int it = 0; it < jobs; it++) {
    const int64_t n = 1 + g() % 40000;
    std::vector<int> hit(n, 0);
    tf::parallel_for(n, 0, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; i++) hit[i]++;
    }, 1 + g() % 2048);
    for (int64_t i = 0; i < n; i++)
      if (hit[i] != 1) return false;
  }
  return true;
}

int main(int argc, char** argv) {
  const int jobs = argc > 1 ? std::atoi(argv[1]) : 20000;
  std::mt19937 g(7);
  if (!cover(g, jobs)) {
    std::printf("parallel_for coverage failed\n");
    return 1;
  }
  bool ok2 = true, ok3 = true;
  {
    std::thread other([&] {
      std::mt19937 h(11);
      ok2 = cover(h, jobs / 4);
    });
    ok3 = cover(g, jobs / 4);
    other.join();
  }
  if (!ok2 || !ok3) {
    std::printf("concurrent parallel_for coverage failed\n");
    return 1;
  }
  for (int trial = 0; trial < 24; trial++) {
    const size_t n = g() % (trial < 12 ? 200000 : 2000000);
    std::vector<std::pair<int, int>> v(n);
    for (size_t i = 0; i < n; i++) v[i] = {(int)(g() % (trial % 2 ? 40 : 1000000)), (int)i};
    auto w = v;
    auto key = [](const std::pair<int, int>& a, const std::pair<int, int>& b) { return a.first < b.first; };
    std::stable_sort(v.begin(), v.end(), key);
    tf::parallel_stable_sort(w.begin(), w.end(), 1 + trial % 9, key);
    if (v != w) {
      std::printf("parallel_stable_sort differs from std::stable_sort (trial %d)\n", trial);
      return 1;
    }
  }
  std::printf("ok\n");
  return 0;
}
