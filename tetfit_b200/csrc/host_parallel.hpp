// Host-side parallel loops for the set-up.  Work is split into contiguous
// index ranges, one per thread, and every caller writes only its own
// positions, so results are the same for any thread count.
#pragma once
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

namespace tf {

// Allocator whose vectors default-initialise their elements: large scratch
// arrays that are filled completely are not zeroed first (on one thread)
// and are first touched by the parallel loops that fill them.
template <typename T, typename A = std::allocator<T>>
struct default_init_allocator : A {
  using A::A;
  template <typename U>
  struct rebind {
    using other = default_init_allocator<U, typename std::allocator_traits<A>::template rebind_alloc<U>>;
  };
  template <typename U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args) {
    std::allocator_traits<A>::construct(static_cast<A&>(*this), p, std::forward<Args>(args)...);
  }
};

// threads <= 0: all hardware threads
inline int host_threads(int threads) {
  if (threads > 0) return threads;
  const unsigned h = std::thread::hardware_concurrency();
  return h ? (int)h : 1;
}

// Persistent workers for the set-up loops, so that the many short parallel
// regions of an iterative set-up step (the stability estimate) do not pay a
// thread start each.  One job at a time: a caller that finds the pool busy
// (another host thread's set-up) starts its own threads instead.  The pool
// belongs to the process that created it (worker threads do not survive a
// fork) and is never destroyed, so no destructor runs while workers wait.
class HostPool {
 public:
  static HostPool* get() {
    static HostPool* p = new HostPool(std::max(1u, std::thread::hardware_concurrency()) - 1);
    return p->pid_ == getpid() ? p : nullptr;
  }
  int workers() const { return (int)workers_.size(); }
  // runs f(k) for k in [0, nt) on the caller and the workers; false if busy
  bool run(int nt, const std::function<void(int)>& f) {
    std::unique_lock<std::mutex> busy(busy_, std::try_to_lock);
    if (!busy.owns_lock()) return false;
    auto job = std::make_shared<Job>(&f, nt);
    {
      std::lock_guard<std::mutex> lk(m_);
      cur_ = job;
      gen_++;
    }
    cv_.notify_all();
    execute(*job);
    {
      std::unique_lock<std::mutex> lk(job->m);
      job->cv.wait(lk, [&] { return job->done; });
    }
    std::lock_guard<std::mutex> lk(m_);
    cur_.reset();
    return true;
  }

 private:
  // One job's own counters: a worker that wakes late still holds the job it
  // woke for, finds its tasks all claimed and leaves, so it can never claim
  // or count a task of a later job.
  struct Job {
    Job(const std::function<void(int)>* fn, int n) : f(fn), n(n), left(n) {}
    const std::function<void(int)>* f;
    const int n;
    std::atomic<int> next{0}, left;
    std::mutex m;
    std::condition_variable cv;
    bool done = false;
  };
  static void execute(Job& j) {
    for (int k = j.next.fetch_add(1); k < j.n; k = j.next.fetch_add(1)) {
      (*j.f)(k);
      if (j.left.fetch_sub(1) == 1) {
        std::lock_guard<std::mutex> lk(j.m);
        j.done = true;
        j.cv.notify_all();
      }
    }
  }
  explicit HostPool(unsigned nw) : pid_(getpid()) {
    for (unsigned k = 0; k < nw; k++)
      workers_.emplace_back([this] {
        uint64_t seen = 0;
        for (;;) {
          std::shared_ptr<Job> job;
          {
            std::unique_lock<std::mutex> lk(m_);
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            job = cur_;
          }
          if (job) execute(*job);
        }
      });
    for (auto& t : workers_) t.detach();
  }
  const pid_t pid_;
  std::mutex busy_, m_;
  std::condition_variable cv_;
  std::vector<std::thread> workers_;
  std::shared_ptr<Job> cur_;
  uint64_t gen_ = 0;
};

// f(begin, end) over [0, n) in up to `threads` contiguous ranges of at
// least `grain` indices; loops below one grain run inline
template <typename F>
void parallel_for(int64_t n, int threads, F&& f, int64_t grain = 4096) {
  const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(host_threads(threads), n / grain));
  if (nt <= 1) {
    if (n > 0) f((int64_t)0, n);
    return;
  }
  HostPool* hp = HostPool::get();
  if (hp && nt <= hp->workers() + 1 &&
      hp->run((int)nt, [&](int k) { f(n * k / nt, n * (k + 1) / nt); }))
    return;
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
