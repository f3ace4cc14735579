// Minimal stand-in for the three oneTBB names the reference CPU path uses, so that
// src/propagate-tor-test_tbb.cpp compiles unmodified in an image without TBB.
//
// TEST INFRASTRUCTURE ONLY (oracle): never linked into the product library.
//
// Used names (reference src/propagate-tor-test_tbb.cpp):
//   tbb::blocked_range<size_t>(begin, end, grain)          TBB:874, TBB:876
//   tbb::parallel_for(range, body)                         TBB:874, TBB:876
//   tbb::global_control(max_allowed_parallelism, n)        TBB:868
//
// Semantics: a static-partition approximation of TBB's scheduler for this program's
// two-level loop (events outside, track blocks inside). Each thread owns a budget of
// threads (the outermost caller gets `max_allowed_parallelism`). A parallel_for splits its
// range into min(budget, ceil(n / grain)) contiguous chunks and runs them on std::threads;
// each worker inherits an equal share of the caller's budget, so a nested parallel_for
// only fans out when the outer loop had fewer chunks than threads (e.g. 10 events with
// grain 4 and 8 threads). With a budget of 1 every loop runs serially in the caller.
#pragma once
#include <algorithm>
#include <cstddef>
#include <thread>
#include <vector>

namespace tbb {

namespace shim_detail {
inline int& thread_limit() {
  static int n = 1;
  return n;
}
// budget of the calling thread; -1 = not inside any parallel_for (use thread_limit())
inline int& my_budget() {
  static thread_local int b = -1;
  return b;
}
}  // namespace shim_detail

inline void tbb_shim_set_threads(int n) { shim_detail::thread_limit() = n < 1 ? 1 : n; }
inline int tbb_shim_threads() { return shim_detail::thread_limit(); }

template <typename T>
class blocked_range {
 public:
  blocked_range(T b, T e, size_t grain = 1) : b_(b), e_(e), g_(grain ? grain : 1) {}
  T begin() const { return b_; }
  T end() const { return e_; }
  size_t grainsize() const { return g_; }
  size_t size() const { return e_ > b_ ? size_t(e_ - b_) : 0; }
  bool empty() const { return !(b_ < e_); }

 private:
  T b_, e_;
  size_t g_;
};

template <typename T, typename Body>
void parallel_for(const blocked_range<T>& r, const Body& body) {
  const size_t n = r.size();
  int budget = shim_detail::my_budget();
  if (budget < 0) budget = shim_detail::thread_limit();
  size_t chunks = std::min<size_t>(size_t(budget), (n + r.grainsize() - 1) / r.grainsize());
  if (chunks <= 1) {
    body(r);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(chunks);
  for (size_t c = 0; c < chunks; ++c) {
    T lo = T(r.begin() + (n * c) / chunks);
    T hi = T(r.begin() + (n * (c + 1)) / chunks);
    int share = int((size_t(budget) * (c + 1)) / chunks - (size_t(budget) * c) / chunks);
    pool.emplace_back([lo, hi, share, &r, &body]() {
      shim_detail::my_budget() = share < 1 ? 1 : share;
      body(blocked_range<T>(lo, hi, r.grainsize()));
    });
  }
  for (auto& t : pool) t.join();
}

class global_control {
 public:
  enum parameter { max_allowed_parallelism = 0, thread_stack_size = 1 };
  global_control(parameter p, size_t value) {
    if (p == max_allowed_parallelism) {
      prev_ = shim_detail::thread_limit();
      shim_detail::thread_limit() = value < 1 ? 1 : int(value);
      active_ = true;
    }
  }
  ~global_control() {
    if (active_) shim_detail::thread_limit() = prev_;
  }

 private:
  int prev_ = 1;
  bool active_ = false;
};

}  // namespace tbb
