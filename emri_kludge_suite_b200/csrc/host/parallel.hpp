// parallel.hpp -- a dynamic work split of [0, n) over host threads.
#pragma once

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace aak {

template <typename F>
void parallel_for(int64_t n, int nthreads, F &&fn) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = (int)std::min<int64_t>(nthreads, n);
  if (nthreads <= 1) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next(0);
  std::vector<std::thread> pool;
  pool.reserve(nthreads);
  for (int t = 0; t < nthreads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        const int64_t i = next.fetch_add(1);
        if (i >= n) break;
        fn(i);
      }
    });
  for (auto &th : pool) th.join();
}

}  // namespace aak
