// Host thread pool for the setup work (copy-table building and compiling):
// runs f(0) .. f(n - 1) on up to min(hardware threads, 16) threads, each
// taking the next index in turn.  Every f(i) writes only its own outputs, so
// the results do not depend on the number of threads.
#pragma once
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

namespace mhd {

template <class F>
void parallel_for(int n, F &&f) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min<unsigned>(std::min(hw, 16u), (unsigned)std::max(n, 0));
  if (nt <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next{0};
  auto work = [&]() {
    for (int i; (i = next.fetch_add(1)) < n;) f(i);
  };
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto &th : pool) th.join();
}

}  // namespace mhd
