// Stress driver for the host thread pool (cuvhs_b200/csrc/workpool.cpp), run
// by tests/test_host_pool.py: every item of every run executes exactly once,
// with primed and unprimed runs, runs of 1..200 items, idle gaps that let the
// workers go back to sleep, and pools of 0..15 worker threads.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <thread>
#include <vector>

#include "cuvhs_internal.h"

int main() {
  long bad = 0;
  for (int threads : {0, 1, 3, 15}) {
    cuvhs::WorkPool pool(threads);
    std::vector<std::atomic<int>> hits(256);
    for (int rep = 0; rep < 6000; rep++) {
      if (rep % 3 == 0) pool.prime();
      const int n = 1 + rep % 200;
      for (int i = 0; i < n; i++) hits[i].store(0);
      pool.run(n, [&](int i) { hits[i].fetch_add(1); });
      for (int i = 0; i < n; i++) bad += hits[i].load() != 1;
      if (rep % 97 == 0) std::this_thread::sleep_for(std::chrono::milliseconds(4));  // past the spin limit
      else if (rep % 7 == 0) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    // a prime with no run after it, then destruction while workers spin
    pool.prime();
  }
  std::printf("bad=%ld\n", bad);
  return bad != 0;
}
