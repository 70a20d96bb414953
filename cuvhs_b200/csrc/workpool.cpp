// Fixed host thread pool for the per-field line-location work.  Jobs are
// handed over under the mutex; a primed worker waits for the next job by
// spinning on the published generation instead of sleeping.
#include <chrono>

#include "cuvhs_internal.h"

namespace cuvhs {

namespace {
inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#elif defined(__aarch64__)
  asm volatile("yield");
#endif
}
}  // namespace

WorkPool::WorkPool(int threads) {
  for (int i = 0; i < threads; i++) threads_.emplace_back([this] { worker(); });
}

WorkPool::~WorkPool() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
    stopping_.store(true);
  }
  cv_.notify_all();
  for (auto& t : threads_) t.join();
}

void WorkPool::prime() {
  if (threads_.empty()) return;
  {
    std::lock_guard<std::mutex> lk(mu_);
    prime_++;
  }
  cv_.notify_all();
}

void WorkPool::worker() {
  unsigned long long seen = 0, seen_prime = 0;
  std::unique_lock<std::mutex> lk(mu_);
  for (;;) {
    cv_.wait(lk, [&] { return stop_ || generation_ != seen || prime_ != seen_prime; });
    if (stop_) return;
    seen_prime = prime_;
    if (generation_ == seen) {
      // primed: spin (bounded) until the job is published
      lk.unlock();
      const auto t0 = std::chrono::steady_clock::now();
      for (int k = 0; published_.load(std::memory_order_acquire) == seen && !stopping_.load(); k++) {
        cpu_relax();
        if ((k & 255) == 255 &&
            std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(kSpinMs))
          break;
      }
      lk.lock();
      if (stop_) return;
      if (generation_ == seen) continue;  // nothing came: sleep again
    }
    seen = generation_;
    // join only a run still in progress: a finished run's counter may be
    // reset for the next run at any moment, and the caller cannot finish a
    // run while a worker holds active_
    if (!job_) continue;
    std::function<void(int)>* job = job_;
    const int n = n_;
    active_++;
    lk.unlock();
    for (int i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) (*job)(i);
    lk.lock();
    if (--active_ == 0) done_cv_.notify_all();
  }
}

void WorkPool::run_impl(int n, std::function<void(int)>& fn) {
  if (n <= 0) return;
  if (threads_.empty() || n == 1) {
    for (int i = 0; i < n; i++) fn(i);
    return;
  }
  {
    std::lock_guard<std::mutex> lk(mu_);
    job_ = &fn;
    n_ = n;
    next_.store(0);
    generation_++;
    published_.store(generation_, std::memory_order_release);
  }
  cv_.notify_all();
  for (int i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) fn(i);
  std::unique_lock<std::mutex> lk(mu_);
  done_cv_.wait(lk, [&] { return active_ == 0 && next_.load() >= n; });
  job_ = nullptr;
}

}  // namespace cuvhs
