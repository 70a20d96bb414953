// Fixed host thread pool for the per-field line-location work.
#include "cuvhs_internal.h"

namespace cuvhs {

WorkPool::WorkPool(int threads) {
  for (int i = 0; i < threads; i++) threads_.emplace_back([this] { worker(); });
}

WorkPool::~WorkPool() {
  {
    std::lock_guard<std::mutex> lk(mu_);
    stop_ = true;
  }
  cv_.notify_all();
  for (auto& t : threads_) t.join();
}

void WorkPool::worker() {
  unsigned long long seen = 0;
  for (;;) {
    std::function<void(int)>* job;
    int n;
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
      if (stop_) return;
      seen = generation_;
      job = job_;
      n = n_;
      active_++;
    }
    for (int i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) (*job)(i);
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (--active_ == 0) done_cv_.notify_all();
    }
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
  }
  cv_.notify_all();
  for (int i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) fn(i);
  std::unique_lock<std::mutex> lk(mu_);
  done_cv_.wait(lk, [&] { return active_ == 0 && next_.load() >= n; });
  job_ = nullptr;
}

}  // namespace cuvhs
