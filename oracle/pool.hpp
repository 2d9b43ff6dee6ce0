// Oracle (test infrastructure only): a persistent fork-join thread pool for the
// CPU baseline's element loops, SpMV and vector kernels. Work is split into
// one static contiguous chunk per thread, so results that depend on the split
// (ordered partial sums) depend only on the thread count, never on timing.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace oracle {

class Pool {
 public:
  static Pool& get() {
    static Pool p;
    return p;
  }
  ~Pool() { stop_all(); }

  int size() const { return n_; }

  // total threads, the calling thread included
  void resize(int n) {
    n = std::max(1, n);
    if (n == n_) return;
    stop_all();
    n_ = n;
    stop_ = false;
    const uint64_t g0 = gen_;  // no job is running: gen_ is stable here
    for (int t = 1; t < n_; ++t) th_.emplace_back([this, t, g0] { worker(t, g0); });
  }

  // f(t) for t = 0 .. size()-1, t = 0 on the calling thread; returns when all are done
  void run(const std::function<void(int)>& f) {
    if (n_ == 1) {
      f(0);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &f;
      pending_ = n_ - 1;
      ++gen_;
    }
    cv_start_.notify_all();
    f(0);
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return pending_ == 0; });
    job_ = nullptr;
  }

 private:
  Pool() = default;

  void worker(int t, uint64_t seen) {
    for (;;) {
      const std::function<void(int)>* job = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_start_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        job = job_;
      }
      (*job)(t);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) cv_done_.notify_one();
    }
  }

  void stop_all() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_start_.notify_all();
    for (auto& t : th_) t.join();
    th_.clear();
    n_ = 1;
  }

  int n_ = 1;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_start_, cv_done_;
  const std::function<void(int)>* job_ = nullptr;
  uint64_t gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

// [lo, hi) of chunk t of n split into p contiguous chunks
inline void chunk_range(long n, int p, int t, long* lo, long* hi) {
  const long c = (n + p - 1) / p;
  *lo = std::min(n, t * c);
  *hi = std::min(n, *lo + c);
}

}  // namespace oracle
