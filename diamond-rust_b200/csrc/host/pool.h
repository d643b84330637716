// A small persistent pool of host threads for the CPU-side steps of a search
// (the exact ALP E-values of the kept HSPs).  One pool per context; the
// calling thread takes part, so a pool of n runs n + 1 ranges at once.
#pragma once
#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace drg {
namespace host {

class Pool {
 public:
  explicit Pool(unsigned workers) {
    for (unsigned i = 0; i < workers; ++i) threads_.emplace_back([this] { loop(); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }
  Pool(const Pool&) = delete;
  Pool& operator=(const Pool&) = delete;

  unsigned size() const { return (unsigned)threads_.size() + 1; }

  // fn(lo, hi) over [0, n) in contiguous ranges of at least `grain` items,
  // at most max_parts of them (0: the pool's size), on the workers and the
  // calling thread; returns when all are done.
  void parallel_for(uint64_t n, uint64_t grain, uint64_t max_parts,
                    const std::function<void(uint64_t, uint64_t)>& fn) {
    uint64_t parts = std::min<uint64_t>(size(), std::max<uint64_t>(1, n / std::max<uint64_t>(grain, 1)));
    if (max_parts) parts = std::min(parts, max_parts);
    if (parts <= 1 || threads_.empty()) {
      if (n) fn(0, n);
      return;
    }
    std::unique_lock<std::mutex> lk(mu_);
    job_ = &fn;
    n_ = n;
    parts_ = parts;
    next_ = 1;  // part 0 is the caller's
    done_ = 0;
    ++gen_;
    lk.unlock();
    cv_.notify_all();
    run_part(0);
    lk.lock();
    // the caller also takes parts the workers have not started
    while (next_ < parts_) {
      const uint64_t p = next_++;
      lk.unlock();
      run_part(p);
      lk.lock();
      ++done_;
    }
    done_cv_.wait(lk, [this] { return done_ + 1 == parts_; });
    job_ = nullptr;
  }

 private:
  void run_part(uint64_t p) {
    const uint64_t lo = n_ * p / parts_, hi = n_ * (p + 1) / parts_;
    if (lo < hi) (*job_)(lo, hi);
  }
  void loop() {
    uint64_t seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return stop_ || (gen_ != seen && job_ && next_ < parts_); });
      if (stop_) return;
      seen = gen_;
      while (job_ && next_ < parts_) {
        const uint64_t p = next_++;
        lk.unlock();
        run_part(p);
        lk.lock();
        ++done_;
        if (done_ + 1 == parts_) done_cv_.notify_all();
      }
    }
  }

  std::vector<std::thread> threads_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(uint64_t, uint64_t)>* job_ = nullptr;
  uint64_t n_ = 0, parts_ = 0, next_ = 0, done_ = 0, gen_ = 0;
  bool stop_ = false;
};

}  // namespace host
}  // namespace drg
