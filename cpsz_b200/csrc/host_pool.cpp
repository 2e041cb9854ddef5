// host_pool.cpp -- the process-wide host worker pool (host_pool.h).
#include "host_pool.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

namespace cpsz {

namespace {

class HostPool {
 public:
  static HostPool& get() {
    static HostPool p;
    return p;
  }
  void run(int n, const std::function<void(int)>& f) {
    if (n <= 0) return;
    if (n == 1 || workers_.empty()) {
      for (int i = 0; i < n; i++) f(i);
      return;
    }
    std::lock_guard<std::mutex> turn(turn_);
    const int helpers = std::min<int>((int)workers_.size(), n - 1);
    {
      std::lock_guard<std::mutex> lk(m_);
      f_ = &f;
      n_ = n;
      helpers_ = helpers;
      next_.store(helpers + 1);
      active_ = helpers;
      gen_++;
    }
    cv_.notify_all();
    // item 0 on the calling thread and item w + 1 on worker w, so a thread
    // gets the same item from call to call (its scratch stays warm); items
    // beyond the helpers go to whoever is free
    f(0);
    drain();
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [&] { return active_ == 0; });
    f_ = nullptr;
  }

 private:
  HostPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    const int nw = (int)std::min(31u, hw > 1 ? hw - 1 : 0u);
    for (int w = 0; w < nw; w++) workers_.emplace_back([this, w] { loop(w); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void drain() {
    for (int i = next_++; i < n_; i = next_++) (*f_)(i);
  }
  void loop(int w) {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        // a job takes workers 0 .. helpers_ - 1
        cv_.wait(lk, [&] { return stop_ || (gen_ != seen && w < helpers_); });
        if (stop_) return;
        seen = gen_;
      }
      (*f_)(w + 1);
      drain();
      std::lock_guard<std::mutex> lk(m_);
      if (--active_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> workers_;
  std::mutex turn_, m_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* f_ = nullptr;
  int n_ = 0, helpers_ = 0, active_ = 0;
  std::atomic<int> next_{0};
  unsigned long long gen_ = 0;
  bool stop_ = false;
};

}  // namespace

void host_parallel_for(int n, const std::function<void(int)>& f) { HostPool::get().run(n, f); }

}  // namespace cpsz
