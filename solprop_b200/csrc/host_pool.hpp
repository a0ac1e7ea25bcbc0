// A small persistent pool of host threads for the scan's per-run host work (the Adams
// stencil and tables before an attempt, the acceptance and step choice after it).  The
// runs are independent, so the pool hands them out one at a time from an atomic counter;
// the calling thread works too.  An exception thrown by a task is caught and the first one
// is rethrown on the caller once every task has finished.
#pragma once
#include <atomic>
#include <condition_variable>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace sp {

class HostPool {
 public:
  // n_threads workers besides the caller (0: everything runs on the caller)
  explicit HostPool(int n_threads) {
    for (int i = 0; i < n_threads; ++i) workers_.emplace_back([this] { work(); });
  }
  HostPool(const HostPool&) = delete;
  HostPool& operator=(const HostPool&) = delete;
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      stop_ = true;
    }
    wake_.notify_all();
    for (auto& t : workers_) t.join();
  }

  int threads() const { return (int)workers_.size() + 1; }

  // body(i) for every i in [0, count), in any order and on any of the pool's threads
  void run(int count, const std::function<void(int)>& body) {
    if (count <= 0) return;
    if (workers_.empty() || count == 1) {
      for (int i = 0; i < count; ++i) body(i);
      return;
    }
    {
      std::lock_guard<std::mutex> lock(mutex_);
      body_ = &body;
      count_ = count;
      next_.store(0);
      busy_ = (int)workers_.size();
      error_ = nullptr;
      ++generation_;
    }
    wake_.notify_all();
    drain();
    std::unique_lock<std::mutex> lock(mutex_);
    done_.wait(lock, [this] { return busy_ == 0; });
    body_ = nullptr;
    if (error_) std::rethrow_exception(error_);
  }

 private:
  void drain() {
    for (int i = next_.fetch_add(1); i < count_; i = next_.fetch_add(1)) {
      try {
        (*body_)(i);
      } catch (...) {
        std::lock_guard<std::mutex> lock(mutex_);
        if (!error_) error_ = std::current_exception();
      }
    }
  }

  void work() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, [&] { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
      }
      drain();
      {
        std::lock_guard<std::mutex> lock(mutex_);
        if (--busy_ == 0) done_.notify_one();
      }
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mutex_;
  std::condition_variable wake_, done_;
  const std::function<void(int)>* body_ = nullptr;
  int count_ = 0, busy_ = 0;
  std::atomic<int> next_{0};
  unsigned long long generation_ = 0;
  bool stop_ = false;
  std::exception_ptr error_;
};

}  // namespace sp
