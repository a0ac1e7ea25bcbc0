// A small persistent pool of host threads for the scan's per-run host work (the Adams
// stencil and tables before an attempt, the acceptance and step choice after it).  The
// runs are independent, so the pool hands them out one at a time from an atomic counter;
// the calling thread works too.  Waiting threads spin for a short while before they sleep,
// since the pool is asked for work every few milliseconds and a sleeping thread takes tens
// of microseconds to wake.  An exception thrown by a task is caught and the first one is
// rethrown on the caller once every task has finished.
#pragma once
#include <atomic>
#include <chrono>
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
      stop_.store(true);
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
      busy_.store((int)workers_.size());
      error_ = nullptr;
      generation_.fetch_add(1);
    }
    wake_.notify_all();
    drain();
    if (!spin([&] { return busy_.load(std::memory_order_acquire) == 0; })) {
      std::unique_lock<std::mutex> lock(mutex_);
      done_.wait(lock, [&] { return busy_.load() == 0; });
    }
    body_ = nullptr;
    if (error_) std::rethrow_exception(error_);
  }

 private:
  static constexpr std::chrono::microseconds kSpin{200};

  static void relax() {
#if defined(__x86_64__) || defined(__i386__)
    __builtin_ia32_pause();
#else
    std::this_thread::yield();
#endif
  }

  // true once ready() holds, false if it still does not after kSpin
  template <class F>
  static bool spin(F&& ready) {
    const auto until = std::chrono::steady_clock::now() + kSpin;
    for (int i = 0;; ++i) {
      if (ready()) return true;
      relax();
      if ((i & 63) == 63 && std::chrono::steady_clock::now() > until) return ready();
    }
  }

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
      auto posted = [&] { return stop_.load() || generation_.load(std::memory_order_acquire) != seen; };
      if (!spin(posted)) {
        std::unique_lock<std::mutex> lock(mutex_);
        wake_.wait(lock, posted);
      }
      if (stop_.load()) return;
      seen = generation_.load(std::memory_order_acquire);
      drain();
      if (busy_.fetch_sub(1, std::memory_order_acq_rel) == 1) {
        std::lock_guard<std::mutex> lock(mutex_);
        done_.notify_one();
      }
    }
  }

  std::vector<std::thread> workers_;
  std::mutex mutex_;
  std::condition_variable wake_, done_;
  const std::function<void(int)>* body_ = nullptr;
  int count_ = 0;
  std::atomic<int> next_{0}, busy_{0};
  std::atomic<unsigned long long> generation_{0};
  std::atomic<bool> stop_{false};
  std::exception_ptr error_;
};

}  // namespace sp
