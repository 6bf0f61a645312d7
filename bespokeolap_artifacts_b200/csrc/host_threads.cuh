// Host threads owned by a context (internal, not part of the ABI).
//
// HostQueue: one background thread that runs posted tasks in order.  The
// streamed join posts its per-query payload gathers there: a task waits for a
// probe chunk's device event, gathers the matching rows' payload, then
// enqueues the copy and the kernel that consume it, so the caller's thread
// never blocks on the device.
//
// HostPool: a fixed set of threads that run one loop at a time, split into
// equal slices.  Idle workers spin for a short while before they sleep, so a
// loop that follows shortly after the previous one starts without a wake-up.
#pragma once

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace bo {

inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#else
  std::this_thread::yield();
#endif
}

class HostPool {
 public:
  using Loop = std::function<void(int64_t, int64_t)>;

  explicit HostPool(int threads) : n_(threads < 1 ? 1 : threads) {
    for (int i = 1; i < n_; ++i) th_.emplace_back([this, i] { worker(i); });
  }
  ~HostPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      gen_.fetch_add(1, std::memory_order_release);
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  HostPool(const HostPool&) = delete;
  HostPool& operator=(const HostPool&) = delete;

  int threads() const { return n_; }

  // Runs fn(begin, end) over disjoint slices covering [0, n); the calling
  // thread takes the first slice.  Loops below `serial_below` run inline.
  void parallel_for(int64_t n, const Loop& fn, int64_t serial_below = 4096) {
    if (n <= 0) return;
    if (n_ == 1 || n < serial_below) {
      fn(0, n);
      return;
    }
    fn_ = &fn;
    count_ = n;
    pending_.store(n_ - 1, std::memory_order_relaxed);
    {
      std::lock_guard<std::mutex> lk(mu_);
      gen_.fetch_add(1, std::memory_order_release);
    }
    cv_.notify_all();
    fn(0, n / n_);
    while (pending_.load(std::memory_order_acquire) != 0) cpu_relax();
  }

 private:
  void worker(int index) {
    uint64_t seen = 0;
    for (;;) {
      uint64_t g = gen_.load(std::memory_order_acquire);
      if (g == seen) {
        const auto t0 = std::chrono::steady_clock::now();
        for (uint32_t spins = 1; (g = gen_.load(std::memory_order_acquire)) == seen; ++spins) {
          cpu_relax();
          if ((spins & 255u) == 0 && std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(300)) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return gen_.load(std::memory_order_acquire) != seen; });
          }
        }
      }
      seen = g;
      if (stop_) return;
      const int64_t n = count_;
      (*fn_)(n * index / n_, n * (index + 1) / n_);
      pending_.fetch_sub(1, std::memory_order_release);
    }
  }

  int n_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::atomic<uint64_t> gen_{0};
  std::atomic<int> pending_{0};
  const Loop* fn_ = nullptr;
  int64_t count_ = 0;
  bool stop_ = false;
};

class HostQueue {
 public:
  // A task returns a status (0 = success) and may fill the message.
  using Task = std::function<int(std::string&)>;

  // `init` runs first on the queue's thread (e.g. to select the CUDA device).
  explicit HostQueue(std::function<void()> init) : th_([this, init] {
      if (init) init();
      run();
    }) {}
  ~HostQueue() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    th_.join();
  }
  HostQueue(const HostQueue&) = delete;
  HostQueue& operator=(const HostQueue&) = delete;

  // Appends a task; returns its ticket (tickets count up from 1).
  uint64_t post(Task t) {
    uint64_t ticket;
    {
      std::lock_guard<std::mutex> lk(mu_);
      q_.push_back(std::move(t));
      ticket = ++posted_;
    }
    cv_.notify_all();
    return ticket;
  }

  // Blocks until the task with this ticket (and every earlier one) has run.
  void wait_for(uint64_t ticket) {
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return finished_ >= ticket; });
  }

  // Blocks until every posted task has run; returns the first failure since
  // the previous drain (0 if none) and its message.
  int drain(std::string* message) {
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return finished_ >= posted_; });
    const int rc = first_rc_;
    if (message) *message = first_msg_;
    first_rc_ = 0;
    first_msg_.clear();
    return rc;
  }

 private:
  void run() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
        if (q_.empty()) return;  // stop requested and nothing left
        t = std::move(q_.front());
        q_.pop_front();
      }
      std::string msg;
      const int rc = t(msg);
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (rc && !first_rc_) {
          first_rc_ = rc;
          first_msg_ = msg;
        }
        ++finished_;
      }
      done_cv_.notify_all();
    }
  }

  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<Task> q_;
  uint64_t posted_ = 0, finished_ = 0;
  int first_rc_ = 0;
  std::string first_msg_;
  bool stop_ = false;
  std::thread th_;  // last: started after every other member exists
};

}  // namespace bo
