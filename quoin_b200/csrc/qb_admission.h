// FIFO admission of requests against a device-memory budget, for the request
// server (qb_serve.cpp).  Requests leave in arrival order: the head is handed
// to a worker once the bytes it will hold fit beside those of the requests
// already running and, with a free-memory probe, within the device memory
// free at that moment (less a reserve); a request that alone exceeds the
// budget is refused when it is submitted.  A head that fits the budget but
// not the free memory waits (re-probing every few milliseconds) while other
// requests run; the probe is called outside the lock and its value reused
// for a short while; with nothing running it is admitted anyway, so the queue
// always moves (its allocations then fail or succeed on their own).
// Host-only code (no CUDA; the probe is a plain function), so the policy is
// testable on CPU.
#pragma once

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <functional>
#include <mutex>
#include <utility>

namespace qb {

template <class T>
class AdmissionQueue {
 public:
  explicit AdmissionQueue(uint64_t budget) : budget_(budget) {}

  // Device memory free right now (e.g. cudaMemGetInfo), consulted before a
  // head request is admitted; `reserve` bytes are kept free.
  void set_free_probe(std::function<uint64_t()> probe, uint64_t reserve) {
    std::lock_guard<std::mutex> l(mu_);
    probe_ = std::move(probe);
    reserve_ = reserve;
  }

  // Queues `item` holding `bytes` while it runs.  False when it can never be
  // admitted (bytes > budget) or the queue is closed.
  bool push(T item, uint64_t bytes) {
    {
      std::lock_guard<std::mutex> l(mu_);
      if (closed_ || bytes > budget_) return false;
      q_.emplace_back(std::move(item), bytes);
    }
    cv_.notify_all();
    return true;
  }

  // Blocks until the head request fits the budget, then removes it and counts
  // its bytes as in use.  False once the queue is closed and drained.
  // The probe runs without the lock (it may wait inside the driver while
  // running requests allocate or free), one caller at a time, and its value
  // is reused for kProbeTtl less the bytes admitted since; it is only
  // consulted again sooner when that estimate says the head does not fit.
  bool pop(T* item, uint64_t* bytes) {
    std::unique_lock<std::mutex> l(mu_);
    for (;;) {
      cv_.wait(l, [&] {
        return (!q_.empty() && in_use_ + q_.front().second <= budget_ && !probing_) || (closed_ && q_.empty());
      });
      if (q_.empty()) return false;
      if (!probe_ || in_use_ == 0) break;
      const uint64_t need = q_.front().second;
      const auto now = std::chrono::steady_clock::now();
      if (have_probe_ && now - probed_at_ < kProbeTtl && in_use_ >= in_use_at_probe_) {
        uint64_t since = in_use_ - in_use_at_probe_;
        uint64_t est = free_at_probe_ > since ? free_at_probe_ - since : 0;
        if (est > reserve_ && need <= est - reserve_) break;
      }
      probing_ = true;
      l.unlock();
      uint64_t fr = probe_();
      l.lock();
      probing_ = false;
      have_probe_ = true;
      probed_at_ = std::chrono::steady_clock::now();
      free_at_probe_ = fr;
      in_use_at_probe_ = in_use_;
      cv_.notify_all();
      if (q_.empty()) continue;
      if (in_use_ == 0 || (in_use_ + q_.front().second <= budget_ && fr > reserve_ && q_.front().second <= fr - reserve_))
        break;
      waits_for_memory_++;
      have_probe_ = false;  // re-probe after the wait: memory frees as running requests end
      cv_.wait_for(l, std::chrono::milliseconds(5));
    }
    *item = std::move(q_.front().first);
    *bytes = q_.front().second;
    q_.pop_front();
    in_use_ += *bytes;
    if (in_use_ > peak_) peak_ = in_use_;
    return true;
  }

  // A popped request finished: its bytes are free again.
  void release(uint64_t bytes) {
    {
      std::lock_guard<std::mutex> l(mu_);
      in_use_ -= bytes;
    }
    cv_.notify_all();
  }

  // No more requests; the queued ones are still handed out.
  void close() {
    {
      std::lock_guard<std::mutex> l(mu_);
      closed_ = true;
    }
    cv_.notify_all();
  }

  uint64_t in_use() const {
    std::lock_guard<std::mutex> l(mu_);
    return in_use_;
  }
  uint64_t peak() const {
    std::lock_guard<std::mutex> l(mu_);
    return peak_;
  }
  size_t waiting() const {
    std::lock_guard<std::mutex> l(mu_);
    return q_.size();
  }
  // Times a head request that fit the budget waited for free device memory.
  uint64_t waits_for_memory() const {
    std::lock_guard<std::mutex> l(mu_);
    return waits_for_memory_;
  }

 private:
  const uint64_t budget_;
  uint64_t in_use_ = 0, peak_ = 0, reserve_ = 0, waits_for_memory_ = 0;
  std::function<uint64_t()> probe_;
  static constexpr std::chrono::milliseconds kProbeTtl{50};
  bool probing_ = false, have_probe_ = false;
  std::chrono::steady_clock::time_point probed_at_{};
  uint64_t free_at_probe_ = 0, in_use_at_probe_ = 0;
  bool closed_ = false;
  std::deque<std::pair<T, uint64_t>> q_;
  mutable std::mutex mu_;
  std::condition_variable cv_;
};

}  // namespace qb
