// FIFO admission of requests against a device-memory budget, for the request
// server (qb_serve.cpp).  Requests leave in arrival order: the head is handed
// to a worker once the bytes it will hold fit beside those of the requests
// already running; a request that alone exceeds the budget is refused when it
// is submitted.  Host-only code (no CUDA), so the policy is testable on CPU.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <utility>

namespace qb {

template <class T>
class AdmissionQueue {
 public:
  explicit AdmissionQueue(uint64_t budget) : budget_(budget) {}

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
  bool pop(T* item, uint64_t* bytes) {
    std::unique_lock<std::mutex> l(mu_);
    cv_.wait(l, [&] { return (!q_.empty() && in_use_ + q_.front().second <= budget_) || (closed_ && q_.empty()); });
    if (q_.empty()) return false;
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

 private:
  const uint64_t budget_;
  uint64_t in_use_ = 0, peak_ = 0;
  bool closed_ = false;
  std::deque<std::pair<T, uint64_t>> q_;
  mutable std::mutex mu_;
  std::condition_variable cv_;
};

}  // namespace qb
