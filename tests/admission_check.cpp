// Host-side checks of the request server's admission queue
// (quoin_b200/csrc/qb_admission.h): budget refusal, strict arrival order,
// the budget never exceeded under concurrent workers, and close/drain.
// Built and run by tests/test_admission.py; prints OK and exits 0.
#include <atomic>
#include <chrono>
#include <cstdio>
#include <random>
#include <thread>
#include <vector>

#include "../quoin_b200/csrc/qb_admission.h"

#define CHECK(c)                                                   \
  do {                                                             \
    if (!(c)) {                                                    \
      std::printf("FAILED line %d: %s\n", __LINE__, #c);           \
      return 1;                                                    \
    }                                                              \
  } while (0)

int main() {
  using Q = qb::AdmissionQueue<int>;
  {  // free-memory admission: a head within the budget waits for free memory
     // while another request runs, and is admitted once memory frees
    Q q(1000);
    std::atomic<uint64_t> free_mem{300};
    q.set_free_probe([&] { return free_mem.load(); }, 50);
    CHECK(q.push(1, 200) && q.push(2, 400));
    int v = 0;
    uint64_t b = 0;
    CHECK(q.pop(&v, &b) && v == 1);  // 200 <= 300 - 50
    std::atomic<int> got{0};
    std::thread t([&] {
      int w = 0;
      uint64_t c = 0;
      if (q.pop(&w, &c)) got = w;
    });
    std::this_thread::sleep_for(std::chrono::milliseconds(60));
    CHECK(got == 0 && q.waits_for_memory() > 0);  // 400 > 300 - 50 although within the budget
    free_mem = 600;
    std::this_thread::sleep_for(std::chrono::milliseconds(60));
    CHECK(got == 2);  // admitted on a re-probe, request 1 still running
    t.join();
    q.release(200);
    q.release(400);
    // with nothing running the head is admitted whatever the probe says
    free_mem = 0;
    CHECK(q.push(3, 500));
    CHECK(q.pop(&v, &b) && v == 3);
    q.release(500);
  }
  {  // a request above the budget is refused; one at the budget is admitted
    Q q(100);
    CHECK(!q.push(1, 101));
    CHECK(q.push(2, 100));
    int v = 0;
    uint64_t b = 0;
    CHECK(q.pop(&v, &b) && v == 2 && b == 100 && q.in_use() == 100);
    q.release(100);
    CHECK(q.in_use() == 0);
  }
  {  // strict arrival order: C fits beside A but waits behind B
    Q q(100);
    CHECK(q.push(1, 60) && q.push(2, 50) && q.push(3, 10));
    int v = 0;
    uint64_t b = 0;
    CHECK(q.pop(&v, &b) && v == 1);
    std::atomic<int> got{0};
    std::thread t([&] {
      int w = 0;
      uint64_t c = 0;
      if (q.pop(&w, &c)) got = w;
    });
    std::this_thread::sleep_for(std::chrono::milliseconds(100));
    CHECK(got == 0 && q.waiting() == 2);  // B (50) does not fit beside A (60)
    q.release(60);
    t.join();
    CHECK(got == 2);
    CHECK(q.pop(&v, &b) && v == 3 && q.in_use() == 60);
  }
  {  // eight workers, random sizes: every request once, the budget never exceeded
    const uint64_t budget = 1000;
    Q q(budget);
    const int n = 20000;
    std::mt19937_64 rng(7);
    std::vector<uint64_t> size(n);
    for (int i = 0; i < n; i++) size[i] = 1 + rng() % 400;
    std::vector<std::atomic<int>> seen(n);
    for (auto& s : seen) s = 0;
    std::atomic<uint64_t> live{0}, live_max{0};
    std::vector<std::thread> th;
    for (int w = 0; w < 8; w++)
      th.emplace_back([&] {
        int v;
        uint64_t b;
        while (q.pop(&v, &b)) {
          uint64_t now = live += b;
          uint64_t m = live_max.load();
          while (now > m && !live_max.compare_exchange_weak(m, now)) {
          }
          seen[v]++;
          live -= b;
          q.release(b);
        }
      });
    for (int i = 0; i < n; i++) CHECK(q.push(i, size[i]));
    q.close();
    for (auto& t : th) t.join();
    for (int i = 0; i < n; i++) CHECK(seen[i] == 1);
    CHECK(q.peak() <= budget && live_max <= budget && q.in_use() == 0);
  }
  {  // after close: pushes fail, queued requests drain, then pop reports the end
    Q q(10);
    CHECK(q.push(1, 5));
    q.close();
    CHECK(!q.push(2, 5));
    int v = 0;
    uint64_t b = 0;
    CHECK(q.pop(&v, &b) && v == 1);
    q.release(b);
    CHECK(!q.pop(&v, &b));
  }
  std::printf("OK\n");
  return 0;
}
