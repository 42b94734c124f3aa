// Request server: compress and decompress requests on device-resident buffers,
// queued in arrival order, admitted against a device-memory budget
// (qb_admission.h) and run by one host worker per context of a pool.  The
// context-side work of each request is the single-column call's, so its bytes
// are too.  No counterpart in the reference (the serving configuration of the
// benchmark drives it).
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/quoin.h"
#include "qb_admission.h"

namespace {

// Working memory a request's context holds beyond the request's own buffers:
// the compacted lane, the encoder's per-value scratch and statistics
// (~48 B/value), or the decoder's per-value scratch and tables (~16 B/value).
uint64_t work_bytes(const QuoinB200Request& r) {
  if (r.op == QUOIN_B200_OP_COMPRESS) return 48ull * r.n + (1u << 20);
  int32_t wire = 0, hv = 0;
  uint64_t n = 0;
  if (r.idx && quoin_b200_index_info(r.idx, &wire, &n, &hv) == QUOIN_OK) return 16ull * n + (1u << 20);
  return 1u << 20;
}

}  // namespace

struct QuoinServer {
  QuoinConfig cfg;
  std::vector<QuoinCtx*> ctxs;
  qb::AdmissionQueue<QuoinB200Request*> queue;
  std::vector<std::thread> workers;
  std::mutex done_mu;
  std::condition_variable done_cv;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  explicit QuoinServer(uint64_t budget) : queue(budget) {}
  uint64_t now_ns() const {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0)
        .count();
  }

  void run(QuoinCtx* c) {
    QuoinB200Request* r = nullptr;
    uint64_t bytes = 0;
    while (queue.pop(&r, &bytes)) {
      r->t_start_ns = now_ns();
      int rc;
      try {
        if (r->op == QUOIN_B200_OP_COMPRESS) {
          size_t len = 0;
          rc = quoin_b200_compress_column_device(c, r->wire_dtype, r->n, r->d_values, r->d_validity, r->scale,
                                                 r->precision, &cfg, r->d_dst, r->dst_cap, &len, nullptr);
          r->out_len = len;
        } else {
          rc = quoin_b200_decompress_indexed_device(c, r->idx, r->d_src, r->d_values_out, r->d_validity_out,
                                                    nullptr);
        }
      } catch (...) {
        rc = QUOIN_ERR_PANIC;
      }
      r->status = rc;
      r->t_end_ns = now_ns();
      queue.release(bytes);
      {
        std::lock_guard<std::mutex> l(done_mu);
        r->done = 1;
      }
      done_cv.notify_all();
    }
  }
};

extern "C" QuoinServer* quoin_b200_server_create(int workers, uint64_t budget_bytes, const QuoinConfig* cfg) {
  if (workers < 1 || workers > 64 || budget_bytes == 0) return nullptr;
  QuoinServer* s = nullptr;
  try {
    s = new QuoinServer(budget_bytes);
    s->cfg = cfg ? *cfg : QuoinConfig{QUOIN_LEVEL_FAST, 0, 16, QUOIN_B200_SELECTION_FULL};
    for (int i = 0; i < workers; i++) {
      QuoinCtx* c = quoin_ctx_create(0);
      if (!c) throw 0;
      s->ctxs.push_back(c);
    }
    // admission also by the device memory free when a request starts (other
    // processes and the contexts' arenas share the GPU); 1 GiB stays free
    int dev = 0;
    cudaGetDevice(&dev);
    s->queue.set_free_probe(
        [dev]() -> uint64_t {
          int prev = 0;
          size_t fr = 0, tot = 0;
          cudaGetDevice(&prev);
          if (prev != dev) cudaSetDevice(dev);
          if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            fr = ~(size_t)0;  // unknown: the budget alone decides
          }
          if (prev != dev) cudaSetDevice(prev);
          return (uint64_t)fr;
        },
        1ull << 30);
    for (QuoinCtx* c : s->ctxs) s->workers.emplace_back([s, c] { s->run(c); });
    return s;
  } catch (...) {
    if (s) {
      s->queue.close();
      for (auto& t : s->workers) t.join();
      for (QuoinCtx* c : s->ctxs) quoin_ctx_free(c);
      delete s;
    }
    return nullptr;
  }
}

extern "C" int quoin_b200_server_submit(QuoinServer* s, QuoinB200Request* r) {
  if (!s || !r) return QUOIN_ERR_NULL;
  if (r->op != QUOIN_B200_OP_COMPRESS && r->op != QUOIN_B200_OP_DECOMPRESS) return QUOIN_ERR_BAD_ARG;
  if (r->op == QUOIN_B200_OP_DECOMPRESS && (!r->idx || !r->d_src)) return QUOIN_ERR_NULL;
  try {
    uint64_t bytes = r->device_bytes + work_bytes(*r);
    r->done = 0;
    r->status = QUOIN_ERR_TIMEOUT;
    r->out_len = 0;
    r->t_submit_ns = s->now_ns();
    r->t_start_ns = r->t_end_ns = 0;
    if (!s->queue.push(r, bytes)) return QUOIN_ERR_OVER_BUDGET;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

extern "C" int quoin_b200_server_wait(QuoinServer* s, QuoinB200Request* r, int timeout_ms) {
  if (!s || !r) return QUOIN_ERR_NULL;
  std::unique_lock<std::mutex> l(s->done_mu);
  auto ready = [&] { return r->done != 0; };
  if (timeout_ms < 0) {
    s->done_cv.wait(l, ready);
  } else if (!s->done_cv.wait_for(l, std::chrono::milliseconds(timeout_ms), ready)) {
    return QUOIN_ERR_TIMEOUT;
  }
  return r->status;
}

extern "C" uint64_t quoin_b200_server_peak_bytes(QuoinServer* s) { return s ? s->queue.peak() : 0; }

extern "C" void quoin_b200_server_free(QuoinServer* s) {
  if (!s) return;
  s->queue.close();
  for (auto& t : s->workers) t.join();
  for (QuoinCtx* c : s->ctxs) quoin_ctx_free(c);
  delete s;
}
