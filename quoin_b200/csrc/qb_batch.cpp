// Many columns in one call (the batched configuration: columns of uneven
// length and mixed dtype).  A batch owns a pool of contexts, each with its own
// CUDA stream and device arenas; a call hands the columns, longest first, to
// one host worker per context, so the short columns' launch and
// synchronisation latencies overlap each other and the long columns' kernels
// on the GPU.  Every column's bytes are those of the single-column call.
#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#include "../../include/quoin.h"

struct QuoinBatch {
  std::vector<QuoinCtx*> ctxs;
};

extern "C" QuoinBatch* quoin_b200_batch_create(int workers) {
  try {
    if (workers < 1 || workers > 64) return nullptr;
    QuoinBatch* b = new QuoinBatch();
    for (int i = 0; i < workers; i++) {
      QuoinCtx* c = quoin_ctx_create(0);
      if (!c) {
        for (QuoinCtx* x : b->ctxs) quoin_ctx_free(x);
        delete b;
        return nullptr;
      }
      b->ctxs.push_back(c);
    }
    return b;
  } catch (...) {
    return nullptr;
  }
}

extern "C" void quoin_b200_batch_free(QuoinBatch* b) {
  if (!b) return;
  for (QuoinCtx* c : b->ctxs) quoin_ctx_free(c);
  delete b;
}

namespace {

// Runs work(ctx, job index) for every job on the batch's workers, jobs taken
// in `order`; returns the first failing job's status in job order, or OK.
template <class W>
int run_batch(QuoinBatch* b, size_t njobs, const std::vector<size_t>& order, std::vector<int>& status, W work) {
  std::atomic<size_t> next{0};
  auto worker = [&](QuoinCtx* c) {
    for (;;) {
      size_t k = next.fetch_add(1);
      if (k >= njobs) break;
      size_t j = order[k];
      try {
        status[j] = work(c, j);
      } catch (...) {
        status[j] = QUOIN_ERR_PANIC;
      }
    }
  };
  size_t nw = std::min(b->ctxs.size(), njobs);
  std::vector<std::thread> th;
  for (size_t i = 1; i < nw; i++) th.emplace_back(worker, b->ctxs[i]);
  if (nw) worker(b->ctxs[0]);
  for (auto& t : th) t.join();
  for (size_t j = 0; j < njobs; j++)
    if (status[j] != QUOIN_OK) return status[j];
  return QUOIN_OK;
}

template <class N>
std::vector<size_t> longest_first(size_t njobs, N size_of) {
  std::vector<size_t> order(njobs);
  for (size_t j = 0; j < njobs; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) { return size_of(a) > size_of(c); });
  return order;
}

}  // namespace

extern "C" int quoin_b200_compress_batch_device(QuoinBatch* b, QuoinB200CompressJob* jobs, size_t njobs,
                                                const QuoinConfig* cfg) {
  if (!b || (!jobs && njobs)) return QUOIN_ERR_NULL;
  try {
    std::vector<int> status(njobs, QUOIN_OK);
    auto order = longest_first(njobs, [&](size_t j) { return jobs[j].n; });
    return run_batch(b, njobs, order, status, [&](QuoinCtx* c, size_t j) {
      QuoinB200CompressJob& J = jobs[j];
      size_t len = 0;
      int rc = quoin_b200_compress_column_device(c, J.wire_dtype, J.n, J.d_values, J.d_validity, J.scale,
                                                 J.precision, cfg, J.d_dst, J.dst_cap, &len, nullptr);
      J.out_len = len;
      J.status = rc;
      return rc;
    });
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

extern "C" int quoin_b200_decompress_batch_device(QuoinBatch* b, QuoinB200DecompressJob* jobs, size_t njobs) {
  if (!b || (!jobs && njobs)) return QUOIN_ERR_NULL;
  try {
    std::vector<int> status(njobs, QUOIN_OK);
    std::vector<uint64_t> sizes(njobs, 0);
    for (size_t j = 0; j < njobs; j++) {
      int32_t wire = 0, hv = 0;
      uint64_t n = 0;
      if (jobs[j].idx && quoin_b200_index_info(jobs[j].idx, &wire, &n, &hv) == QUOIN_OK) sizes[j] = n;
    }
    auto order = longest_first(njobs, [&](size_t j) { return sizes[j]; });
    return run_batch(b, njobs, order, status, [&](QuoinCtx* c, size_t j) {
      QuoinB200DecompressJob& J = jobs[j];
      int rc = J.idx ? quoin_b200_decompress_indexed_device(c, J.idx, J.d_src, J.d_values_out, J.d_validity_out,
                                                             nullptr)
                     : QUOIN_ERR_NULL;
      J.status = rc;
      return rc;
    });
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}
