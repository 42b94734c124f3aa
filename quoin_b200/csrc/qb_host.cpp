// Host side of the B200 quoin library: stream format writer/reader
// (reference src/format.rs, src/decoder.rs:43-118, src/decimal.rs), column
// lowering orchestration (src/lib.rs:389-508), the GPU pipeline drivers and
// the C ABI of include/quoin.h (capi/src/lib.rs, capi/src/typed.rs).
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/quoin.h"
#include "qb_kernels.h"
#include "qb_layout.h"

namespace qb {

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }

}  // namespace qb

using namespace qb;

// ---------------------------------------------------------------------------
// Optional per-kernel-class CUDA-event timing (recorded on the launching
// stream, resolved after the call's final synchronisation).
// ---------------------------------------------------------------------------
namespace {
enum TimerClass { T_COMPETE = 0, T_EMIT, T_DECODE, T_FINALIZE, T_LOWER, T_PLAN, T_VALIDITY, T_OTHER, T_READ,
                  T_COUNT };
struct Timing {
  std::atomic<bool> on{false};
  std::mutex mu;
  double ms[T_COUNT] = {};
  uint64_t calls[T_COUNT] = {};
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
};
Timing g_timing;

cudaEvent_t take_event() {
  if (!g_timing.pool.empty()) {
    cudaEvent_t e = g_timing.pool.back();
    g_timing.pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

struct TimedRegion {
  int cls;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  TimedRegion(int c, cudaStream_t s) : cls(c), st(s) {
    if (!g_timing.on.load()) return;
    std::lock_guard<std::mutex> l(g_timing.mu);
    a = take_event();
    b = take_event();
    cudaEventRecord(a, st);
  }
  ~TimedRegion() {
    if (!a) return;
    cudaEventRecord(b, st);
    std::lock_guard<std::mutex> l(g_timing.mu);
    g_timing.pending.push_back({cls, {a, b}});
  }
};

// Called after a stream synchronisation: folds finished event pairs in.
void resolve_timing() {
  if (!g_timing.on.load()) return;
  std::lock_guard<std::mutex> l(g_timing.mu);
  for (auto& p : g_timing.pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(p.second.second) == cudaSuccess &&
        cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) {
      g_timing.ms[p.first] += ms;
      g_timing.calls[p.first] += 1;
    } else {
      cudaGetLastError();
    }
    g_timing.pool.push_back(p.second.first);
    g_timing.pool.push_back(p.second.second);
  }
  g_timing.pending.clear();
}
}  // namespace

namespace {

enum { WT_F64 = 0, WT_I64, WT_U64, WT_I32, WT_U32, WT_F32, WT_DEC128, WT_DEC256 };
enum { K_OK = 0, K_BAD_MAGIC = 1, K_VERSION = 2, K_TRUNC = 3, K_UNKNOWN_MODE = 4, K_CORRUPT = 5,
       K_LENGTH = 6, K_DTYPE = 7, K_DTYPE_MISMATCH = 8, K_UNSUPPORTED = 9 };
constexpr uint64_t kMaxBlockValues = 131072;
constexpr uint64_t kBaseQuantumH = 32768;
constexpr uint64_t kMaxBitmapBytes = 1ull << 36;
// Columns longer than this cannot be allocated on any host the reference runs
// on; its decoder reports the failed allocation as CorruptPayload.
constexpr uint64_t kMaxLogicalValues = 1ull << 36;

inline uint32_t lane_bytes_h(int dt) { return (dt == WT_I32 || dt == WT_U32 || dt == WT_F32) ? 4u : 8u; }
inline uint32_t native_width(int dt) {
  switch (dt) {
    case WT_I32: case WT_U32: case WT_F32: return 4;
    case WT_DEC128: return 16;
    case WT_DEC256: return 32;
    default: return 8;
  }
}
inline uint32_t varint_len_h(uint64_t v) {
  uint32_t n = 1;
  while (v >= 0x80) { v >>= 7; n++; }
  return n;
}
inline void put_varint_h(std::vector<uint8_t>& o, uint64_t v) {
  for (;;) {
    uint8_t b = (uint8_t)(v & 0x7f);
    v >>= 7;
    if (v) o.push_back(b | 0x80); else { o.push_back(b); return; }
  }
}
inline uint64_t rd64(const uint8_t* p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
  return v;
}
inline uint32_t rd32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
// LEB128 (reference varint.rs:24-39); returns a K_* kind.
int rd_varint_h(const uint8_t* p, uint64_t len, uint64_t* pos, uint64_t* out) {
  uint64_t r = 0;
  uint32_t shift = 0;
  for (;;) {
    if (*pos >= len) return K_TRUNC;
    uint8_t b = p[(*pos)++];
    r |= (uint64_t)(b & 0x7f) << shift;
    if (!(b & 0x80)) { *out = r; return K_OK; }
    shift += 7;
    if (shift >= 64) return K_CORRUPT;
  }
}
inline int kind_to_code(int kind) {
  switch (kind) {
    case K_OK: return QUOIN_OK;
    case K_BAD_MAGIC: return QUOIN_ERR_BAD_MAGIC;
    case K_VERSION: return QUOIN_ERR_UNSUPPORTED_VERSION;
    case K_TRUNC: return QUOIN_ERR_TRUNCATED;
    case K_UNKNOWN_MODE: return QUOIN_ERR_UNKNOWN_MODE;
    case K_CORRUPT: return QUOIN_ERR_CORRUPT_PAYLOAD;
    case K_LENGTH: return QUOIN_ERR_LENGTH_MISMATCH;
    case K_DTYPE: return QUOIN_ERR_UNSUPPORTED_DTYPE;
    case K_DTYPE_MISMATCH: return QUOIN_ERR_DTYPE_MISMATCH;
    default: return QUOIN_ERR_UNSUPPORTED;
  }
}
inline bool mode_known(int id) {  // reference mode.rs:60-84
  switch (id) {
    case 0: case 1: case 2: case 3: case 4: case 5: case 7: case 9: case 11: case 17:
    case 19: case 20: case 25: case 29: case 45: case 50: case 51: case 52: case 53: case 54:
      return true;
    default: return false;
  }
}
inline uint64_t popcount_bits(const uint8_t* bm, uint64_t n) {  // reference validity.rs:28-37
  uint64_t c = 0, full = n / 8;
  uint64_t i = 0;
  for (; i + 8 <= full; i += 8) {
    uint64_t w;
    memcpy(&w, bm + i, 8);
    c += (uint64_t)__builtin_popcountll(w);
  }
  for (; i < full; i++) c += (uint64_t)__builtin_popcount(bm[i]);
  uint64_t rem = n & 7;
  if (rem) c += (uint64_t)__builtin_popcount(bm[full] & ((1u << rem) - 1u));
  return c;
}
// Public code for the reference symbols.
inline int plain_code(int ext) {
  if (ext == QUOIN_OK || ext == QUOIN_ERR_NULL || ext == QUOIN_ERR_BUFFER_TOO_SMALL) return ext;
  if (ext == QUOIN_ERR_CUDA || ext == QUOIN_ERR_BAD_ARG) return QUOIN_ERR_PANIC;
  return QUOIN_ERR_CORRUPT;
}

}  // namespace

// ---------------------------------------------------------------------------
// Context: CUDA stream + grow-only device arenas.
// ---------------------------------------------------------------------------
enum Slot {
  S_IN, S_BM, S_RANK, S_LANE, S_GROW, S_FRAMES, S_NB, S_SIZES, S_TILE, S_SCRATCH, S_OUT, S_VTMP, S_VBLOB,
  S_MISC, S_LIMBS, S_LIMBOUT, S_SRC, S_DSCR, S_ERR, S_OUTVALS, S_DFRAMES, S_DBM, S_DRANK, S_DAUX, S_SUBST, S_FMST,
  S_SMP16, S_WINBITS, S_DSEL, S_DITEMS, S_PRE, S_ENT, S_ENTREC, S_DPMISC, S_DPCAND, S_DPJ, S_DPRUNS, S_BATCH, S_BSCR, S_BHOST, S_COUNT
};

struct QuoinCtx {
  int device = 0;
  cudaStream_t stream = nullptr;
  void* buf[S_COUNT] = {};
  size_t cap[S_COUNT] = {};
  std::mutex mu;
  QuoinDecodeIndex* hidx = nullptr;  // host-side parsed index reused by the host-buffer decodes
  uint64_t* hbox = nullptr;          // 512 B of pinned host memory for the small device -> host reads

  // Grows slot s to at least `bytes` (contents not kept).  The outgrown
  // buffer is retired, not freed: cudaFree waits for the whole device, which
  // would stall every other context's work (batches, the server); retired
  // buffers are freed when the context is, or when an allocation fails.
  // Growth at least doubles, so a slot's retired buffers stay below its size.
  cudaError_t ensure(int s, size_t bytes) {
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~(size_t)255;
    if (cap[s] >= bytes) return cudaSuccess;
    if (buf[s]) retired.push_back(buf[s]);
    buf[s] = nullptr;
    size_t want = bytes + bytes / 4;
    if (cap[s] && want < 2 * cap[s]) want = 2 * cap[s];
    cap[s] = 0;
    cudaError_t e = cudaMalloc(&buf[s], want);
    if (e != cudaSuccess) {  // free what was retired (after the device's work) and try the exact size
      cudaGetLastError();
      free_retired();
      e = cudaMalloc(&buf[s], bytes);
      want = bytes;
    }
    if (e == cudaSuccess) cap[s] = want; else cudaGetLastError();
    return e;
  }
  void free_retired() {
    if (retired.empty()) return;
    cudaDeviceSynchronize();
    for (void* p : retired) cudaFree(p);
    retired.clear();
  }
  std::vector<void*> retired;
  template <class T>
  T* p(int s) { return reinterpret_cast<T*>(buf[s]); }
};

namespace {

QuoinCtx* ctx_new() {
  QuoinCtx* c = new (std::nothrow) QuoinCtx();
  if (!c) return nullptr;
  if (cudaGetDevice(&c->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete c;
    return nullptr;
  }
  if (cudaHostAlloc(reinterpret_cast<void**>(&c->hbox), 512, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();  // reads then go to pageable memory
    c->hbox = nullptr;
  }
  return c;
}

// Reads `bytes` (at most 512) of device memory into host `out` and waits for
// the stream.  Through the context's pinned mailbox the copy is a plain DMA
// (a pageable destination takes the driver's staging path and its locks).
cudaError_t read_small(QuoinCtx* c, cudaStream_t st, void* out, const void* d_src, size_t bytes) {
  void* tgt = (c->hbox && bytes <= 512) ? static_cast<void*>(c->hbox) : out;
  cudaError_t e = cudaMemcpyAsync(tgt, d_src, bytes, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && tgt != out) memcpy(out, tgt, bytes);
  return e;
}

QuoinCtx* g_default = nullptr;
std::mutex g_default_mu;
QuoinCtx* default_ctx() {
  std::lock_guard<std::mutex> l(g_default_mu);
  if (!g_default) g_default = ctx_new();
  return g_default;
}
QuoinCtx* pick(const QuoinCtx* c) { return c ? const_cast<QuoinCtx*>(c) : default_ctx(); }

struct DeviceScope {
  int prev = -1;
  bool changed = false;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) {
      cudaSetDevice(dev);
      changed = true;
    }
  }
  ~DeviceScope() {
    if (changed) cudaSetDevice(prev);
  }
};

#define CK(x)                    \
  do {                           \
    cudaError_t _e = (x);        \
    if (_e != cudaSuccess) {     \
      cudaGetLastError();        \
      return QUOIN_ERR_CUDA;     \
    }                            \
  } while (0)

// ---------------------------------------------------------------------------
// Encoder pipeline
// ---------------------------------------------------------------------------
struct LaneJob {
  const uint64_t* lane;  // device, n_valid values
  uint64_t n_valid;
  int dtype;
  uint64_t logical_n;
  const uint8_t* d_bm;  // device bitmap when the column has nulls, else null
  int level;
  uint64_t block_size;  // 0 = adaptive, else clamped to [1, 131072]
  uint8_t plog2;
  bool vb_raw = false;  // the bitmap's transition count proves the RAW validity blob
};

uint64_t max_blocks_for(uint64_t n, uint64_t bs) {
  if (n == 0) return 0;
  return bs ? (n + bs - 1) / bs : (n + kBaseQuantumH - 1) / kBaseQuantumH;
}

// Bound on a lane stream's length: header, validity blob and, per block, a
// 9-byte frame header plus at most the RAW payload (RAW always competes and
// has no penalty, so no winner is longer).
uint64_t lane_bound(uint64_t n_valid, uint64_t logical_n, int dtype, bool validity, uint64_t bs) {
  uint64_t b = 16 + (validity ? 12 + (logical_n + 7) / 8 : 0);
  b += 9 * max_blocks_for(n_valid, bs) + (uint64_t)lane_bytes_h(dtype) * n_valid;
  return b + 64;
}

// Runs the GPU competition and emission for one lane (reference
// encoder.rs:184-214).  Writes the stream at d_dst and its length to *out_len.
// LaneJob::level carries Selection::Sample as kSelectSample beside the level.
constexpr int kSelectSample = 0x100;

int encode_lane(QuoinCtx* c, cudaStream_t st, const LaneJob& j, uint8_t* d_dst, size_t dst_cap, size_t* out_len) {
  const int level = j.level & 0xFF;
  const bool sample = (j.level & kSelectSample) != 0;
  uint64_t n = j.n_valid;
  uint64_t bs = j.block_size ? (j.block_size > kMaxBlockValues ? kMaxBlockValues : j.block_size) : 0;
  uint64_t maxb = max_blocks_for(n, bs);
  CK(c->ensure(S_MISC, 64 * 8));
  uint64_t* d_misc = c->p<uint64_t>(S_MISC);  // [0] frames base, [1] frames bytes, [2] blob len
  if (dst_cap < 16) {
    *out_len = lane_bound(n, j.logical_n, j.dtype, j.d_bm != nullptr, bs);
    return QUOIN_ERR_BUFFER_TOO_SMALL;
  }
  Bytes16 h;
  memcpy(h.b, "FCR1", 4);
  h.b[4] = 2;
  h.b[5] = j.d_bm ? 1 : 0;
  h.b[6] = j.plog2;
  h.b[7] = (uint8_t)j.dtype;
  for (int i = 0; i < 8; i++) h.b[8 + i] = (uint8_t)(j.logical_n >> (8 * i));
  launch_put_header(d_dst, h, d_misc, st);
  if (j.d_bm) {
    uint64_t ln = j.logical_n, nw = (ln + 31) / 32;
    uint64_t blob_cap = 1 + (ln + 7) / 8 + 16;
    if (dst_cap < 16 + 10 + blob_cap) {
      *out_len = lane_bound(n, ln, j.dtype, true, bs);
      return QUOIN_ERR_BUFFER_TOO_SMALL;
    }
    TimedRegion tr(T_VALIDITY, st);
    if (j.vb_raw) {
      launch_put_validity_raw(d_dst + 16, 16, j.d_bm, ln, d_misc, st);
    } else {
      CK(c->ensure(S_VTMP, (validity_tmp_words(ln) + scan_tile_count(nw) + 16) * 8));
      CK(c->ensure(S_VBLOB, blob_cap));
      uint64_t* vtmp = c->p<uint64_t>(S_VTMP);
      uint64_t* vtile = vtmp + validity_tmp_words(ln);
      launch_validity_blob(j.d_bm, ln, vtmp, vtile, c->p<uint8_t>(S_VBLOB), d_misc + 2, st);
      launch_put_validity(d_dst + 16, 16, c->p<uint8_t>(S_VBLOB), d_misc + 2, d_misc, st);
    }
  }
  if (maxb == 0) {
    uint64_t base = 0;
    CK(read_small(c, st, &base, d_misc, 8));
    *out_len = base;
    return QUOIN_OK;
  }
  CK(c->ensure(S_FRAMES, maxb * sizeof(FrameDesc)));
  CK(c->ensure(S_NB, 64));
  CK(c->ensure(S_SIZES, maxb * 8));
  CK(c->ensure(S_TILE, (scan_tile_count(maxb) + 16) * 8));
  CK(c->ensure(S_SCRATCH, n * kEncScratchPerValue + 256));
  uint64_t nwin = (n + kBaseQuantumH - 1) / kBaseQuantumH;
  uint64_t items = sub_stats_items(n, bs);
  bool fl = j.dtype == WT_F64 || j.dtype == WT_F32;
  CK(c->ensure(S_GROW, nwin + 16));
  CK(c->ensure(S_SUBST, (items + 1) * sub_stats_bytes()));
  CK(c->ensure(S_WINBITS, (nwin + 1) * kWinWords * 4));
  if (fl) {
    CK(c->ensure(S_FMST, (items + 1) * fm_stats_bytes()));
    CK(c->ensure(S_SMP16, (n / 16 + 2) * 8));
  }
  void* ent = nullptr;  // Balanced in-pool: the chosen rANS-coded parts per block
  if (level >= 2) {
    CK(c->ensure(S_ENTREC, maxb * ent_rec_bytes()));
    ent = c->p<void>(S_ENTREC);
  }
  FrameDesc* fr = c->p<FrameDesc>(S_FRAMES);
  uint32_t* nb = c->p<uint32_t>(S_NB);
  {
    TimedRegion tr(T_PLAN, st);
    launch_sub_stats(j.lane, n, bs, j.dtype, level, c->p<void>(S_SUBST), fl ? c->p<void>(S_FMST) : nullptr,
                     fl ? c->p<uint64_t>(S_SMP16) : nullptr, c->p<uint8_t>(S_GROW), c->p<uint32_t>(S_WINBITS), st);
    launch_plan(c->p<uint8_t>(S_GROW), n, bs, fr, nb, st);
  }
  {
    TimedRegion tr(T_COMPETE, st);
    launch_decide(j.lane, fr, nb, (uint32_t)maxb, bs, j.dtype, level, c->p<void>(S_SUBST),
                  fl ? c->p<void>(S_FMST) : nullptr, fl ? c->p<uint64_t>(S_SMP16) : nullptr,
                  c->p<uint32_t>(S_WINBITS), c->p<uint8_t>(S_SCRATCH), ent, sample, st);
  }
  {
    TimedRegion tr(T_OTHER, st);
    launch_frame_offsets(fr, nb, (uint32_t)maxb, d_misc, c->p<uint64_t>(S_SIZES), c->p<uint64_t>(S_TILE),
                         d_misc + 1, st);
  }
  {  // frames past dst_cap are skipped on the device; the total decides afterwards
    TimedRegion tr(T_EMIT, st);
    launch_emit(j.lane, fr, nb, (uint32_t)maxb, bs, j.dtype, c->p<void>(S_SUBST), fl ? c->p<void>(S_FMST) : nullptr,
                c->p<uint8_t>(S_SCRATCH), d_dst, dst_cap, ent, st);
  }
  uint64_t hm[2] = {0, 0};
  CK(read_small(c, st, hm, d_misc, 16));
  resolve_timing();
  uint64_t total = hm[0] + hm[1];
  *out_len = total;
  if (total > dst_cap) return QUOIN_ERR_BUFFER_TOO_SMALL;
  return QUOIN_OK;
}

// *level gets kSelectSample added for Selection::Sample (Fastest and Fast).
int check_level(const QuoinConfig* cfg, int* level, uint64_t* bs, uint8_t* plog2) {
  int lv = cfg ? cfg->level : QUOIN_LEVEL_FAST;
  int32_t sel = cfg ? cfg->selection : QUOIN_B200_SELECTION_FULL;
  if (sel != QUOIN_B200_SELECTION_FULL && sel != QUOIN_B200_SELECTION_SAMPLE) return QUOIN_ERR_BAD_ARG;
  if (lv == QUOIN_B200_LEVEL_BALANCED_INPOOL) {
    lv = QUOIN_LEVEL_BALANCED;  // Balanced's candidate pool without Lz and Pco
    if (sel == QUOIN_B200_SELECTION_SAMPLE) return QUOIN_ERR_UNSUPPORTED;
  } else {
    if (lv < 0 || lv > 4) return QUOIN_ERR_BAD_ARG;
    if (lv >= QUOIN_LEVEL_BALANCED) return QUOIN_ERR_UNSUPPORTED;
  }
  if (sel == QUOIN_B200_SELECTION_SAMPLE) lv |= kSelectSample;
  int64_t b = cfg ? cfg->block_size : 0;
  int32_t p = cfg ? cfg->predictor_log2 : 16;
  *level = lv;
  *bs = b <= 0 ? 0 : (uint64_t)b;
  *plog2 = (uint8_t)(p < 10 ? 10 : p > 16 ? 16 : p);  // reference lib.rs:236-238
  return QUOIN_OK;
}

// Count the valid bits of a device bitmap; fills S_RANK with per-word ranks.
// Valid count and word ranks of a device bitmap; *vb_raw tells whether the
// bitmap's transitions already prove the RAW validity blob (validity.rs:40-70).
int device_valid_count(QuoinCtx* c, cudaStream_t st, const uint8_t* d_bm, uint64_t n, uint64_t* n_valid,
                       bool* vb_raw) {
  uint64_t nw = (n + 31) / 32;
  CK(c->ensure(S_RANK, nw * 8 + 64));
  CK(c->ensure(S_TILE, (scan_tile_count(nw) + 16) * 8));
  CK(c->ensure(S_MISC, 64 * 8));
  uint64_t* rank = c->p<uint64_t>(S_RANK);
  uint64_t* misc = c->p<uint64_t>(S_MISC);
  {
    TimedRegion tr(T_VALIDITY, st);
    if (nw <= kSmallWords) {  // one launch for a short column
      launch_valid_small(d_bm, n, rank, misc + 8, reinterpret_cast<unsigned long long*>(misc + 9), st);
    } else {
      CK(cudaMemsetAsync(misc + 9, 0, 8, st));
      launch_word_popcount(d_bm, n, rank, st);
      launch_scan_sum(rank, rank, nw, c->p<uint64_t>(S_TILE), misc + 8, st);
      launch_bitmap_transitions(d_bm, n, reinterpret_cast<unsigned long long*>(misc + 9), st);
    }
  }
  uint64_t h[2] = {0, 0};
  CK(read_small(c, st, h, misc + 8, 16));
  *n_valid = h[0];
  *vb_raw = h[1] + 1 >= (n + 7) / 8;
  return QUOIN_OK;
}

uint64_t column_bound(int wire, uint64_t n, bool validity, uint64_t bs) {
  if (wire == WT_DEC128 || wire == WT_DEC256) {
    uint64_t nl = wire == WT_DEC128 ? 2 : 4;
    return 19 + 32 + (validity ? 12 + (n + 7) / 8 : 0) + nl * (10 + lane_bound(n, n, WT_U64, false, bs)) + 64;
  }
  return lane_bound(n, n, wire, validity, bs);
}

// Decimal container (reference decimal.rs:56-85, 174-212, 339-377).
int compress_decimal_device(QuoinCtx* c, cudaStream_t st, int wire, uint64_t n, const uint8_t* d_values,
                            const uint8_t* d_validity, int8_t scale, uint8_t precision, int level, uint64_t bs,
                            uint8_t plog2, uint8_t* d_dst, size_t dst_cap, size_t* out_len) {
  int nl = wire == WT_DEC128 ? 2 : 4;
  uint64_t n_valid = n;
  const uint8_t* d_bm = nullptr;
  bool vb_raw = false;
  if (d_validity && n) {
    int rc = device_valid_count(c, st, d_validity, n, &n_valid, &vb_raw);
    if (rc) return rc;
    if (n_valid < n) d_bm = d_validity;
  }
  CK(c->ensure(S_VTMP, (148 * 4 * 5 + 64) * 8));
  CK(c->ensure(S_MISC, 64 * 8));
  uint64_t* d_vmin = c->p<uint64_t>(S_MISC) + 16;
  launch_decimal_vmin(d_values, nl, d_bm, n, c->p<uint64_t>(S_VTMP), d_vmin, st);
  CK(c->ensure(S_LIMBS, (uint64_t)nl * n_valid * 8 + 64));
  uint64_t* limbs = c->p<uint64_t>(S_LIMBS);
  launch_decimal_split(d_values, nl, d_bm, d_bm ? c->p<uint64_t>(S_RANK) : nullptr, n, d_vmin, limbs, n_valid, st);
  uint64_t vmin[4] = {0, 0, 0, 0};
  CK(read_small(c, st, vmin, d_vmin, 32));
  std::vector<uint8_t> hdr;
  const char* magic = "FCR1";
  hdr.insert(hdr.end(), magic, magic + 4);
  hdr.push_back(2);
  hdr.push_back((uint8_t)(2 | (d_bm ? 1 : 0)));
  hdr.push_back(0);
  hdr.push_back((uint8_t)wire);
  for (int i = 0; i < 8; i++) hdr.push_back((uint8_t)(n >> (8 * i)));
  hdr.push_back((uint8_t)scale);
  hdr.push_back(precision);
  hdr.push_back((uint8_t)nl);
  for (int k = 0; k < nl; k++)
    for (int i = 0; i < 8; i++) hdr.push_back((uint8_t)(vmin[k] >> (8 * i)));
  uint64_t need_bound = column_bound(wire, n, d_bm != nullptr, bs);
  if (dst_cap < hdr.size()) {
    *out_len = need_bound;
    return QUOIN_ERR_BUFFER_TOO_SMALL;
  }
  CK(cudaMemcpyAsync(d_dst, hdr.data(), hdr.size(), cudaMemcpyHostToDevice, st));
  uint64_t pos = hdr.size();
  if (d_bm) {
    uint64_t nw = (n + 31) / 32;
    uint64_t blob_cap = 1 + (n + 7) / 8 + 16;
    if (dst_cap < pos + 10 + blob_cap) {
      *out_len = need_bound;
      return QUOIN_ERR_BUFFER_TOO_SMALL;
    }
    uint64_t* d_misc = c->p<uint64_t>(S_MISC);
    if (vb_raw) {
      launch_put_validity_raw(d_dst + pos, pos, d_bm, n, d_misc + 3, st);
    } else {
      CK(c->ensure(S_VTMP, (validity_tmp_words(n) + scan_tile_count(nw) + 16) * 8));
      CK(c->ensure(S_VBLOB, blob_cap));
      uint64_t* vtmp = c->p<uint64_t>(S_VTMP);
      launch_validity_blob(d_bm, n, vtmp, vtmp + validity_tmp_words(n), c->p<uint8_t>(S_VBLOB), d_misc + 2, st);
      launch_put_validity(d_dst + pos, pos, c->p<uint8_t>(S_VBLOB), d_misc + 2, d_misc + 3, st);
    }
    uint64_t np = 0;
    CK(read_small(c, st, &np, d_misc + 3, 8));
    pos = np;
  }
  uint64_t sub_cap = lane_bound(n_valid, n_valid, WT_U64, false, bs);
  CK(c->ensure(S_LIMBOUT, sub_cap));
  for (int k = 0; k < nl; k++) {
    LaneJob j{limbs + (uint64_t)k * n_valid, n_valid, WT_U64, n_valid, nullptr, level, bs, plog2};
    size_t sl = 0;
    int rc = encode_lane(c, st, j, c->p<uint8_t>(S_LIMBOUT), sub_cap, &sl);
    if (rc) return rc;
    std::vector<uint8_t> vl;
    put_varint_h(vl, sl);
    if (pos + vl.size() + sl > dst_cap) {
      *out_len = need_bound;
      return QUOIN_ERR_BUFFER_TOO_SMALL;
    }
    CK(cudaMemcpyAsync(d_dst + pos, vl.data(), vl.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_dst + pos + vl.size(), c->p<uint8_t>(S_LIMBOUT), sl, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    pos += vl.size() + sl;
  }
  *out_len = pos;
  return QUOIN_OK;
}

// compress_column (reference lib.rs:429-455) with device buffers.
// Lowers a non-decimal column to its lane (valid values as u64) on the
// device, as compress_column_device does; *lane points at the input itself
// when no copy is needed.
int lower_column(QuoinCtx* c, cudaStream_t st, int wire, uint64_t n, const void* d_values,
                 const uint8_t* d_validity, const uint64_t** lane, uint64_t* n_valid, const uint8_t** d_bm,
                 bool* vb_raw) {
  *n_valid = n;
  *d_bm = nullptr;
  *vb_raw = false;
  if (d_validity && n) {
    int rc = device_valid_count(c, st, d_validity, n, n_valid, vb_raw);
    if (rc) return rc;
    if (*n_valid < n) *d_bm = d_validity;
  }
  bool direct = !*d_bm && lane_bytes_h(wire) == 8 && wire != WT_F32 && ((uintptr_t)d_values & 7) == 0;
  if (direct) {
    *lane = (const uint64_t*)d_values;
    return QUOIN_OK;
  }
  CK(c->ensure(S_LANE, *n_valid * 8 + 64));
  TimedRegion tr(T_LOWER, st);
  launch_lower(d_values, wire, *d_bm, *d_bm ? c->p<uint64_t>(S_RANK) : nullptr, n, c->p<uint64_t>(S_LANE), st);
  *lane = c->p<uint64_t>(S_LANE);
  return QUOIN_OK;
}

int compress_column_device(QuoinCtx* c, cudaStream_t st, int wire, uint64_t n, const void* d_values,
                           const uint8_t* d_validity, int8_t scale, uint8_t precision, const QuoinConfig* cfg,
                           uint8_t* d_dst, size_t dst_cap, size_t* out_len) {
  if (wire < 0 || wire > 7) return QUOIN_ERR_BAD_ARG;
  int level;
  uint64_t bs;
  uint8_t plog2;
  int rc = check_level(cfg, &level, &bs, &plog2);
  if (rc) return rc;
  if (wire == WT_DEC128 || wire == WT_DEC256)
    return compress_decimal_device(c, st, wire, n, (const uint8_t*)d_values, d_validity, scale, precision, level, bs,
                                   plog2, d_dst, dst_cap, out_len);
  uint64_t n_valid = n;
  const uint8_t* d_bm = nullptr;
  bool vb_raw = false;
  const uint64_t* lane = nullptr;
  rc = lower_column(c, st, wire, n, d_values, d_validity, &lane, &n_valid, &d_bm, &vb_raw);
  if (rc) return rc;
  LaneJob j{lane, n_valid, wire, n, d_bm, level, bs, plog2, vb_raw};
  return encode_lane(c, st, j, d_dst, dst_cap, out_len);
}

// The block plan's window probe over a column's lane (reference
// encoder.rs:154-178, probe_block_features encoder.rs:705-750): one byte per
// 32,768-value window of the valid values, 1 where plan_blocks grows a block
// starting at that window to 131,072 values.  The plan itself is a scan over
// these bytes, so a column split at window boundaries can be probed in parts.
int probe_windows_device(QuoinCtx* c, cudaStream_t st, int wire, uint64_t n, const void* d_values,
                         const uint8_t* d_validity, uint8_t* grow_out, uint64_t grow_cap, uint64_t* n_windows) {
  if (wire < 0 || wire > 7) return QUOIN_ERR_BAD_ARG;
  if (wire == WT_DEC128 || wire == WT_DEC256) return QUOIN_ERR_UNSUPPORTED;
  const uint64_t* lane = nullptr;
  uint64_t nv = 0;
  const uint8_t* d_bm = nullptr;
  bool vb_raw = false;
  int rc = lower_column(c, st, wire, n, d_values, d_validity, &lane, &nv, &d_bm, &vb_raw);
  if (rc) return rc;
  uint64_t nwin = (nv + kBaseQuantumH - 1) / kBaseQuantumH;
  *n_windows = nwin;
  if (nwin > grow_cap) return QUOIN_ERR_BUFFER_TOO_SMALL;
  if (!nwin) return QUOIN_OK;
  uint64_t items = sub_stats_items(nv, 0);
  bool fl = wire == WT_F64 || wire == WT_F32;
  CK(c->ensure(S_GROW, nwin + 16));
  CK(c->ensure(S_SUBST, (items + 1) * sub_stats_bytes()));
  CK(c->ensure(S_WINBITS, (nwin + 1) * kWinWords * 4));
  if (fl) {
    CK(c->ensure(S_FMST, (items + 1) * fm_stats_bytes()));
    CK(c->ensure(S_SMP16, (nv / 16 + 2) * 8));
  }
  {
    TimedRegion tr(T_PLAN, st);
    launch_sub_stats(lane, nv, 0, wire, QUOIN_LEVEL_FAST, c->p<void>(S_SUBST), fl ? c->p<void>(S_FMST) : nullptr,
                     fl ? c->p<uint64_t>(S_SMP16) : nullptr, c->p<uint8_t>(S_GROW), c->p<uint32_t>(S_WINBITS), st);
  }
  CK(cudaMemcpyAsync(grow_out, c->p<uint8_t>(S_GROW), nwin, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  resolve_timing();
  for (uint64_t w = 0; w < nwin; w++) grow_out[w] = grow_out[w] ? 1 : 0;
  return QUOIN_OK;
}

// The bytes of a stream before its first frame (reference encoder.rs:184-214):
// the 16-byte header and, when the column has nulls, the validity blob.
int stream_prefix_device(QuoinCtx* c, cudaStream_t st, int wire, uint64_t n, const uint8_t* d_validity,
                         const QuoinConfig* cfg, uint8_t* d_dst, size_t dst_cap, size_t* out_len) {
  if (wire < 0 || wire > 7) return QUOIN_ERR_BAD_ARG;
  if (wire == WT_DEC128 || wire == WT_DEC256) return QUOIN_ERR_UNSUPPORTED;
  int level;
  uint64_t bs;
  uint8_t plog2;
  int rc = check_level(cfg, &level, &bs, &plog2);
  if (rc) return rc;
  uint64_t n_valid = n;
  const uint8_t* d_bm = nullptr;
  bool vb_raw = false;
  if (d_validity && n) {
    rc = device_valid_count(c, st, d_validity, n, &n_valid, &vb_raw);
    if (rc) return rc;
    if (n_valid < n) d_bm = d_validity;
  }
  LaneJob j{nullptr, 0, wire, n, d_bm, level, bs, plog2, vb_raw};  // no values: no frames
  return encode_lane(c, st, j, d_dst, dst_cap, out_len);
}

// ---------------------------------------------------------------------------
// Decoder: host-side header / validity / frame walk (reference
// decoder.rs:43-94, decimal.rs:100-168), device decode.
// ---------------------------------------------------------------------------
struct LaneIdx {
  int dtype = 0;
  uint32_t plog2 = 16;  // header byte 6 (format.rs:56-94): the FCM / DFCM table size
  uint64_t logical_n = 0, n_total = 0;
  bool has_validity = false;
  std::vector<uint8_t> bitmap;  // ceil(n/8), trailing bits cleared
  std::vector<FrameDesc> frames;
  bool any_dict = false;  // frames that need the decode scratch range (DICT, RLE, ALP-RD)
  uint64_t frame_base = 0;
  // warp-item decode tables (launch_decode_items) and their offsets in the
  // index-wide device table
  std::vector<ItemRef> pre_items, main_items;
  std::vector<uint2> frame_pre;
  std::vector<uint32_t> list;
  bool need_scan = false;
  uint64_t ent_bytes = 0;  // device area for the entropy-coded parts of listed frames
  uint64_t main_base = 0, pre_base = 0, fp_base = 0, list_base = 0;  // index of the first frame in the device table
  // table sizes the decode launches use (the vectors' sizes after a host
  // parse; the device reader's counts when the tables were built on the device)
  uint64_t nf = 0, nmain = 0, npre = 0, nlist = 0;

  // Back to the empty state, keeping every buffer's capacity (a context
  // reuses its parsed index, so repeated decodes touch no fresh pages).
  void reset() {
    dtype = 0;
    plog2 = 16;
    logical_n = n_total = 0;
    has_validity = false;
    bitmap.clear();
    frames.clear();
    any_dict = false;
    frame_base = 0;
    pre_items.clear();
    main_items.clear();
    frame_pre.clear();
    list.clear();
    need_scan = false;
    ent_bytes = 0;
    main_base = pre_base = fp_base = list_base = 0;
    nf = nmain = npre = nlist = 0;
  }
  void take_counts() {
    nf = frames.size();
    nmain = main_items.size();
    npre = pre_items.size();
    nlist = list.size();
  }
};

// Reference validity.rs:73-119.
int validity_decode_h(const uint8_t* blob, uint64_t blen, uint64_t n, std::vector<uint8_t>& bm) {
  uint64_t raw_len = (n + 7) / 8;
  if (n > UINT64_MAX - 7 || raw_len > kMaxBitmapBytes) return K_CORRUPT;
  if (blen == 0) return K_TRUNC;
  uint8_t tag = blob[0];
  const uint8_t* rest = blob + 1;
  uint64_t rlen = blen - 1;
  if (tag == 0) {
    if (rlen < raw_len) return K_TRUNC;
    bm.assign(rest, rest + raw_len);
    if (n & 7) bm[raw_len - 1] &= (uint8_t)((1u << (n & 7)) - 1u);
    return K_OK;
  }
  if (tag == 1) {
    bm.assign(raw_len, 0);
    uint64_t pos = 0, i = 0;
    int cur = 0;
    while (i < n) {
      uint64_t run;
      int k = rd_varint_h(rest, rlen, &pos, &run);
      if (k) return k;
      if (run > n - i) return K_CORRUPT;
      uint64_t end = i + run;
      if (cur == 1) {
        uint64_t a = i;
        while (a < end && (a & 7)) { bm[a >> 3] |= (uint8_t)(1u << (a & 7)); a++; }
        uint64_t full_end = end & ~7ull;
        if (a < full_end) { memset(bm.data() + (a >> 3), 0xFF, (full_end - a) >> 3); a = full_end; }
        while (a < end) { bm[a >> 3] |= (uint8_t)(1u << (a & 7)); a++; }
      }
      i = end;
      cur ^= 1;
    }
    return K_OK;
  }
  return K_CORRUPT;
}

// Reference format.rs:65-94 + decoder.rs:43-94 for the lane stream at
// src[base .. base + len).  Frame payload offsets are relative to `src`.
int parse_lane(const uint8_t* src, uint64_t base, uint64_t len, LaneIdx& L) {
  const uint8_t* s = src + base;
  if (len < 16) return K_TRUNC;
  if (memcmp(s, "FCR1", 4) != 0) return K_BAD_MAGIC;
  if (s[4] != 2) return K_VERSION;
  if (s[5] & ~1u) return K_CORRUPT;
  if (s[6] < 10 || s[6] > 16) return K_CORRUPT;
  if (s[7] > 7) return K_DTYPE;
  L.dtype = s[7];
  L.plog2 = s[6];
  L.has_validity = s[5] & 1;
  L.logical_n = rd64(s + 8);
  if (L.logical_n > kMaxLogicalValues) return K_CORRUPT;  // decoder.rs:105-106 / validity.rs:135-136 allocation
  uint64_t pos = 16;
  L.n_total = L.logical_n;
  if (L.has_validity) {
    uint64_t vlen;
    int k = rd_varint_h(s, len, &pos, &vlen);
    if (k) return k;
    if (vlen > len - pos) return K_TRUNC;
    k = validity_decode_h(s + pos, vlen, L.logical_n, L.bitmap);
    if (k) return k;
    pos += vlen;
    L.n_total = popcount_bits(L.bitmap.data(), L.logical_n);
  }
  uint64_t counted = 0;
  while (counted < L.n_total) {
    if (len - pos < 9) return K_TRUNC;
    int mode = s[pos];
    if (!mode_known(mode)) return K_UNKNOWN_MODE;
    uint64_t fn = rd32(s + pos + 1), plen = rd32(s + pos + 5);
    pos += 9;
    if (fn > kMaxBlockValues) return K_CORRUPT;
    if (len - pos < plen) return K_TRUNC;
    FrameDesc f;
    f.payload_off = base + pos;
    f.value_off = counted;
    f.n = (uint32_t)fn;
    f.plen = (uint32_t)plen;
    f.mode = (uint32_t)mode;
    f.aux = 0;
    L.frames.push_back(f);
    if (mode == 19 || mode == 53 || mode == 52) L.any_dict = true;
    pos += plen;
    counted += fn;
    if (counted > L.n_total) return K_CORRUPT;
  }
  return K_OK;
}

// ALP-RD header up to the rights tag (reference alp_rd.rs:208-250): the
// exception count and the two part tags; false when it does not parse here
// (the device walk then reports the error).
bool alprd_tags_h(const uint8_t* p, uint64_t plen, uint64_t* nexc, uint32_t* ctag, uint32_t* rtag) {
  if (plen < 2 || p[1] > 8) return false;
  uint64_t pos = 2 + 8ull * p[1], clen = 0;
  if (pos > plen || rd_varint_h(p, plen, &pos, nexc) != K_OK) return false;
  for (uint64_t x = 0; x < *nexc; x++) {
    uint64_t pp;
    if (rd_varint_h(p, plen, &pos, &pp) != K_OK || plen - pos < 8) return false;
    pos += 8;
  }
  if (pos >= plen) return false;
  *ctag = p[pos++];
  if (rd_varint_h(p, plen, &pos, &clen) != K_OK || clen > plen - pos) return false;
  pos += clen;
  if (pos >= plen) return false;
  *rtag = p[pos];
  return true;
}

// Whether a frame may hold an entropy-coded part (Balanced and above: the
// rANS stage of entropy/mod.rs:152-178), decoded by the frame kernel in a
// device area of its own.  Errs on the side of yes when the header does not
// parse: BYTE_TRANSPOSE always; FLOAT_MULT tag 1 (float_mult.rs:100-133);
// ALP-RD codes or rights tag 1; DICT values tag 2 or codes tag 1
// (dict.rs:154-207).
bool entropy_frame_h(const uint8_t* p, uint64_t plen, uint32_t mode) {
  switch (mode) {
    case 11: case 7: case 20: case 45:  // BYTE_TRANSPOSE; ORDERED_DELTA, DELTA2, DELTA_DP (linear.rs)
    case 0: case 25: case 29:           // PRED, PRED2, PRED_RC (pred.rs; PRED needs only the table)
    case 4:                             // LZ (lz.rs)
      return true;
    case 17:
      return plen < 2 || p[0] == 1;
    case 52: {
      uint64_t nexc = 0;
      uint32_t ct = 0, rt = 0;
      return !alprd_tags_h(p, plen, &nexc, &ct, &rt) || ct == 1 || rt == 1;
    }
    case 19: {
      uint64_t pos = 0, card = 0, vlen = 0;
      if (rd_varint_h(p, plen, &pos, &card) != K_OK || pos >= plen) return true;
      uint32_t vtag = p[pos++];
      if (vtag == 2) return true;
      if (rd_varint_h(p, plen, &pos, &vlen) != K_OK || vlen > plen - pos) return true;
      pos += vlen;
      return pos >= plen || p[pos] == 1;
    }
    default:
      return false;
  }
}

// Warp items of every frame (512 values, or kXorzItemBytes payload bytes for XORZ).
// Frames the items do not cover, or whose header cannot be read here, go to
// the frame list; the device walk reports their errors.  Listed frames with
// an entropy-coded part get a device area (ent_area_bytes: the mode's layout,
// the range coder's model, a predictor table, the LZ cascade's scratch)
// (128-byte units, 1 + its offset in FrameDesc::aux; 0 = none).
void build_items(const uint8_t* src, LaneIdx& L) {
  const uint32_t V = 512, B = 512;
  {  // one reservation (items of 512 values or 512+ XORZ bytes, prepass items at most as many)
    uint64_t est = 0;
    for (const FrameDesc& d : L.frames) est += (d.n + V - 1) / V + (d.plen + B - 1) / B;
    L.main_items.reserve(est);
    L.pre_items.reserve(est);
    L.frame_pre.reserve(L.frames.size());
  }
  for (uint32_t f = 0; f < (uint32_t)L.frames.size(); f++) {
    const FrameDesc& d = L.frames[f];
    const uint8_t* p = src + d.payload_off;
    uint64_t n = d.n, plen = d.plen;
    uint32_t pre0 = (uint32_t)L.pre_items.size();
    uint32_t nv = (uint32_t)((n + V - 1) / V);
    auto add_main = [&](uint32_t cnt) {
      for (uint32_t j = 0; j < cnt; j++) L.main_items.push_back(ItemRef{f, j});
    };
    auto add_pre = [&](uint32_t cnt) {
      for (uint32_t j = 0; j < cnt; j++) L.pre_items.push_back(ItemRef{f, j});
    };
    switch (d.mode) {
      case 5: case 1: case 2: case 50: case 9:  // RAW CONST STRIDE FOR ALP
        add_main(nv);
        break;
      case 17:  // FLOAT_MULT: items for the bit-packed form (tag 0)
        if (plen >= 2 && p[0] == 0) add_main(nv);
        else L.list.push_back(f);
        break;
      case 51:  // DELTA
        add_pre(nv);
        add_main(nv);
        L.need_scan = true;
        break;
      case 3: {  // XORZ
        uint32_t nb = (uint32_t)((plen + kXorzItemBytes - 1) / kXorzItemBytes);
        add_pre(nb);
        add_main(nb);
        L.need_scan = true;
        break;
      }
      case 53: {  // RLE: varint(nruns) first
        uint64_t pos = 0, nr = 0;
        if (rd_varint_h(p, plen, &pos, &nr) != K_OK || nr > n) {
          L.list.push_back(f);
          break;
        }
        add_pre((uint32_t)((nr + 1023) / 1024));
        add_main(nv);
        L.need_scan = true;
        break;
      }
      case 52: {  // ALP-RD: items only without exceptions and with both parts bit-packed
        uint64_t nexc = 1;
        uint32_t ct = 1, rt = 1;
        if (alprd_tags_h(p, plen, &nexc, &ct, &rt) && nexc == 0 && ct == 0 && rt == 0) add_main(nv);
        else L.list.push_back(f);
        break;
      }
      default:
        L.list.push_back(f);
        break;
    }
    L.frame_pre.push_back(make_uint2(pre0, (uint32_t)L.pre_items.size() - pre0));
  }
  for (uint32_t f : L.list) {
    FrameDesc& d = L.frames[f];
    if (!entropy_frame_h(src + d.payload_off, d.plen, d.mode)) continue;
    d.aux = (uint32_t)(1 + L.ent_bytes / 128);
    L.ent_bytes += ent_area_bytes(d.n, d.mode, L.plog2);
  }
}

// Bytes of the index-wide item table; assigns each lane's offsets.
uint64_t layout_items(std::vector<LaneIdx>& lanes) {
  uint64_t m = 0, pr = 0, fp = 0, li = 0;
  for (auto& L : lanes) {
    L.main_base = m;
    L.pre_base = pr;
    L.fp_base = fp;
    L.list_base = li;
    m += L.main_items.size();
    pr += L.pre_items.size();
    fp += L.frame_pre.size();
    li += L.list.size();
  }
  for (auto& L : lanes) {
    L.pre_base += m;
    L.fp_base = m + pr + L.fp_base;
    L.list_base = m + pr + fp + L.list_base;
  }
  return (m + pr + fp + li) * 8 + 64;  // ItemRef / uint2 are 8 bytes, list entries padded to 8
}

}  // namespace

cudaStream_t qb::ctx_stream(QuoinCtx* c, void* stream) {
  if (stream) return static_cast<cudaStream_t>(stream);
  QuoinCtx* x = pick(c);
  return x ? x->stream : nullptr;
}

struct QuoinDecodeIndex {
  int wire = 0;
  uint64_t n = 0;
  bool has_validity = false, decimal = false;
  int8_t scale = 0;
  uint8_t precision = 0;
  int nl = 0;
  uint64_t vmin[4] = {0, 0, 0, 0};
  uint64_t n_valid = 0;
  std::vector<uint8_t> bitmap;  // logical bitmap (decimal container or lane)
  std::vector<LaneIdx> lanes;
  // device copies (owned when `owned`)
  bool owned = false;
  int device = 0;
  FrameDesc* d_frames = nullptr;
  uint8_t* d_bm = nullptr;
  uint64_t* d_rank = nullptr;
  uint64_t* d_sel = nullptr;
  uint64_t* d_vmin = nullptr;
  uint64_t* d_items = nullptr;  // item tables of every lane (layout_items)
  uint64_t items_bytes = 0;
  uint64_t max_pre = 0;
};

namespace {

int parse_stream_lanes(const uint8_t* src, uint64_t len, QuoinDecodeIndex& X);

// Reference lib.rs:462-490 + decimal.rs:100-168: parse a whole stream, then lay
// out the warp-item tables of its lanes.
int parse_stream(const uint8_t* src, uint64_t len, QuoinDecodeIndex& X) {
  int k = parse_stream_lanes(src, len, X);
  if (k) return k;
  X.items_bytes = layout_items(X.lanes);
  X.max_pre = 0;
  for (auto& L : X.lanes) {
    L.take_counts();
    X.max_pre = L.npre > X.max_pre ? L.npre : X.max_pre;
  }
  return K_OK;
}

// Lane k of X, emptied (its buffers keep their capacity).
LaneIdx& lane_slot(QuoinDecodeIndex& X, size_t k) {
  if (X.lanes.size() <= k) X.lanes.resize(k + 1);
  X.lanes[k].reset();
  return X.lanes[k];
}

// The header, validity and frame tables of the stream's lane(s).  X may be a
// reused host index: every field is set again.
int parse_stream_lanes(const uint8_t* src, uint64_t len, QuoinDecodeIndex& X) {
  X.wire = 0;
  X.n = 0;
  X.has_validity = false;
  X.decimal = false;
  X.scale = 0;
  X.precision = 0;
  X.nl = 0;
  for (auto& m : X.vmin) m = 0;
  X.n_valid = 0;
  X.bitmap.clear();
  X.items_bytes = 0;
  X.max_pre = 0;
  size_t nlanes = 0;
  struct Trim {  // lanes beyond the parsed ones are dropped on every return
    QuoinDecodeIndex& X;
    size_t& n;
    ~Trim() {
      if (X.lanes.size() > n) X.lanes.resize(n);
    }
  } trim{X, nlanes};
  if (len > 5 && (src[5] & 2)) {  // decimal container (decimal.rs:39-41)
    if (len < 8) return K_TRUNC;
    if (src[7] > 7) return K_DTYPE;
    int expect = src[7] == WT_DEC256 ? WT_DEC256 : WT_DEC128;
    if (len < 19) return K_TRUNC;
    if (memcmp(src, "FCR1", 4) != 0) return K_BAD_MAGIC;
    if (src[4] != 2) return K_VERSION;
    if (src[7] != expect) return K_DTYPE_MISMATCH;
    X.decimal = true;
    X.wire = expect;
    X.has_validity = src[5] & 1;
    X.n = rd64(src + 8);
    if (X.n > kMaxLogicalValues) return K_CORRUPT;
    X.scale = (int8_t)src[16];
    X.precision = src[17];
    int nl = src[18];
    if (nl == 0 || nl > 4) return K_CORRUPT;
    uint64_t vmin_off = 19, pos = 19 + (uint64_t)nl * 8;
    if (pos > len) return K_TRUNC;
    X.n_valid = X.n;
    if (X.has_validity) {
      uint64_t vlen;
      int k = rd_varint_h(src, len, &pos, &vlen);
      if (k) return k;
      if (vlen > len - pos) return K_TRUNC;
      k = validity_decode_h(src + pos, vlen, X.n, X.bitmap);
      if (k) return k;
      pos += vlen;
      X.n_valid = popcount_bits(X.bitmap.data(), X.n);
    }
    for (int k = 0; k < nl; k++) {
      uint64_t sl;
      int r = rd_varint_h(src, len, &pos, &sl);
      if (r) return r;
      if (sl > len - pos) return K_TRUNC;
      LaneIdx& L = lane_slot(X, nlanes++);
      r = parse_lane(src, pos, sl, L);
      if (r) return r;
      build_items(src, L);
      if (L.logical_n != X.n_valid) return K_CORRUPT;
      pos += sl;
    }
    int want = expect == WT_DEC128 ? 2 : 4;
    if (nl != want) return K_CORRUPT;
    X.nl = nl;
    for (int k = 0; k < nl; k++) X.vmin[k] = rd64(src + vmin_off + 8 * k);
    return K_OK;
  }
  LaneIdx& L = lane_slot(X, nlanes++);
  int r = parse_lane(src, 0, len, L);
  if (r) return r;
  build_items(src, L);
  if (L.dtype == WT_DEC128 || L.dtype == WT_DEC256) return K_CORRUPT;  // lib.rs:503-505
  X.wire = L.dtype;
  X.n = L.logical_n;
  X.has_validity = L.has_validity;
  X.bitmap.swap(L.bitmap);  // the stream's bitmap is the column's
  X.n_valid = L.n_total;
  return K_OK;
}

uint64_t total_frames(const QuoinDecodeIndex& X) {
  uint64_t t = 0;
  for (auto& L : X.lanes) t += L.frames.size();
  return t;
}

// Upload the index tables into device buffers (dfr, dbm, drank, dvmin) and
// compute the validity word ranks on the device.
uint64_t sel_bytes(const QuoinDecodeIndex& X) {
  uint64_t nv = X.decimal || X.lanes.empty() ? 0 : X.lanes[0].n_total;
  return (nv / 512 + 2) * 8;
}

int upload_index(QuoinCtx* c, cudaStream_t st, QuoinDecodeIndex& X, FrameDesc* dfr, uint8_t* dbm, uint64_t* drank,
                 uint64_t* dsel, uint64_t* dvmin, uint64_t* ditems) {
  uint64_t fb = 0;
  for (auto& L : X.lanes) {
    L.frame_base = fb;
    if (!L.frames.empty())
      CK(cudaMemcpyAsync(dfr + fb, L.frames.data(), L.frames.size() * sizeof(FrameDesc), cudaMemcpyHostToDevice, st));
    fb += L.frames.size();
  }
  std::vector<uint64_t> tab(X.items_bytes / 8, 0);
  for (auto& L : X.lanes) {
    if (!L.main_items.empty()) memcpy(tab.data() + L.main_base, L.main_items.data(), L.main_items.size() * 8);
    if (!L.pre_items.empty()) memcpy(tab.data() + L.pre_base, L.pre_items.data(), L.pre_items.size() * 8);
    if (!L.frame_pre.empty()) memcpy(tab.data() + L.fp_base, L.frame_pre.data(), L.frame_pre.size() * 8);
    if (!L.list.empty()) memcpy(tab.data() + L.list_base, L.list.data(), L.list.size() * 4);
  }
  if (!tab.empty()) CK(cudaMemcpyAsync(ditems, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, st));
  if (X.has_validity && X.n) {
    uint64_t nw = (X.n + 31) / 32;
    CK(cudaMemcpyAsync(dbm, X.bitmap.data(), X.bitmap.size(), cudaMemcpyHostToDevice, st));
    CK(c->ensure(S_TILE, (scan_tile_count(nw) + 16) * 8));
    launch_word_popcount(dbm, X.n, drank, st);
    launch_scan_sum(drank, drank, nw, c->p<uint64_t>(S_TILE), nullptr, st);
    if (!X.decimal) launch_select_table(dbm, X.n, drank, X.lanes[0].n_total, dsel, st);
  }
  if (X.decimal) CK(cudaMemcpyAsync(dvmin, X.vmin, 32, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  return QUOIN_OK;
}

// Decode the lanes of an uploaded index from the device stream d_src.
ItemPlan lane_plan(const LaneIdx& L, const uint64_t* ditems) {
  ItemPlan P;
  P.main_items = reinterpret_cast<const ItemRef*>(ditems + L.main_base);
  P.nmain = (uint32_t)L.nmain;
  P.pre_items = reinterpret_cast<const ItemRef*>(ditems + L.pre_base);
  P.npre = (uint32_t)L.npre;
  P.frame_pre = reinterpret_cast<const uint2*>(ditems + L.fp_base);
  P.list = reinterpret_cast<const uint32_t*>(ditems + L.list_base);
  P.nlist = (uint32_t)L.nlist;
  P.need_scan = L.need_scan;
  P.ent = nullptr;
  return P;
}

int decode_indexed(QuoinCtx* c, cudaStream_t st, const QuoinDecodeIndex& X, const FrameDesc* dfr, const uint8_t* dbm,
                   const uint64_t* drank, const uint64_t* dsel, const uint64_t* dvmin, const uint64_t* ditems,
                   const uint8_t* d_src, void* d_out, uint8_t* d_valid_out) {
  CK(c->ensure(S_ERR, 64));
  unsigned long long* d_err = c->p<unsigned long long>(S_ERR);
  CK(cudaMemsetAsync(d_err, 0xFF, 8, st));
  const uint8_t* bm = X.has_validity ? dbm : nullptr;
  uint64_t max_nf = 1;
  for (auto& L : X.lanes) max_nf = L.nf > max_nf ? L.nf : max_nf;
  CK(c->ensure(S_DAUX, decode_aux_bytes((int)max_nf)));
  void* daux = c->p<void>(S_DAUX);
  CK(c->ensure(S_PRE, (X.max_pre + 1) * prepass_rec_bytes()));
  void* dpre = c->p<void>(S_PRE);
  uint64_t ent_bytes = 0;  // lanes decode one after another on the stream: one area serves all
  for (auto& L : X.lanes) ent_bytes = L.ent_bytes > ent_bytes ? L.ent_bytes : ent_bytes;
  uint8_t* dent = nullptr;
  if (ent_bytes) {
    CK(c->ensure(S_ENT, ent_bytes));
    dent = c->p<uint8_t>(S_ENT);
  }
  auto plan_of = [&](const LaneIdx& L) {
    ItemPlan P = lane_plan(L, ditems);
    P.ent = L.ent_bytes ? dent : nullptr;
    return P;
  };
  if (!X.decimal) {
    const LaneIdx& L = X.lanes[0];
    uint32_t w = native_width(X.wire);
    uint64_t* scr = nullptr;
    if (L.any_dict) {
      CK(c->ensure(S_DSCR, L.n_total * 8 + 64));
      scr = c->p<uint64_t>(S_DSCR);
    }
    // Fused: decoded values go straight to the typed column (narrowed, and
    // scattered through the bitmap when there is one).
    bool fused = ((uintptr_t)d_out % w) == 0;
    if (fused) {
      DecodeOut O{d_out, X.wire, X.has_validity ? reinterpret_cast<const uint32_t*>(dbm) : nullptr, drank, dsel, X.n,
                  L.n_total};
      O.plog2 = L.plog2;
      {
        TimedRegion tr(T_DECODE, st);
        launch_decode_items(d_src, dfr + L.frame_base, (int)L.nf, X.wire, O, plan_of(L), dpre,
                            scr, daux, d_err, st);
      }
      if (L.n_total == 0 && X.n) CK(cudaMemsetAsync(d_out, 0, X.n * w, st));  // all null
    } else {
      CK(c->ensure(S_LANE, L.n_total * 8 + 64));
      uint64_t* lane_out = c->p<uint64_t>(S_LANE);
      DecodeOut O{lane_out, WT_U64, nullptr, nullptr, nullptr, L.n_total, L.n_total};
      O.plog2 = L.plog2;
      {
        TimedRegion tr(T_DECODE, st);
        launch_decode_items(d_src, dfr + L.frame_base, (int)L.nf, X.wire, O, plan_of(L), dpre,
                            scr, daux, d_err, st);
      }
      if (X.n) {
        TimedRegion tr(T_FINALIZE, st);
        launch_finalize(lane_out, bm, drank, X.n, X.wire, d_out, st);
      }
    }
  } else {
    CK(c->ensure(S_LIMBS, (uint64_t)X.nl * X.n_valid * 8 + 64));
    uint64_t* limbs = c->p<uint64_t>(S_LIMBS);
    uint64_t scr_need = 0;
    for (auto& L : X.lanes)
      if (L.any_dict) scr_need = L.n_total;
    uint64_t* scr = nullptr;
    if (scr_need) {
      CK(c->ensure(S_DSCR, scr_need * 8 + 64));
      scr = c->p<uint64_t>(S_DSCR);
    }
    for (int k = 0; k < X.nl; k++) {
      const LaneIdx& L = X.lanes[k];
      DecodeOut O{limbs + (uint64_t)k * X.n_valid, WT_U64, nullptr, nullptr, nullptr, X.n_valid, X.n_valid};
      O.plog2 = L.plog2;
      TimedRegion tr(T_DECODE, st);
      launch_decode_items(d_src, dfr + L.frame_base, (int)L.nf, WT_U64, O, plan_of(L), dpre, scr,
                          daux, d_err, st);
    }
    if (X.n) {
      TimedRegion tr(T_FINALIZE, st);
      launch_decimal_combine(limbs, X.n_valid, X.nl, dvmin, bm, drank, X.n, (uint8_t*)d_out, st);
    }
  }
  if (d_valid_out && X.has_validity && X.n)
    CK(cudaMemcpyAsync(d_valid_out, dbm, (X.n + 7) / 8, cudaMemcpyDeviceToDevice, st));
  unsigned long long herr = 0;
  CK(read_small(c, st, &herr, d_err, 8));
  resolve_timing();
  if (herr != ~0ull) return kind_to_code((int)(herr & 0xFF));
  return QUOIN_OK;
}

// Decode a host stream into host buffers (values_out: n native values;
// validity_out: ceil(n/8) bytes or null).  *X_out receives the parsed index.
// The context's reusable host index (its buffers keep their capacity).
QuoinDecodeIndex& host_index(QuoinCtx* c) {
  if (!c->hidx) c->hidx = new QuoinDecodeIndex();
  return *c->hidx;
}

// First half of a host-buffer decode: the stream's copy to the device (S_SRC)
// starts, and the host parses the stream meanwhile.  After a parse error the
// copy is waited for (the caller owns src) and the error returned.
int begin_decode(QuoinCtx* c, const uint8_t* src, uint64_t len, QuoinDecodeIndex& X) {
  cudaStream_t st = c->stream;
  CK(c->ensure(S_SRC, len + 64));
  if (len) CK(cudaMemcpyAsync(c->p<uint8_t>(S_SRC), src, len, cudaMemcpyHostToDevice, st));
  int k = parse_stream(src, len, X);
  if (k) {
    cudaStreamSynchronize(st);
    return kind_to_code(k);
  }
  return QUOIN_OK;
}

// Second half: uploads the index, decodes, copies the values (and the
// validity bitmap) out.  Every return waits for the stream's work.
int finish_decode(QuoinCtx* c, QuoinDecodeIndex* X, void* values_out, uint8_t* validity_out) {
  cudaStream_t st = c->stream;
  uint64_t nf = total_frames(*X);
  CK(c->ensure(S_DFRAMES, (nf + 1) * sizeof(FrameDesc)));
  CK(c->ensure(S_DBM, X->bitmap.size() + 16));
  CK(c->ensure(S_DRANK, ((X->n + 31) / 32 + 1) * 8));
  CK(c->ensure(S_MISC, 64 * 8));
  uint64_t* dvmin = c->p<uint64_t>(S_MISC) + 32;
  CK(c->ensure(S_DSEL, sel_bytes(*X)));
  CK(c->ensure(S_DITEMS, X->items_bytes));
  int rc = upload_index(c, st, *X, c->p<FrameDesc>(S_DFRAMES), c->p<uint8_t>(S_DBM), c->p<uint64_t>(S_DRANK),
                        c->p<uint64_t>(S_DSEL), dvmin, c->p<uint64_t>(S_DITEMS));
  if (rc) {
    cudaStreamSynchronize(st);
    return rc;
  }
  uint64_t out_bytes = X->n * native_width(X->wire);
  CK(c->ensure(S_OUTVALS, out_bytes + 64));
  rc = decode_indexed(c, st, *X, c->p<FrameDesc>(S_DFRAMES), c->p<uint8_t>(S_DBM), c->p<uint64_t>(S_DRANK),
                      c->p<uint64_t>(S_DSEL), dvmin, c->p<uint64_t>(S_DITEMS), c->p<uint8_t>(S_SRC),
                      c->p<void>(S_OUTVALS), nullptr);
  if (rc) return rc;
  if (out_bytes) CK(cudaMemcpyAsync(values_out, c->p<void>(S_OUTVALS), out_bytes, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (validity_out && X->has_validity && X->n) memcpy(validity_out, X->bitmap.data(), X->bitmap.size());
  return QUOIN_OK;
}

int decompress_host(QuoinCtx* c, const uint8_t* src, uint64_t len, void* values_out, uint8_t* validity_out,
                    QuoinDecodeIndex* X) {
  int rc = begin_decode(c, src, len, *X);
  if (rc) return rc;
  return finish_decode(c, X, values_out, validity_out);
}

// ---------------------------------------------------------------------------
// Decode of a device-resident stream, parsed on the device (qb_dparse.cu).
// ---------------------------------------------------------------------------
struct DpMisc {  // the reader's small results, read back in one copy
  DpLaneOut lanes[4];
  uint64_t nvalid;
  uint64_t ncand[4];
  uint64_t nruns;  // runs of an RLE validity blob
  uint64_t ctl[4][2];  // per lane: chain resolved, chain frames
};
constexpr uint64_t kDpHeadOff = 0, kDpMiscOff = 512;
static_assert(sizeof(DpHead) <= kDpMiscOff && sizeof(DpMisc) <= 512, "reader results fit their slot");

// Decodes of device streams read by the device reader, and those the host
// reader took (with the reason of the last: 1 header, 2 a lane's chain, 3 a
// lane still over capacity after the exact count).
std::atomic<uint64_t> g_reads_device{0}, g_reads_host{0}, g_reads_host_reason{0};
std::atomic<uint64_t> g_last_ncand{0}, g_last_attempts{0};  // the last device read: candidates, table rounds
std::atomic<uint64_t> g_batch_columns{0};  // columns decoded by the batched path

// Candidate capacity of a lane whose frames span `bytes`: encoder streams
// hold far fewer frames (one per 32,768 values for adaptive blocks); a lane
// with more candidates is read again with the exact count.
uint64_t dp_cap(uint64_t bytes) { return bytes / 512 + 8192; }

// The host reader's route for the streams the device reader leaves to it: a
// host copy, parsed and uploaded as for a host-buffer decode.
int decode_device_via_host(QuoinCtx* c, cudaStream_t st, const uint8_t* d_src, uint64_t len, void* d_out,
                           uint64_t out_cap_bytes, uint8_t* d_valid_out, int32_t* wire_out, uint64_t* n_out,
                           int reason) {
  g_reads_host.fetch_add(1);
  g_reads_host_reason.store((uint64_t)reason);
  std::vector<uint8_t> h(len);
  if (len) CK(cudaMemcpyAsync(h.data(), d_src, len, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  QuoinDecodeIndex& X = host_index(c);
  int k = parse_stream(h.data(), len, X);
  if (k) return kind_to_code(k);
  *wire_out = X.wire;
  *n_out = X.n;
  if (X.n * (uint64_t)native_width(X.wire) > out_cap_bytes) return QUOIN_ERR_BUFFER_TOO_SMALL;
  uint64_t nf = total_frames(X);
  CK(c->ensure(S_DFRAMES, (nf + 1) * sizeof(FrameDesc)));
  CK(c->ensure(S_DBM, X.bitmap.size() + 16));
  CK(c->ensure(S_DRANK, ((X.n + 31) / 32 + 1) * 8));
  CK(c->ensure(S_MISC, 64 * 8));
  uint64_t* dvmin = c->p<uint64_t>(S_MISC) + 32;
  CK(c->ensure(S_DSEL, sel_bytes(X)));
  CK(c->ensure(S_DITEMS, X.items_bytes));
  int rc = upload_index(c, st, X, c->p<FrameDesc>(S_DFRAMES), c->p<uint8_t>(S_DBM), c->p<uint64_t>(S_DRANK),
                        c->p<uint64_t>(S_DSEL), dvmin, c->p<uint64_t>(S_DITEMS));
  if (rc) return rc;
  return decode_indexed(c, st, X, c->p<FrameDesc>(S_DFRAMES), c->p<uint8_t>(S_DBM), c->p<uint64_t>(S_DRANK),
                        c->p<uint64_t>(S_DSEL), dvmin, c->p<uint64_t>(S_DITEMS), d_src, d_out, d_valid_out);
}

// Reference decoder.rs:43-118 (+ decimal.rs:100-168, lib.rs:462-508) for a
// stream in device memory: header, validity and frame table are read by the
// device reader, then the block decoder runs as for an indexed decode.  Three
// host synchronisations: the header (output sizes), the frame tables (launch
// sizes), the final status.
int decode_device(QuoinCtx* c, cudaStream_t st, const uint8_t* d_src, uint64_t len, void* d_out,
                  uint64_t out_cap_bytes, uint8_t* d_valid_out, int32_t* wire_out, uint64_t* n_out) {
  CK(c->ensure(S_DPMISC, 1024));
  uint8_t* misc = c->p<uint8_t>(S_DPMISC);
  DpHead* dH = reinterpret_cast<DpHead*>(misc + kDpHeadOff);
  DpMisc* dM = reinterpret_cast<DpMisc*>(misc + kDpMiscOff);
  CK(cudaMemsetAsync(dM, 0, sizeof(DpMisc), st));  // the valid count stays 0 without a bitmap
  {
    TimedRegion tr(T_READ, st);
    launch_dp_head(d_src, len, dH, st);
  }
  DpHead H;
  CK(read_small(c, st, &H, dH, sizeof(H)));
  if (H.kind)
    return decode_device_via_host(c, st, d_src, len, d_out, out_cap_bytes, d_valid_out, wire_out, n_out, 1);
  *wire_out = (int32_t)H.wire;
  *n_out = H.n;
  uint32_t w = native_width((int)H.wire);
  if (H.n * (uint64_t)w > out_cap_bytes) return QUOIN_ERR_BUFFER_TOO_SMALL;
  const uint64_t n = H.n;
  const uint64_t nw = (n + 31) / 32;
  // validity: bitmap, word ranks, valid count, select table
  if (H.has_validity && n) {
    TimedRegion tr(T_READ, st);
    CK(c->ensure(S_DBM, (nw + 2) * 4 + 16));
    CK(c->ensure(S_DRANK, (nw + 1) * 8));
    CK(c->ensure(S_TILE, (scan_tile_count(nw + 4096) + 16) * 8));
    if (H.vtag == 0) {
      launch_dp_bitmap(d_src, dH, n, c->p<uint8_t>(S_DBM), c->p<uint64_t>(S_DRANK), st);
    } else {  // run lengths: at most one run per blob byte
      CK(c->ensure(S_DPRUNS, (H.vblob_len + 2) * 8));
      launch_dp_bitmap_rle(d_src, dH, n, c->p<uint64_t>(S_DPRUNS), &dM->nruns, c->p<uint8_t>(S_DBM),
                           c->p<uint64_t>(S_DRANK), st);
    }
    launch_scan_sum(c->p<uint64_t>(S_DRANK), c->p<uint64_t>(S_DRANK), nw, c->p<uint64_t>(S_TILE), &dM->nvalid, st);
    if (!H.decimal) {
      // the valid count is only known on the device: n bounds it (every
      // table entry the kernel writes is below the count anyway)
      CK(c->ensure(S_DSEL, (n / 512 + 2) * 8));
      launch_select_table(c->p<uint8_t>(S_DBM), n, c->p<uint64_t>(S_DRANK), n, c->p<uint64_t>(S_DSEL), st);
    }
  }
  // per-lane regions of the candidate, frame and item tables
  const int nl = (int)H.nl;
  uint64_t caps[4], cnt_off[4], slot_off[4], cand_off[4], node_off[4], j_off[4], fr_off[4], main_b[4], pre_b[4],
      fp_b[4], list_b[4], moff_b[4];
  uint64_t caps_min[4] = {0, 0, 0, 0};
  for (int attempt = 0; attempt < 2; attempt++) {
    uint64_t cand_bytes = 0, j_bytes = 0, frames_n = 0, items_u64 = 0, max_chunks = 0;
    for (int k = 0; k < nl; k++) {
      const DpLane& L = H.lanes[k];
      uint64_t fb = L.base + L.len - L.fstart;
      caps[k] = dp_cap(fb) > caps_min[k] ? dp_cap(fb) : caps_min[k];
      cnt_off[k] = cand_bytes;
      cand_bytes += (dp_chunks(fb) + 2) * 8;
      max_chunks = dp_chunks(fb) + 1 > max_chunks ? dp_chunks(fb) + 1 : max_chunks;
      slot_off[k] = cand_bytes;
      cand_bytes += (dp_slot_bytes(fb) + 255) & ~255ull;
      cand_off[k] = cand_bytes;
      cand_bytes += caps[k] * sizeof(DpCand);
      node_off[k] = cand_bytes;
      cand_bytes += (caps[k] * sizeof(DpNode) + 255) & ~255ull;
      j_off[k] = j_bytes;
      j_bytes += (caps[k] * 9 + 255) & ~255ull;
      fr_off[k] = frames_n;
      frames_n += caps[k];
      uint64_t nmax = L.logical_n / 512 + fb / 512 + 2 * caps[k] + 16;  // items of either kind
      main_b[k] = items_u64;
      items_u64 += nmax;
      pre_b[k] = items_u64;
      items_u64 += nmax;
      fp_b[k] = items_u64;
      items_u64 += caps[k];
      list_b[k] = items_u64;
      items_u64 += (caps[k] + 1) / 2 + 1;
      moff_b[k] = items_u64;
      items_u64 += caps[k] + 1;
    }
    CK(c->ensure(S_DPCAND, cand_bytes));
    CK(c->ensure(S_DPJ, j_bytes));
    CK(c->ensure(S_DFRAMES, (frames_n + 1) * sizeof(FrameDesc)));
    CK(c->ensure(S_DITEMS, items_u64 * 8 + 64));
    CK(c->ensure(S_TILE, (scan_tile_count(max_chunks + nw + 4096) + 16) * 8));
    uint8_t* cb = c->p<uint8_t>(S_DPCAND);
    uint64_t* ditems = c->p<uint64_t>(S_DITEMS);
    const uint64_t* d_nvalid = H.has_validity ? &dM->nvalid : nullptr;
    for (int k = 0; k < nl; k++) {
      TimedRegion tr(T_READ, st);
      const DpLane& L = H.lanes[k];
      uint64_t fb = L.base + L.len - L.fstart;
      DpCand* cand = reinterpret_cast<DpCand*>(cb + cand_off[k]);
      launch_dp_candidates(d_src, len, dH, k, fb, reinterpret_cast<uint64_t*>(cb + cnt_off[k]),
                           reinterpret_cast<DpCand*>(cb + slot_off[k]), c->p<uint64_t>(S_TILE), &dM->ncand[k], cand,
                           caps[k], st);
      uint8_t* jb = c->p<uint8_t>(S_DPJ) + j_off[k];
      DpTables T;
      T.frames = c->p<FrameDesc>(S_DFRAMES) + fr_off[k];
      T.frame_pre = reinterpret_cast<uint2*>(ditems + fp_b[k]);
      T.main_off = ditems + moff_b[k];
      T.list = reinterpret_cast<uint32_t*>(ditems + list_b[k]);
      T.main_items = reinterpret_cast<ItemRef*>(ditems + main_b[k]);
      T.pre_items = reinterpret_cast<ItemRef*>(ditems + pre_b[k]);
      launch_dp_chain(d_src, dH, k, d_nvalid, cand, &dM->ncand[k], caps[k],
                      reinterpret_cast<DpNode*>(cb + node_off[k]), reinterpret_cast<uint32_t*>(jb), jb + caps[k] * 8,
                      dM->ctl[k], T, &dM->lanes[k], st);
    }
    DpMisc M;
    CK(read_small(c, st, &M, dM, sizeof(M)));
    uint64_t ncand = 0;
    for (int k = 0; k < nl; k++) ncand += M.ncand[k];
    g_last_ncand.store(ncand);
    g_last_attempts.store((uint64_t)attempt + 1);
    bool grow = false, host = false;
    for (int k = 0; k < nl; k++) {
      if (!M.lanes[k].status) continue;
      if (M.lanes[k].ncand > caps[k] && attempt == 0) {
        caps_min[k] = M.lanes[k].ncand + 1024;
        grow = true;
      } else {
        host = true;
      }
    }
    if (host)
      return decode_device_via_host(c, st, d_src, len, d_out, out_cap_bytes, d_valid_out, wire_out, n_out,
                                    attempt ? 3 : 2);
    if (grow) continue;
    // the index the block decoder runs from
    QuoinDecodeIndex X;
    X.wire = (int)H.wire;
    X.n = n;
    X.has_validity = H.has_validity;
    X.decimal = H.decimal;
    X.scale = (int8_t)H.scale;
    X.precision = (uint8_t)H.precision;
    X.nl = H.decimal ? nl : 0;
    X.n_valid = H.has_validity ? M.nvalid : n;
    X.lanes.resize(nl);
    X.max_pre = 0;
    for (int k = 0; k < nl; k++) {
      LaneIdx& L = X.lanes[k];
      const DpLaneOut& O = M.lanes[k];
      L.dtype = (int)H.lanes[k].dtype;
      L.plog2 = H.lanes[k].plog2;
      L.logical_n = H.lanes[k].logical_n;
      L.has_validity = H.lanes[k].has_validity;
      L.n_total = (!H.decimal && L.has_validity) ? M.nvalid : L.logical_n;
      L.any_dict = O.any_dict;
      L.need_scan = O.need_scan;
      L.ent_bytes = O.ent_bytes;
      L.frame_base = fr_off[k];
      L.main_base = main_b[k];
      L.pre_base = pre_b[k];
      L.fp_base = fp_b[k];
      L.list_base = list_b[k];
      L.nf = O.nframes;
      L.nmain = O.nmain;
      L.npre = O.npre;
      L.nlist = O.nlist;
      X.max_pre = L.npre > X.max_pre ? L.npre : X.max_pre;
    }
    g_reads_device.fetch_add(1);
    const uint64_t* dvmin = reinterpret_cast<const uint64_t*>(misc + kDpHeadOff + offsetof(DpHead, vmin));
    return decode_indexed(c, st, X, c->p<FrameDesc>(S_DFRAMES), c->p<uint8_t>(S_DBM), c->p<uint64_t>(S_DRANK),
                          c->p<uint64_t>(S_DSEL), dvmin, ditems, d_src, d_out, d_valid_out);
  }
  return decode_device_via_host(c, st, d_src, len, d_out, out_cap_bytes, d_valid_out, wire_out, n_out, 3);
}

// ---------------------------------------------------------------------------
// Batched decode of device streams (qb_dparse.cu batch reader + one launch of
// each block-decoder kernel over all columns).
// ---------------------------------------------------------------------------
struct BumpAlloc {  // carves 256-byte aligned pieces out of one buffer
  uint64_t off = 0;
  uint64_t take(uint64_t bytes) {
    uint64_t o = off;
    off += (bytes + 255) & ~255ull;
    return o;
  }
};

int decode_queue(QuoinCtx* c, cudaStream_t st, QuoinB200DeviceDecodeJob* jobs, size_t nj) {
  for (size_t i = 0; i < nj; i++) {
    jobs[i].wire = 0;
    jobs[i].n = 0;
    jobs[i].status = QUOIN_ERR_NULL;
  }
  if (nj == 0) return QUOIN_OK;
  std::vector<char> single(nj, 1);  // decoded one by one after the batch
  // headers of every stream
  {
    BumpAlloc ba;
    uint64_t o_src = ba.take(nj * 8), o_len = ba.take(nj * 8), o_h = ba.take(nj * sizeof(DpHead));
    CK(c->ensure(S_BHOST, ba.off));
    std::vector<uint64_t> hv(2 * nj);
    for (size_t i = 0; i < nj; i++) {
      hv[i] = (uint64_t)(uintptr_t)jobs[i].d_src;
      hv[nj + i] = jobs[i].d_src ? jobs[i].src_len : 0;
    }
    uint8_t* base = c->p<uint8_t>(S_BHOST);
    CK(cudaMemcpyAsync(base + o_src, hv.data(), nj * 8, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(base + o_len, hv.data() + nj, nj * 8, cudaMemcpyHostToDevice, st));
    launch_dp_batch_heads(reinterpret_cast<const uint8_t* const*>(base + o_src),
                          reinterpret_cast<const uint64_t*>(base + o_len), (int)nj,
                          reinterpret_cast<DpHead*>(base + o_h), st);
    std::vector<DpHead> H(nj);
    CK(cudaMemcpyAsync(H.data(), base + o_h, nj * sizeof(DpHead), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    // the columns the batch takes, in job order
    std::vector<size_t> take;
    for (size_t i = 0; i < nj; i++) {
      const QuoinB200DeviceDecodeJob& J = jobs[i];
      const DpHead& h = H[i];
      if (!J.d_src || !J.d_values_out || h.kind || h.n == 0) continue;
      uint32_t w = native_width((int)h.wire);
      if (h.n * (uint64_t)w > J.values_cap_bytes || ((uintptr_t)J.d_values_out % w) != 0) continue;
      take.push_back(i);
    }
    if (!take.empty()) {
      // one batch lane per plain column, one per limb of a decimal container
      // (its first limb lane reads the container's bitmap)
      std::vector<int> lane_job, lane_limb, col_lane0(take.size());
      for (size_t t = 0; t < take.size(); t++) {
        const DpHead& h = H[take[t]];
        col_lane0[t] = (int)lane_job.size();
        int nlimb = h.decimal ? (int)h.nl : 1;
        for (int k = 0; k < nlimb; k++) {
          lane_job.push_back((int)t);
          lane_limb.push_back(k);
        }
      }
      const int nl = (int)lane_job.size();
      std::vector<DpBLane> lanes(nl);
      std::vector<uint64_t> word0(nl + 1), chunk0(nl + 1), limb_off(nl, 0);
      uint64_t words = 0, chunks = 0, sels = 0, cap = 0, item_cap = 0, scr = 0, rle_len = 0, limbs = 0;
      std::vector<uint32_t> rle_cols;
      for (int k = 0; k < nl; k++) {
        const QuoinB200DeviceDecodeJob& J = jobs[take[lane_job[k]]];
        const DpHead& h = H[take[lane_job[k]]];
        const int limb = lane_limb[k];
        DpBLane& B = lanes[k];
        B = DpBLane{};
        B.s = J.d_src;
        B.buf_len = J.src_len;
        B.L = h.lanes[limb];
        B.decimal = h.decimal;
        B.vlane = col_lane0[lane_job[k]];
        B.has_bm = h.has_validity && limb == 0;
        B.bm_n = h.n;
        B.vblob_off = h.vblob_off;
        B.vblob_len = h.vblob_len;
        B.vtag = B.has_bm ? h.vtag : 0;
        B.rle_off = rle_len;
        if (B.has_bm && h.vtag == 1) {
          rle_cols.push_back((uint32_t)k);
          rle_len += h.vblob_len + 2;
        }
        B.nw = B.has_bm ? (h.n + 31) / 32 : 0;
        B.word0 = word0[k] = words;
        words += B.nw + 1;
        B.sel0 = sels;
        sels += h.n / 512 + 2;
        uint64_t fb = B.L.base + B.L.len - B.L.fstart;
        B.chunk0 = chunk0[k] = chunks;
        chunks += dp_chunks(fb);
        uint64_t cc = dp_cap(fb);
        cap += cc;
        item_cap += B.L.logical_n / 512 + fb / 512 + 2 * cc + 16;
        scr += h.n;
        B.valid_out = B.has_bm ? J.d_validity_out : nullptr;
        if (h.decimal) {  // the limb's values, n at most (the stride of k_decimal_combine)
          limb_off[k] = limbs;
          limbs += h.n;
        }
      }
      word0[nl] = words;
      chunk0[nl] = chunks;
      BumpAlloc a;
      uint64_t o_lanes = a.take(nl * sizeof(DpBLane)), o_w0 = a.take((nl + 1) * 8), o_c0 = a.take((nl + 1) * 8),
               o_out = a.take(nl * sizeof(DpBLaneOut)), o_tot = a.take(sizeof(DpBTotals)),
               o_bm = a.take(words * 4), o_rk = a.take((words + 1) * 8), o_rb = a.take(nl * 8),
               o_sel = a.take(sels * 8), o_cnt = a.take((chunks + 1) * 8), o_slots = a.take(dp_batch_slot_bytes(chunks)),
               o_cand = a.take(cap * sizeof(DpCand)), o_cl = a.take(cap * 4), o_nodes = a.take(cap * sizeof(DpNode)),
               o_J = a.take(cap * 8), o_mk = a.take(cap), o_ft = a.take(cap * 16), o_fl = a.take(cap * 4),
               o_fr = a.take((cap + 1) * sizeof(FrameDesc)), o_fc = a.take((cap + 1) * 4),
               o_fp = a.take((cap + 1) * 8), o_mi = a.take(item_cap * 8), o_pi = a.take(item_cap * 8),
               o_li = a.take((cap + 1) * 4), o_cols = a.take(nl * sizeof(BatchCol)), o_err = a.take(64),
               o_rle = a.take((rle_len + 1) * 8), o_rln = a.take(nl * 8), o_rlc = a.take((rle_cols.size() + 1) * 4),
               o_vmin = a.take(take.size() * 32), o_limbs = a.take((limbs + 1) * 8);
      CK(c->ensure(S_BATCH, a.off));
      uint8_t* bb = c->p<uint8_t>(S_BATCH);
      CK(cudaMemcpyAsync(bb + o_lanes, lanes.data(), nl * sizeof(DpBLane), cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(bb + o_w0, word0.data(), (nl + 1) * 8, cudaMemcpyHostToDevice, st));
      CK(cudaMemcpyAsync(bb + o_c0, chunk0.data(), (nl + 1) * 8, cudaMemcpyHostToDevice, st));
      if (!rle_cols.empty())
        CK(cudaMemcpyAsync(bb + o_rlc, rle_cols.data(), rle_cols.size() * 4, cudaMemcpyHostToDevice, st));
      DpBatch B;
      B.lanes = reinterpret_cast<DpBLane*>(bb + o_lanes);
      B.word0 = reinterpret_cast<const uint64_t*>(bb + o_w0);
      B.chunk0 = reinterpret_cast<const uint64_t*>(bb + o_c0);
      B.out = reinterpret_cast<DpBLaneOut*>(bb + o_out);
      B.tot = reinterpret_cast<DpBTotals*>(bb + o_tot);
      B.nlanes = nl;
      B.bm32 = reinterpret_cast<uint32_t*>(bb + o_bm);
      B.ranks = reinterpret_cast<uint64_t*>(bb + o_rk);
      B.rbase = reinterpret_cast<uint64_t*>(bb + o_rb);
      B.sel = reinterpret_cast<uint64_t*>(bb + o_sel);
      B.cnt = reinterpret_cast<uint64_t*>(bb + o_cnt);
      B.slots = reinterpret_cast<DpCand*>(bb + o_slots);
      B.cand = reinterpret_cast<DpCand*>(bb + o_cand);
      B.cand_lane = reinterpret_cast<uint32_t*>(bb + o_cl);
      B.nodes = reinterpret_cast<DpNode*>(bb + o_nodes);
      B.gJ = reinterpret_cast<uint32_t*>(bb + o_J);
      B.gmarks = bb + o_mk;
      B.ftmp = reinterpret_cast<uint4*>(bb + o_ft);
      B.flist = reinterpret_cast<uint32_t*>(bb + o_fl);
      B.cap = cap;
      B.words = words;
      B.chunks = chunks;
      B.frames = reinterpret_cast<FrameDesc*>(bb + o_fr);
      B.frame_col = reinterpret_cast<uint32_t*>(bb + o_fc);
      B.frame_pre = reinterpret_cast<uint2*>(bb + o_fp);
      B.main_items = reinterpret_cast<ItemRef*>(bb + o_mi);
      B.pre_items = reinterpret_cast<ItemRef*>(bb + o_pi);
      B.list = reinterpret_cast<uint32_t*>(bb + o_li);
      B.item_cap = item_cap;
      B.rle_ends = reinterpret_cast<uint64_t*>(bb + o_rle);
      B.rle_nruns = reinterpret_cast<uint64_t*>(bb + o_rln);
      B.rle_cols = reinterpret_cast<const uint32_t*>(bb + o_rlc);
      B.nrle = (int)rle_cols.size();
      CK(c->ensure(S_TILE, (scan_tile_count((words > chunks ? words : chunks) + 1) + 16) * 8));
      {
        TimedRegion tr(T_READ, st);
        CK(cudaMemsetAsync(B.out, 0, nl * sizeof(DpBLaneOut), st));
        launch_dp_batch_read(B, c->p<uint64_t>(S_TILE), st);
      }
      std::vector<DpBLaneOut> out(nl);
      DpBTotals tot;
      uint64_t ktot = 0;
      CK(cudaMemcpyAsync(out.data(), B.out, nl * sizeof(DpBLaneOut), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(&tot, B.tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(&ktot, B.cnt + chunks, 8, cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      if (ktot <= cap && tot.nmain <= item_cap && tot.npre <= item_cap) {
        bool dict = false;
        for (int k = 0; k < nl; k++) dict = dict || (out[k].status == 0 && out[k].any_dict);
        if (dict) CK(c->ensure(S_BSCR, scr * 8 + 64));
        std::vector<BatchCol> cols(nl);
        uint64_t so = 0;
        uint64_t* limb_base = reinterpret_cast<uint64_t*>(bb + o_limbs);
        for (int k = 0; k < nl; k++) {
          const DpHead& h = H[take[lane_job[k]]];
          BatchCol& C = cols[k];
          C = BatchCol{};
          if (h.decimal) {  // limbs, dense, into the limb area
            uint64_t nv = out[lanes[k].vlane].nvalid;
            C.O.out = limb_base + limb_off[k];
            C.O.dtype = WT_U64;
            C.O.n = nv;
            C.O.nvalid = nv;
            C.dtype = WT_U64;
          } else {
            C.O.out = jobs[take[lane_job[k]]].d_values_out;
            C.O.dtype = (int)h.wire;
            C.O.bm32 = h.has_validity ? B.bm32 + lanes[k].word0 : nullptr;
            C.O.wrank = B.ranks + lanes[k].word0;
            C.O.sel = B.sel + lanes[k].sel0;
            C.O.n = h.n;
            C.O.nvalid = out[k].nvalid;
            C.dtype = (int)h.wire;
          }
          C.O.plog2 = lanes[k].L.plog2;
          C.scratch = dict ? c->p<uint64_t>(S_BSCR) + so : nullptr;
          so += h.n;
        }
        // a decimal column is batched when all its limb lanes are
        std::vector<char> col_ok(take.size(), 1);
        for (int k = 0; k < nl; k++)
          if (out[k].status != 0) col_ok[lane_job[k]] = 0;
        std::vector<uint64_t> vmins(take.size() * 4, 0);
        for (size_t t = 0; t < take.size(); t++)
          for (int q = 0; q < 4; q++) vmins[4 * t + q] = H[take[t]].vmin[q];
        CK(cudaMemcpyAsync(bb + o_vmin, vmins.data(), vmins.size() * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(bb + o_cols, cols.data(), nl * sizeof(BatchCol), cudaMemcpyHostToDevice, st));
        unsigned long long* d_err = reinterpret_cast<unsigned long long*>(bb + o_err);
        CK(cudaMemsetAsync(d_err, 0xFF, 8, st));
        CK(c->ensure(S_DAUX, decode_aux_bytes((int)(tot.nframes + 1))));
        CK(c->ensure(S_PRE, (tot.npre + 1) * prepass_rec_bytes()));
        ItemPlan P;
        P.pre_items = B.pre_items;
        P.npre = (uint32_t)tot.npre;
        P.main_items = B.main_items;
        P.nmain = (uint32_t)tot.nmain;
        P.frame_pre = B.frame_pre;
        P.list = B.list;
        P.nlist = (uint32_t)tot.nlist;
        P.need_scan = tot.need_scan != 0;
        P.ent = nullptr;
        BatchView bv{B.frame_col, reinterpret_cast<const BatchCol*>(bb + o_cols)};
        DecodeOut none{};
        {
          TimedRegion tr(T_DECODE, st);
          launch_decode_items(nullptr, B.frames, (int)tot.nframes, 0, none, P, c->p<void>(S_PRE), nullptr,
                              c->p<void>(S_DAUX), d_err, st, &bv);
        }
        {  // decimal containers: vmin + the limbs, through the container's bitmap
          TimedRegion tr(T_FINALIZE, st);
          for (size_t t = 0; t < take.size(); t++) {
            const DpHead& h = H[take[t]];
            if (!h.decimal || !col_ok[t]) continue;
            int k0 = col_lane0[t];
            const bool bm = h.has_validity != 0;
            launch_decimal_combine(limb_base + limb_off[k0], h.n, (int)h.nl,
                                   reinterpret_cast<const uint64_t*>(bb + o_vmin) + 4 * t,
                                   bm ? reinterpret_cast<const uint8_t*>(B.bm32 + lanes[k0].word0) : nullptr,
                                   bm ? B.ranks + lanes[k0].word0 : nullptr, h.n,
                                   static_cast<uint8_t*>(jobs[take[t]].d_values_out), st);
          }
        }
        unsigned long long herr = 0;
        CK(read_small(c, st, &herr, d_err, 8));
        resolve_timing();
        if (herr == ~0ull) {  // every batch column decoded: the others go one by one
          uint64_t ncols = 0;
          for (size_t t = 0; t < take.size(); t++) {
            if (!col_ok[t]) continue;
            QuoinB200DeviceDecodeJob& J = jobs[take[t]];
            J.wire = (int32_t)H[take[t]].wire;
            J.n = H[take[t]].n;
            J.status = QUOIN_OK;
            single[take[t]] = 0;
            ncols++;
          }
          g_batch_columns.fetch_add(ncols);
        }
      }
    }
  }
  // the columns left to the single-column path (and any failing batch)
  int first = QUOIN_OK;
  for (size_t i = 0; i < nj; i++) {
    QuoinB200DeviceDecodeJob& J = jobs[i];
    if (single[i]) {
      if (!J.d_src || !J.d_values_out) {
        J.status = QUOIN_ERR_NULL;
      } else {
        int32_t w = 0;
        uint64_t n = 0;
        J.status = decode_device(c, st, J.d_src, J.src_len, J.d_values_out, J.values_cap_bytes, J.d_validity_out,
                                 &w, &n);
        J.wire = w;
        J.n = n;
      }
    }
    if (J.status != QUOIN_OK && first == QUOIN_OK) first = J.status;
  }
  return first;
}

// Host-buffer compress of a typed column (wire dtype, native little-endian values).
int compress_host(QuoinCtx* c, int wire, uint64_t n, const void* values, const uint8_t* validity, int8_t scale,
                  uint8_t precision, const QuoinConfig* cfg, uint8_t* dst, size_t dst_cap, size_t* out_len) {
  if (wire < 0 || wire > 7) return QUOIN_ERR_BAD_ARG;
  cudaStream_t st = c->stream;
  uint64_t bytes = n * native_width(wire);
  CK(c->ensure(S_IN, bytes + 64));
  if (bytes) CK(cudaMemcpyAsync(c->p<uint8_t>(S_IN), values, bytes, cudaMemcpyHostToDevice, st));
  const uint8_t* d_bm = nullptr;
  if (validity && n) {
    CK(c->ensure(S_BM, (n + 7) / 8 + 64));
    CK(cudaMemcpyAsync(c->p<uint8_t>(S_BM), validity, (n + 7) / 8, cudaMemcpyHostToDevice, st));
    d_bm = c->p<uint8_t>(S_BM);
  }
  uint64_t bs = cfg && cfg->block_size > 0 ? (uint64_t)cfg->block_size : 0;
  uint64_t bound = column_bound(wire, n, validity != nullptr, bs > kMaxBlockValues ? kMaxBlockValues : bs);
  CK(c->ensure(S_OUT, bound + 64));
  size_t len = 0;
  int rc = compress_column_device(c, st, wire, n, c->p<void>(S_IN), d_bm, scale, precision, cfg, c->p<uint8_t>(S_OUT),
                                  bound, &len);
  if (rc) return rc;
  *out_len = len;
  if (len > dst_cap) return QUOIN_ERR_BUFFER_TOO_SMALL;
  if (len) CK(cudaMemcpyAsync(dst, c->p<uint8_t>(S_OUT), len, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return QUOIN_OK;
}

const QuoinConfig kFastCfg = {QUOIN_LEVEL_FAST, 0, 16};

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* quoin_version(void) { return "quoin-b200 0.1.0 (sm_100a)"; }

size_t quoin_compress_bound(size_t n_values) {
  size_t a = n_values > SIZE_MAX / 9 ? SIZE_MAX : n_values * 9;
  return a > SIZE_MAX - 1024 ? SIZE_MAX : a + 1024;
}

static int compress_f64(const QuoinCtx* cc, const double* src, size_t n, uint8_t* dst, size_t cap, size_t* out_len) {
  if (!src || !dst || !out_len) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(cc);
    if (!c) return QUOIN_ERR_PANIC;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    size_t len = 0;
    int rc = compress_host(c, WT_F64, n, src, nullptr, 0, 0, &kFastCfg, dst, cap, &len);
    if (rc == QUOIN_ERR_BUFFER_TOO_SMALL) {
      *out_len = len;
      return rc;
    }
    if (rc) return plain_code(rc);
    *out_len = len;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

static int decompress_f64(const QuoinCtx* cc, const uint8_t* src, size_t len, double* dst, size_t cap,
                          size_t* out_values) {
  if (!src || !dst || !out_values) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(cc);
    if (!c) return QUOIN_ERR_PANIC;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    QuoinDecodeIndex& X = host_index(c);
    if (begin_decode(c, src, len, X)) return QUOIN_ERR_CORRUPT;
    if (X.wire != WT_F64) {  // DTypeMismatch (lib.rs:522-527)
      cudaStreamSynchronize(c->stream);
      return QUOIN_ERR_CORRUPT;
    }
    std::vector<double> tmp;
    double* out = dst;
    if (X.n > cap) {
      tmp.resize(X.n ? X.n : 1);
      out = tmp.data();
    }
    int rc = finish_decode(c, &X, out, nullptr);
    if (rc) return plain_code(rc);
    *out_values = X.n;
    if (X.n > cap) return QUOIN_ERR_BUFFER_TOO_SMALL;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_compress(const double* src, size_t n, uint8_t* dst, size_t cap, size_t* out_len) {
  return compress_f64(nullptr, src, n, dst, cap, out_len);
}
int quoin_decompress(const uint8_t* src, size_t len, double* dst, size_t cap, size_t* out_values) {
  return decompress_f64(nullptr, src, len, dst, cap, out_values);
}
int quoin_compress_ctx(const QuoinCtx* ctx, const double* src, size_t n, uint8_t* dst, size_t cap, size_t* out_len) {
  return compress_f64(ctx, src, n, dst, cap, out_len);
}
int quoin_decompress_ctx(const QuoinCtx* ctx, const uint8_t* src, size_t len, double* dst, size_t cap,
                         size_t* out_values) {
  return decompress_f64(ctx, src, len, dst, cap, out_values);
}

ptrdiff_t quoin_decompressed_value_count(const uint8_t* src, size_t len) {
  if (!src) return QUOIN_ERR_NULL;
  // Header::read (format.rs:65-94)
  if (len < 16 || memcmp(src, "FCR1", 4) != 0 || src[4] != 2 || (src[5] & ~1u) || src[6] < 10 || src[6] > 16 ||
      src[7] > 7)
    return QUOIN_ERR_CORRUPT;
  uint64_t n = rd64(src + 8);
  if (n > (uint64_t)PTRDIFF_MAX) return QUOIN_ERR_CORRUPT;
  return (ptrdiff_t)n;
}

QuoinCtx* quoin_ctx_create(size_t threads) {
  (void)threads;
  try {
    return ctx_new();
  } catch (...) {
    return nullptr;
  }
}

void quoin_ctx_free(QuoinCtx* ctx) {
  if (!ctx) return;
  {
    DeviceScope ds(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (int s = 0; s < S_COUNT; s++)
      if (ctx->buf[s]) cudaFree(ctx->buf[s]);
    for (void* p : ctx->retired) cudaFree(p);
    ctx->retired.clear();
    cudaStreamDestroy(ctx->stream);
    if (ctx->hbox) cudaFreeHost(ctx->hbox);
  }
  delete ctx->hidx;
  delete ctx;
}

size_t quoin_dtype_width(int32_t dtype) {  // capi/src/typed.rs:50-61
  switch (dtype) {
    case QUOIN_DTYPE_BOOL: case QUOIN_DTYPE_I8: case QUOIN_DTYPE_U8: return 1;
    case QUOIN_DTYPE_I16: case QUOIN_DTYPE_U16: return 2;
    case QUOIN_DTYPE_I32: case QUOIN_DTYPE_U32: case QUOIN_DTYPE_F32: case QUOIN_DTYPE_DECIMAL32: return 4;
    case QUOIN_DTYPE_I64: case QUOIN_DTYPE_U64: case QUOIN_DTYPE_F64: case QUOIN_DTYPE_DECIMAL64: return 8;
    case QUOIN_DTYPE_DECIMAL128: return 16;
    case QUOIN_DTYPE_DECIMAL256: return 32;
    default: return 0;
  }
}

size_t quoin_typed_compress_bound(int32_t dtype, size_t n) {  // capi/src/typed.rs:65-69
  size_t w = quoin_dtype_width(dtype);
  if (w < 8) w = 8;
  size_t a = n > SIZE_MAX / (w + 1) ? SIZE_MAX : n * (w + 1);
  return a > SIZE_MAX - 1024 ? SIZE_MAX : a + 1024;
}

// capi/src/typed.rs:125-174: widen the Arrow dtype to a lane dtype.
static size_t typed_compress_impl(int32_t dtype, size_t n, const void* values, const uint8_t* validity, int8_t scale,
                                  uint8_t precision, bool decimal_call, uint8_t* dst, size_t cap) {
  if (!values || !dst) return 0;
  try {
    QuoinCtx* c = default_ctx();
    if (!c) return 0;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    const uint8_t* in = (const uint8_t*)values;
    std::vector<uint8_t> conv;
    int wire;
    auto widen = [&](size_t from, bool sgn, size_t to) {
      conv.resize(n * to);
      for (size_t i = 0; i < n; i++) {
        int64_t v = 0;
        uint64_t u = 0;
        memcpy(&u, in + i * from, from);
        if (sgn) {
          int sh = 64 - (int)from * 8;
          v = (int64_t)(u << sh) >> sh;
        } else {
          v = (int64_t)u;
        }
        for (size_t b = 0; b < to; b++) conv[i * to + b] = b < 8 ? (uint8_t)((uint64_t)v >> (8 * b)) : (uint8_t)(v < 0 ? 0xFF : 0);
      }
      in = conv.data();
    };
    if (!decimal_call) {
      switch (dtype) {
        case QUOIN_DTYPE_F64: wire = WT_F64; break;
        case QUOIN_DTYPE_F32: wire = WT_F32; break;
        case QUOIN_DTYPE_I64: wire = WT_I64; break;
        case QUOIN_DTYPE_U64: wire = WT_U64; break;
        case QUOIN_DTYPE_I32: wire = WT_I32; break;
        case QUOIN_DTYPE_U32: wire = WT_U32; break;
        case QUOIN_DTYPE_I16: widen(2, true, 4); wire = WT_I32; break;
        case QUOIN_DTYPE_I8: widen(1, true, 4); wire = WT_I32; break;
        case QUOIN_DTYPE_U16: widen(2, false, 4); wire = WT_U32; break;
        case QUOIN_DTYPE_U8: case QUOIN_DTYPE_BOOL: widen(1, false, 4); wire = WT_U32; break;
        default: return 0;
      }
    } else {
      switch (dtype) {
        case QUOIN_DTYPE_DECIMAL128: wire = WT_DEC128; break;
        case QUOIN_DTYPE_DECIMAL256: wire = WT_DEC256; break;
        case QUOIN_DTYPE_DECIMAL64: widen(8, true, 16); wire = WT_DEC128; break;
        case QUOIN_DTYPE_DECIMAL32: widen(4, true, 16); wire = WT_DEC128; break;
        default: return 0;
      }
    }
    size_t len = 0;
    int rc = compress_host(c, wire, n, in, validity, scale, precision, &kFastCfg, dst, cap, &len);
    if (rc) return 0;
    return len;
  } catch (...) {
    return 0;
  }
}

size_t quoin_typed_compress(int32_t dtype, size_t n, const void* values, const uint8_t* validity, uint8_t* dst,
                            size_t dst_cap) {
  return typed_compress_impl(dtype, n, values, validity, 0, 0, false, dst, dst_cap);
}

size_t quoin_typed_compress_decimal(int32_t dtype, size_t n, const void* values, const uint8_t* validity,
                                    int8_t scale, uint8_t precision, uint8_t* dst, size_t dst_cap) {
  return typed_compress_impl(dtype, n, values, validity, scale, precision, true, dst, dst_cap);
}

// capi/src/typed.rs:232-338
int quoin_typed_decompress(int32_t dtype, size_t n, const uint8_t* src, size_t src_len, void* values_out,
                           uint8_t* validity_out) {
  if (!src || !values_out) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = default_ctx();
    if (!c) return QUOIN_ERR_PANIC;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    QuoinDecodeIndex& X = host_index(c);
    if (begin_decode(c, src, src_len, X)) return QUOIN_ERR_CORRUPT;
    // (Arrow dtype, decoded column) pairs accepted by scatter_values (typed.rs:256-273)
    int narrow_to = 0;  // bytes when narrowing
    bool sgn = false;
    bool ok = false;
    switch (dtype) {
      case QUOIN_DTYPE_F64: ok = X.wire == WT_F64; break;
      case QUOIN_DTYPE_F32: ok = X.wire == WT_F32; break;
      case QUOIN_DTYPE_I64: ok = X.wire == WT_I64; break;
      case QUOIN_DTYPE_U64: ok = X.wire == WT_U64; break;
      case QUOIN_DTYPE_I32: ok = X.wire == WT_I32; break;
      case QUOIN_DTYPE_U32: ok = X.wire == WT_U32; break;
      case QUOIN_DTYPE_I16: ok = X.wire == WT_I32; narrow_to = 2; sgn = true; break;
      case QUOIN_DTYPE_I8: ok = X.wire == WT_I32; narrow_to = 1; sgn = true; break;
      case QUOIN_DTYPE_U16: ok = X.wire == WT_U32; narrow_to = 2; break;
      case QUOIN_DTYPE_U8: case QUOIN_DTYPE_BOOL: ok = X.wire == WT_U32; narrow_to = 1; break;
      case QUOIN_DTYPE_DECIMAL128: ok = X.wire == WT_DEC128; break;
      case QUOIN_DTYPE_DECIMAL256: ok = X.wire == WT_DEC256; break;
      case QUOIN_DTYPE_DECIMAL64: ok = X.wire == WT_DEC128; narrow_to = 8; sgn = true; break;
      case QUOIN_DTYPE_DECIMAL32: ok = X.wire == WT_DEC128; narrow_to = 4; sgn = true; break;
      default: ok = false;
    }
    (void)sgn;
    uint32_t w = native_width(X.wire);
    uint8_t* out = (uint8_t*)values_out;
    bool direct = ok && X.n == n && !narrow_to;  // decode straight into the caller's buffer
    std::vector<uint8_t> full(direct ? 0 : X.n * w + 8);
    int rc = finish_decode(c, &X, direct ? values_out : (void*)full.data(), nullptr);
    if (rc) return plain_code(rc);
    if (!ok || X.n != n) return QUOIN_ERR_CORRUPT;
    if (!direct && !narrow_to) {
      memcpy(out, full.data(), n * w);
    } else if (!direct) {
      for (size_t i = 0; i < n; i++) memcpy(out + i * narrow_to, full.data() + i * w, narrow_to);  // `as` truncation
    }
    if (validity_out) {  // typed.rs:280-300
      size_t nbytes = (n + 7) / 8;
      if (X.has_validity) {
        size_t take = X.bitmap.size() < nbytes ? X.bitmap.size() : nbytes;
        memcpy(validity_out, X.bitmap.data(), take);
        if (take < nbytes) memset(validity_out + take, 0, nbytes - take);
      } else if (nbytes) {
        memset(validity_out, 0xFF, nbytes);
        if (n % 8) validity_out[nbytes - 1] = (uint8_t)((1u << (n % 8)) - 1u);
      }
    }
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

// ---------------- B200 extensions ----------------

int quoin_b200_compress_column(QuoinCtx* ctx, int32_t wire, size_t n, const void* values, const uint8_t* validity,
                               int8_t scale, uint8_t precision, const QuoinConfig* cfg, uint8_t* dst, size_t dst_cap,
                               size_t* out_len) {
  if (!out_len || (!values && n) || !dst) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    static const uint8_t kZero[8] = {0};
    return compress_host(c, wire, n, values ? values : kZero, validity, scale, precision, cfg, dst, dst_cap, out_len);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_stream_info(const uint8_t* src, size_t len, int32_t* wire, uint64_t* n, int32_t* has_validity,
                           int8_t* scale, uint8_t* precision) {
  if (!src || !wire || !n || !has_validity || !scale || !precision) return QUOIN_ERR_NULL;
  if (len > 5 && (src[5] & 2)) {
    if (len < 19) return QUOIN_ERR_TRUNCATED;
    if (src[7] > 7) return QUOIN_ERR_UNSUPPORTED_DTYPE;
    *wire = src[7];
    *n = rd64(src + 8);
    *has_validity = src[5] & 1;
    *scale = (int8_t)src[16];
    *precision = src[17];
    return QUOIN_OK;
  }
  if (len < 16) return QUOIN_ERR_TRUNCATED;
  if (memcmp(src, "FCR1", 4) != 0) return QUOIN_ERR_BAD_MAGIC;
  if (src[4] != 2) return QUOIN_ERR_UNSUPPORTED_VERSION;
  if ((src[5] & ~1u) || src[6] < 10 || src[6] > 16) return QUOIN_ERR_CORRUPT_PAYLOAD;
  if (src[7] > 7) return QUOIN_ERR_UNSUPPORTED_DTYPE;
  *wire = src[7];
  *n = rd64(src + 8);
  *has_validity = src[5] & 1;
  *scale = 0;
  *precision = 0;
  return QUOIN_OK;
}

int quoin_b200_parse(const uint8_t* src, size_t len, int32_t* wire, uint64_t* n, int32_t* has_validity) {
  if (!src || !wire || !n || !has_validity) return QUOIN_ERR_NULL;
  try {
    QuoinDecodeIndex X;
    int k = parse_stream(src, len, X);
    if (k) return kind_to_code(k);
    *wire = X.wire;
    *n = X.n;
    *has_validity = X.has_validity;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_decompress_column(QuoinCtx* ctx, const uint8_t* src, size_t len, void* values_out,
                                 uint8_t* validity_out) {
  if (!src || !values_out) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    return decompress_host(c, src, len, values_out, validity_out, &host_index(c));
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_compress_column_device(QuoinCtx* ctx, int32_t wire, size_t n, const void* d_values,
                                      const uint8_t* d_validity, int8_t scale, uint8_t precision,
                                      const QuoinConfig* cfg, uint8_t* d_dst, size_t dst_cap, size_t* out_len,
                                      void* stream) {
  if (!out_len || (!d_values && n) || !d_dst) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return compress_column_device(c, st, wire, n, d_values, d_validity, scale, precision, cfg, d_dst, dst_cap,
                                  out_len);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_probe_windows_device(QuoinCtx* ctx, int32_t wire, size_t n, const void* d_values,
                                    const uint8_t* d_validity, uint8_t* grow_out, size_t grow_cap,
                                    uint64_t* n_windows, void* stream) {
  if (!n_windows || (!d_values && n) || (!grow_out && grow_cap)) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return probe_windows_device(c, st, wire, n, d_values, d_validity, grow_out, grow_cap, n_windows);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_stream_prefix_device(QuoinCtx* ctx, int32_t wire, size_t n, const uint8_t* d_validity,
                                    const QuoinConfig* cfg, uint8_t* d_dst, size_t dst_cap, size_t* out_len,
                                    void* stream) {
  if (!out_len || !d_dst) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return stream_prefix_device(c, st, wire, n, d_validity, cfg, d_dst, dst_cap, out_len);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_index_create(QuoinCtx* ctx, const uint8_t* src, size_t len, QuoinDecodeIndex** out) {
  if (!src || !out) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    QuoinDecodeIndex* X = new QuoinDecodeIndex();
    int k = parse_stream(src, len, *X);
    if (k) {
      delete X;
      return kind_to_code(k);
    }
    X->owned = true;
    X->device = c->device;
    uint64_t nf = total_frames(*X);
    bool ok = cudaMalloc(&X->d_frames, (nf + 1) * sizeof(FrameDesc)) == cudaSuccess &&
              cudaMalloc(&X->d_bm, X->bitmap.size() + 16) == cudaSuccess &&
              cudaMalloc(&X->d_rank, ((X->n + 31) / 32 + 1) * 8) == cudaSuccess &&
              cudaMalloc(&X->d_sel, sel_bytes(*X)) == cudaSuccess &&
              cudaMalloc(&X->d_items, X->items_bytes) == cudaSuccess &&
              cudaMalloc(&X->d_vmin, 64) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      quoin_b200_index_free(X);
      return QUOIN_ERR_CUDA;
    }
    int rc = upload_index(c, c->stream, *X, X->d_frames, X->d_bm, X->d_rank, X->d_sel, X->d_vmin, X->d_items);
    if (rc) {
      quoin_b200_index_free(X);
      return rc;
    }
    *out = X;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

void quoin_b200_index_free(QuoinDecodeIndex* X) {
  if (!X) return;
  if (X->owned) {
    DeviceScope ds(X->device);
    if (X->d_frames) cudaFree(X->d_frames);
    if (X->d_bm) cudaFree(X->d_bm);
    if (X->d_rank) cudaFree(X->d_rank);
    if (X->d_sel) cudaFree(X->d_sel);
    if (X->d_items) cudaFree(X->d_items);
    if (X->d_vmin) cudaFree(X->d_vmin);
  }
  delete X;
}

int quoin_b200_index_decimal(const QuoinDecodeIndex* X, int8_t* scale, uint8_t* precision, uint64_t* n_valid) {
  if (!X || !scale || !precision || !n_valid) return QUOIN_ERR_NULL;
  *scale = X->scale;
  *precision = X->precision;
  *n_valid = X->has_validity ? X->n_valid : X->n;
  return QUOIN_OK;
}

int quoin_b200_index_info(const QuoinDecodeIndex* X, int32_t* wire, uint64_t* n, int32_t* has_validity) {
  if (!X || !wire || !n || !has_validity) return QUOIN_ERR_NULL;
  *wire = X->wire;
  *n = X->n;
  *has_validity = X->has_validity;
  return QUOIN_OK;
}

int quoin_b200_decompress_indexed_device(QuoinCtx* ctx, const QuoinDecodeIndex* X, const uint8_t* d_src,
                                         void* d_values_out, uint8_t* d_validity_out, void* stream) {
  if (!X || !d_src || !d_values_out) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return decode_indexed(c, st, *X, X->d_frames, X->d_bm, X->d_rank, X->d_sel, X->d_vmin, X->d_items, d_src,
                          d_values_out, d_validity_out);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_decompress_queue_device(QuoinCtx* ctx, QuoinB200DeviceDecodeJob* jobs, size_t njobs, void* stream) {
  if (!jobs && njobs) return QUOIN_ERR_NULL;
  try {
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return decode_queue(c, st, jobs, njobs);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

int quoin_b200_decompress_column_device(QuoinCtx* ctx, const uint8_t* d_src, size_t src_len, void* d_values_out,
                                        size_t values_cap_bytes, uint8_t* d_validity_out, int32_t* wire_out,
                                        uint64_t* n_out, void* stream) {
  if (!d_src || !d_values_out || !wire_out || !n_out) return QUOIN_ERR_NULL;
  try {
    *wire_out = 0;
    *n_out = 0;
    QuoinCtx* c = pick(ctx);
    if (!c) return QUOIN_ERR_CUDA;
    std::lock_guard<std::mutex> l(c->mu);
    DeviceScope ds(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    return decode_device(c, st, d_src, src_len, d_values_out, values_cap_bytes, d_validity_out, wire_out, n_out);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

void quoin_b200_reader_stats(uint64_t out[6]) {
  if (!out) return;
  out[0] = g_reads_device.load();
  out[1] = g_reads_host.load();
  out[2] = g_reads_host_reason.load();
  out[3] = g_last_ncand.load();
  out[4] = g_last_attempts.load();
  out[5] = g_batch_columns.load();
}

void quoin_b200_mode_win_counts(uint64_t out[64]) {
  if (!out) return;
  memset(out, 0, 64 * 8);
  unsigned long long* d = device_win_counters();
  if (!d) return;
  if (cudaMemcpy(out, d, 64 * 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    memset(out, 0, 64 * 8);
  }
}

void quoin_b200_reset_mode_win_counts(void) {
  unsigned long long* d = device_win_counters();
  if (d && cudaMemset(d, 0, 64 * 8) != cudaSuccess) cudaGetLastError();
}

uint64_t quoin_b200_kernel_launches(void) { return launches_total(); }

void quoin_b200_timing_enable(int on) {
  std::lock_guard<std::mutex> l(g_timing.mu);
  for (int k = 0; k < T_COUNT; k++) {
    g_timing.ms[k] = 0;
    g_timing.calls[k] = 0;
  }
  g_timing.on.store(on != 0);
}

int quoin_b200_timing_read(double* ms_out, uint64_t* calls_out, int n) {
  if (!ms_out || !calls_out) return QUOIN_ERR_NULL;
  resolve_timing();
  std::lock_guard<std::mutex> l(g_timing.mu);
  for (int k = 0; k < n && k < T_COUNT; k++) {
    ms_out[k] = g_timing.ms[k];
    calls_out[k] = g_timing.calls[k];
  }
  return T_COUNT;
}

}  // extern "C"
