// Device-side stream reader: the header, the validity blob and the frame
// table of a device-resident stream (reference src/format.rs:65-94,
// src/decoder.rs:43-118, src/decimal.rs:100-168), so a column decodes from
// device memory without the host ever holding the stream.
//
// The frame table is a chain: frame k+1 starts 9 + plen_k bytes after frame
// k, and the walk stops once the frames hold the lane's value count.  One
// thread following it pays one memory latency per frame (thousands per
// column), so the chain is resolved in parallel instead:
//   1. every byte position of a lane whose 9 bytes could be a frame header
//      (mode id known, 1 <= n <= 131072, plen < 2^24 and within the lane) and
//      whose payload passes its mode's first decode checks is a candidate:
//      one pass over the lane, with a zero-byte test on 8-byte words that
//      rejects most positions in a few instructions (k_dp_cand_scan, a scan
//      of the per-chunk counts, k_dp_cand_compact, in position order);
//   2. each candidate's successor (the candidate at pos + 9 + plen) is found
//      by binary search (k_dp_succ, across the GPU); marks spread from the
//      lane's first frame along the successors by pointer doubling, so after
//      log2(K) rounds exactly the frames on the chain are marked (every jump
//      from a chain frame lands on a chain frame), and chain order is
//      position order (k_dp_marks, one CTA);
//   3. the marked frames' warp items (512 values, or 2048 XORZ payload bytes)
//      are counted as the host reader's build_items does (k_dp_items, across
//      the GPU), the frames cut where their values reach the lane's count and
//      laid out (k_dp_layout, one CTA), and the items listed (k_dp_expand).
// Validity blobs are read here too: RAW bitmaps copied into words, RLE
// varint runs expanded by a run table.  A stream the fast path cannot take
// (a header or validity error, a chain frame that is not a candidate, a count
// mismatch, more candidates than the tables hold) is flagged, and the host
// reader parses a host copy instead, so every error kind stays the
// reference's.  The batched reader (k_dpb_*) flags columns with
// entropy-coded frames as well; those decode one by one.
#include "qb_common.cuh"
#include "qb_kernels.h"
#include "qb_layout.h"
#include "qb_scan.cuh"

namespace qb {
namespace {

constexpr int kDpThreads = 256;
constexpr int kDpSteps = 4;
constexpr uint64_t kDpStep = (uint64_t)kDpThreads * 16;  // positions per CTA step
constexpr uint64_t kDpChunk = kDpStep * kDpSteps;        // positions per candidate CTA
constexpr int kChainThreads = 1024;
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint64_t kMaxLogicalD = 1ull << 36;  // the host reader's allocation limit (decoder.rs:105-106)

// A varint within p[pos .. lim) (at most 10 bytes), or false.
__device__ inline bool dp_varint(const uint8_t* s, uint64_t pos, uint64_t lim, uint64_t* v) {
  uint64_t r = 0;
  for (uint32_t k = 0; k < 10 && pos + k < lim; k++) {
    uint32_t b = s[pos + k];
    r |= (uint64_t)(b & 0x7F) << (7 * k);
    if (!(b & 0x80)) {
      *v = r;
      return true;
    }
  }
  return false;
}

// What every frame of `mode` that decodes satisfies (the codec decoders'
// first checks: raw.rs, const_block.rs, stride.rs, xorz.rs:18-32,
// for_bitpack.rs:108-120, delta_bitpack.rs:48-64, alp.rs:168-180,
// float_mult.rs:100-110, dict.rs:150-160, rle.rs:45-55, alp_rd.rs:208-215,
// and entropy/mod.rs:152-178 for the entropy-coded modes: a tag 0..3, then a
// varint length no larger than the decode bound).  A frame that fails it
// cannot decode, so leaving it out only sends damaged streams to the host
// reader.
__device__ __noinline__ bool dp_frame_plausible(const uint8_t* s, uint64_t pl0, uint32_t n, uint32_t plen, uint32_t mode,
                                   uint32_t lane_bytes_) {
  uint64_t lim = pl0 + plen, v = 0;
  switch (mode) {
    case 5: return (uint64_t)plen == (uint64_t)n * lane_bytes_;
    case 1: return plen == 8;
    case 2: return plen == 16;
    case 3: return plen >= n && (uint64_t)plen <= 10ull * n && s[lim - 1] < 0x80;
    case 50: case 9: return dp_varint(s, pl0, lim, &v) && v == n;
    case 51: return plen >= 9 && dp_varint(s, pl0 + 8, lim, &v) && v == n;
    case 17: return plen >= 2 && s[pl0] <= 1 && s[pl0 + 1] < 7;
    case 19: case 53: return dp_varint(s, pl0, lim, &v) && v <= n;
    case 52: return plen >= 2 && s[pl0] >= 1 && s[pl0] <= 63 && s[pl0 + 1] <= 8;
    case 11: case 4: case 7: case 20: case 45: case 25: case 29: {
      uint64_t mx = mode == 11 ? 8ull * n + 16 : (mode == 4 ? 16ull * n + 1024 : 10ull * n + 16);
      return plen >= 2 && s[pl0] <= 3 && dp_varint(s, pl0 + 1, lim, &v) && v <= mx;
    }
    default: return true;  // PCO: no reader here, its decode reports it
  }
}

// ---------------------------------------------------------------------------
// Header (one thread).  Any error, or a form the device reader leaves to the
// host (a limb lane with its own bitmap), sets kind = 1.
// ---------------------------------------------------------------------------
__device__ bool dp_lane_header(const uint8_t* s, uint64_t base, uint64_t len, DpLane& L) {
  const uint8_t* h = s + base;
  if (len < 16) return false;
  if (h[0] != 'F' || h[1] != 'C' || h[2] != 'R' || h[3] != '1') return false;
  if (h[4] != 2 || (h[5] & ~1u) || h[6] < 10 || h[6] > 16 || h[7] > 7) return false;
  L.base = base;
  L.len = len;
  L.dtype = h[7];
  L.plog2 = h[6];
  L.has_validity = h[5] & 1;
  L.logical_n = ld_u64(h + 8);
  L.fstart = base + 16;
  return L.logical_n <= kMaxLogicalD;
}

// The validity blob at s[pos .. pos + vlen) (validity.rs:73-119): tag 0 then
// ceil(n/8) bitmap bytes, or tag 1 then varint run lengths.
__device__ bool dp_validity(const uint8_t* s, uint64_t len, uint64_t* pos, uint64_t n, DpHead& H) {
  uint64_t vlen;
  if (rd_varint(s, len, pos, &vlen) != E_OK || vlen > len - *pos || vlen == 0) return false;
  uint32_t tag = s[*pos];
  uint64_t raw = (n + 7) / 8;
  if (tag > 1 || (tag == 0 && vlen - 1 < raw)) return false;
  H.vtag = tag;
  H.vblob_off = *pos + 1;
  H.vblob_len = tag == 0 ? raw : vlen - 1;
  *pos += vlen;
  return true;
}

__device__ void dp_parse_head(const uint8_t* __restrict__ s, uint64_t len, DpHead& H) {
  memset(&H, 0, sizeof(H));
  H.kind = 1;
  do {
    if (len > 5 && (s[5] & 2)) {  // decimal container (decimal.rs:39-41, 100-168)
      if (len < 19) break;
      if (s[0] != 'F' || s[1] != 'C' || s[2] != 'R' || s[3] != '1' || s[4] != 2) break;
      if (s[7] != DT_DEC128 && s[7] != DT_DEC256) break;
      H.decimal = 1;
      H.wire = s[7];
      H.has_validity = s[5] & 1;
      H.n = ld_u64(s + 8);
      if (H.n > kMaxLogicalD) break;
      H.scale = (int8_t)s[16];
      H.precision = s[17];
      uint32_t nl = s[18];
      if (nl != (H.wire == DT_DEC128 ? 2u : 4u)) break;
      uint64_t pos = 19 + 8ull * nl;
      if (pos > len) break;
      for (uint32_t k = 0; k < nl; k++) H.vmin[k] = ld_u64(s + 19 + 8 * k);
      if (H.has_validity && !dp_validity(s, len, &pos, H.n, H)) break;
      bool ok = true;
      for (uint32_t k = 0; k < nl && ok; k++) {
        uint64_t sl;
        if (rd_varint(s, len, &pos, &sl) != E_OK || sl > len - pos) { ok = false; break; }
        ok = dp_lane_header(s, pos, sl, H.lanes[k]) && !H.lanes[k].has_validity;
        pos += sl;
      }
      if (!ok) break;
      H.nl = nl;
      H.kind = 0;
    } else {
      DpLane& L = H.lanes[0];
      if (!dp_lane_header(s, 0, len, L)) break;
      if (L.dtype == DT_DEC128 || L.dtype == DT_DEC256) break;  // lib.rs:503-505
      H.wire = L.dtype;
      H.n = L.logical_n;
      H.has_validity = L.has_validity;
      uint64_t pos = 16;
      if (H.has_validity && !dp_validity(s, len, &pos, H.n, H)) break;
      L.fstart = pos;
      H.nl = 1;
      H.kind = 0;
    }
  } while (false);
}

__global__ void k_dp_head(const uint8_t* __restrict__ s, uint64_t len, DpHead* __restrict__ out) {
  if (threadIdx.x || blockIdx.x) return;
  DpHead H;
  dp_parse_head(s, len, H);
  *out = H;
}

// Bitmap words of the RAW blob (bits past n cleared) and each word's
// popcount, one word per thread; the word after the last is zeroed (readers
// of whole words stop there).
__global__ void k_dp_bitmap(const uint8_t* __restrict__ s, const DpHead* __restrict__ H, uint32_t* __restrict__ bm32,
                            uint64_t* __restrict__ cnt) {
  const uint8_t* src = s + H->vblob_off;
  uint64_t nb = H->vblob_len, n = H->n, nw = (n + 31) / 32;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w <= nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    if (w < nw) {
      uint64_t b0 = 4 * w;
      if (b0 + 4 <= nb) {
        bits = ld_u32(src + b0);
      } else {
        for (uint64_t k = 0; k < 4 && b0 + k < nb; k++) bits |= (uint32_t)src[b0 + k] << (8 * k);
      }
      uint64_t rem = n - 32 * w;
      if (rem < 32) bits &= (1u << rem) - 1u;
      cnt[w] = (uint64_t)__popc(bits);
    }
    bm32[w] = bits;
  }
}

// RLE blob (validity.rs:92-119): alternating run lengths (LEB128), nulls
// first, read until the runs cover n positions.  One CTA reads the blob 16 KB
// a round: terminator bytes (high bit clear) end varints, a scan numbers
// them, the thread holding a terminator assembles its varint (at most 10
// bytes back, as rd_varint reads), and a scan of the run lengths gives each
// run's end position.  Anything the sequential reader would reject (a run
// past n, a varint over 10 bytes, a blob that ends first) sets H->kind; an
// odd byte after the last run is left unread, as the sequential reader
// leaves it (the round's check covers only varints before the last run).
constexpr int kRleThreads = 1024;
// The whole CTA: run ends of the RLE blob b[0 .. blen) covering n positions;
// false when the sequential reader would reject it.
__device__ bool dp_rle_runs(const uint8_t* __restrict__ b, uint64_t blen, uint64_t n, uint64_t* __restrict__ ends,
                            uint64_t* __restrict__ nruns, uint64_t* s_warp) {
  const int tid = threadIdx.x;
  uint64_t carry_pos = 0, carry_k = 0;
  int64_t prev_term = -1;  // the last terminator before the round (blob offset)
  bool bad = false, done = n == 0;
  for (uint64_t base = 0; base < blen && !done; base += 16ull * kRleThreads) {
    uint64_t a = base + 16ull * tid;
    uint32_t tm = 0;
    for (int i = 0; i < 16; i++)
      if (a + i < blen && !(b[a + i] & 0x80)) tm |= 1u << i;
    int64_t mylast = tm ? (int64_t)(a + 31 - __clz(tm)) : -1;
    uint64_t rk, mt;
    uint64_t k0 = block_excl_scan<ScanSum>((uint64_t)__popc(tm), s_warp, &rk);
    // previous terminator before the thread's bytes: max over earlier threads
    uint64_t pm = block_excl_scan<ScanMax>((uint64_t)(mylast + 1), s_warp, &mt);
    int64_t prev = (int64_t)pm - 1 > prev_term ? (int64_t)pm - 1 : prev_term;
    // the thread's varints: lengths summed in order; a too-long one is bad
    uint64_t sum = 0;
    bool mybad = false;
    {
      int64_t pv = prev;
      uint32_t m = tm;
      while (m) {
        int64_t j = (int64_t)a + (__ffs(m) - 1);
        m &= m - 1;
        int64_t st = pv + 1;
        if (j - st + 1 > 10) mybad = true;
        uint64_t v = 0;
        for (int64_t q = st; q <= j && q < st + 10; q++) v |= (uint64_t)(b[q] & 0x7F) << (7 * (q - st));
        sum += v;
        pv = j;
      }
    }
    uint64_t tot;
    uint64_t sx = block_excl_scan<ScanSum>(sum, s_warp, &tot);
    // write run ends; the first run reaching n ends the reading
    uint64_t pos = carry_pos + sx, k = carry_k + k0;
    bool reach = false, over = false;
    {
      int64_t pv = prev;
      uint32_t m = tm;
      while (m) {
        int64_t j = (int64_t)a + (__ffs(m) - 1);
        m &= m - 1;
        int64_t st = pv + 1;
        uint64_t v = 0;
        for (int64_t q = st; q <= j && q < st + 10; q++) v |= (uint64_t)(b[q] & 0x7F) << (7 * (q - st));
        bool before_end = pos < n;  // this run is read by the sequential reader
        if (before_end) {
          if (v > n - pos) over = true;
          ends[k] = pos + v;
          if (pos + v >= n) {
            reach = true;
            *nruns = k + 1;
          }
        }
        pos += v;
        k++;
        pv = j;
      }
    }
    // a too-long varint counts when it starts before the covering run ends:
    // conservatively, any in a round that reads at least one run
    bad = __syncthreads_or(over || (mybad && carry_pos < n)) || bad;
    done = __syncthreads_or(reach) != 0;
    carry_pos += tot;
    carry_k += rk;
    if ((int64_t)mt - 1 > prev_term) prev_term = (int64_t)mt - 1;
  }
  if (tid == 0 && n == 0) *nruns = 0;
  return !bad && done;
}

__global__ void __launch_bounds__(kRleThreads) k_dp_rle_runs(const uint8_t* __restrict__ s, DpHead* __restrict__ H,
                                                             uint64_t n, uint64_t* __restrict__ ends,
                                                             uint64_t* __restrict__ nruns) {
  __shared__ uint64_t s_warp[33];
  bool ok = dp_rle_runs(s + H->vblob_off, H->vblob_len, n, ends, nruns, s_warp);
  if (threadIdx.x == 0 && !ok) H->kind = 1;  // the host reader reports the error
}

// Bitmap word w (of an n-bit bitmap) from nr run ends: runs alternate null /
// valid from a null run; the word's bits come from the runs overlapping
// [32w, 32w + 32).
__device__ uint32_t dp_rle_word(const uint64_t* __restrict__ ends, uint64_t nr, uint64_t n, uint64_t w) {
  uint64_t lo = w * 32, hi = lo + 32;
  uint32_t bits = 0;
  if (!nr || lo >= n) return 0;
  uint64_t a = 0, z = nr;  // first run whose end is above lo
  while (a < z) {
    uint64_t mid = (a + z) >> 1;
    if (ends[mid] <= lo) a = mid + 1; else z = mid;
  }
  for (uint64_t r = a; r < nr; r++) {
    uint64_t st = r ? ends[r - 1] : 0, en = ends[r];
    if (st >= hi) break;
    if (r & 1) {
      uint64_t x = st > lo ? st : lo, y = en < hi ? en : hi;
      if (y > x) {
        uint32_t len = (uint32_t)(y - x), sh = (uint32_t)(x - lo);
        bits |= (len == 32 ? 0xFFFFFFFFu : ((1u << len) - 1u)) << sh;
      }
    }
  }
  if (hi > n) bits &= (n - lo) >= 32 ? 0xFFFFFFFFu : ((1u << (uint32_t)(n - lo)) - 1u);
  return bits;
}


// Bitmap word w from the run ends: runs alternate null / valid from a null
// run; word w's bits come from the runs overlapping [32w, 32w + 32).
__global__ void k_dp_rle_fill(const DpHead* __restrict__ H, uint64_t n, const uint64_t* __restrict__ ends,
                              const uint64_t* __restrict__ nruns_p, uint32_t* __restrict__ bm32,
                              uint64_t* __restrict__ cnt) {
  uint64_t nw = (n + 31) / 32, nr = H->kind ? 0 : *nruns_p;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw + 1; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bits = w < nw ? dp_rle_word(ends, nr, n, w) : 0u;
    if (w < nw) cnt[w] = (uint64_t)__popc(bits);
    bm32[w] = bits;  // the word past the end stays 0
  }
}

// ---------------------------------------------------------------------------
// Candidates: CTA j of a lane covers kDpChunk positions (dp_thread_cands).
// ---------------------------------------------------------------------------
// Mode ids a frame candidate may carry, as a bit mask (every id is below 64):
// every mode of mode.rs:60-84 except PRED (0).  A PRED payload is bare LEB128
// with no tag or length, so in the zero-rich bytes of bit-packed payloads
// "00 n n n 00 p p p 00" passes as a PRED header everywhere; a stream with
// PRED frames (High/Max only) breaks the chain and is read by the host reader.
constexpr uint64_t kCandModes = (1ull << 1) | (1ull << 2) | (1ull << 3) | (1ull << 4) | (1ull << 5) | (1ull << 7) |
                                (1ull << 9) | (1ull << 11) | (1ull << 17) | (1ull << 19) | (1ull << 20) |
                                (1ull << 25) | (1ull << 29) | (1ull << 45) | (1ull << 50) | (1ull << 51) |
                                (1ull << 52) | (1ull << 53) | (1ull << 54);
static_assert(((kCandModes >> 0) & 1) == 0, "PRED is not a candidate mode");

// Chunk j of a lane starts at the 16-byte aligned address at or below its
// first frame offset, plus j * kDpChunk, and is read in kDpSteps steps of
// kDpThreads * 16 positions; in a step thread t takes the 16 positions from
// 16t: one aligned 16-byte load, and the 8 bytes after it from the next lane
// (the last lane loads them).  Bytes past the buffer read as 0xFF, which no
// test below takes for a header byte.  Returns the candidate positions among
// a .. a+15 as a bit mask (bit i = position a + i).  All 32 lanes of the warp
// call it.
__device__ inline uint64_t dp_chunk_base(const uint8_t* s, const DpLane& L) {
  return L.fstart - (((uintptr_t)(s + L.fstart)) & 15);
}
struct DpWin {
  uint4 v;     // bytes a .. a+15
  uint2 next;  // bytes a+16 .. a+23 (loaded by the warp's last lane only)
};
__device__ __forceinline__ DpWin dp_load(const uint8_t* __restrict__ s, uint64_t buf_len, uint64_t a) {
  DpWin w;
  if (a + 16 <= buf_len) {
    w.v = __ldg(reinterpret_cast<const uint4*>(s + a));
  } else {
    uint32_t q[4] = {0, 0, 0, 0};
    for (int i = 0; i < 16; i++) q[i >> 2] |= (uint32_t)((a + i < buf_len) ? s[a + i] : 0xFF) << (8 * (i & 3));
    w.v = make_uint4(q[0], q[1], q[2], q[3]);
  }
  w.next = make_uint2(0, 0);
  if ((threadIdx.x & 31) == 31) {
    if (a + 24 <= buf_len) {
      w.next = __ldg(reinterpret_cast<const uint2*>(s + a + 16));
    } else {
      uint32_t q[2] = {0, 0};
      for (int i = 0; i < 8; i++) q[i >> 2] |= (uint32_t)((a + 16 + i < buf_len) ? s[a + 16 + i] : 0xFF) << (8 * (i & 3));
      w.next = make_uint2(q[0], q[1]);
    }
  }
  return w;
}

// Per byte of x, 0x80 where the byte AND ~keep is zero (keep = the bits a
// byte may hold), else 0: ((x & 0x7F..) + 0x7F..) sets bit 7 of every byte
// with a low bit set, and x's own bit 7 the others.
template <uint32_t kKeep>
__device__ __forceinline__ uint32_t bytes_within(uint32_t x) {
  constexpr uint32_t kClear = ~(kKeep * 0x01010101u);
  uint32_t t = (x & kClear & 0x7F7F7F7Fu) + 0x7F7F7F7Fu;
  return ~(t | (x & kClear) | 0x7F7F7F7Fu);
}

// The candidates among survivor positions m (bit i: position a + i passed
// the byte tests): mode id, n and plen ranges, then the mode's first decode
// checks.  Out of line: survivors are rare, and one copy of this code keeps
// the scan loop small.
__device__ __noinline__ uint32_t dp_check_survivors(const uint8_t* __restrict__ s, const DpLane& L, uint64_t a,
                                                    uint32_t m, uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3,
                                                    uint32_t x4, uint32_t x5) {
  const uint32_t x[6] = {x0, x1, x2, x3, x4, x5};
  const uint64_t end = L.base + L.len;
  const uint32_t lb = lane_bytes((int)L.dtype);
  uint32_t out = 0;
  while (m) {
    uint32_t i = __ffs(m) - 1;
    m &= m - 1;
    uint32_t k = i >> 2, j = i & 3;
    uint32_t h0 = __funnelshift_r(x[k], x[k + 1], 8 * j);      // mode, n (low 3 bytes)
    uint32_t h1 = __funnelshift_r(x[k + 1], x[k + 2], 8 * j);  // byte +4 (zero), plen (3 bytes)
    uint32_t mode = h0 & 0xFF, n = h0 >> 8, plen = h1 >> 8;
    uint64_t p = a + i;
    if (((kCandModes >> mode) & 1) && n >= 1 && n <= (uint32_t)kMaxBlock && plen <= end - p - 9 &&
        dp_frame_plausible(s, p + 9, n, plen, mode, lb))
      out |= 1u << i;
  }
  return out;
}

__device__ inline uint32_t dp_thread_cands(const uint8_t* __restrict__ s, const DpLane& L, uint64_t a,
                                           const DpWin& W) {
  const uint64_t end = L.base + L.len;
  uint32_t n0 = __shfl_down_sync(0xffffffffu, W.v.x, 1), n1 = __shfl_down_sync(0xffffffffu, W.v.y, 1);
  if ((threadIdx.x & 31) == 31) {
    n0 = W.next.x;
    n1 = W.next.y;
  }
  // positions that can hold a header: from the first frame offset, with 9
  // bytes before the lane's end
  if (a + 15 < L.fstart || a + 9 > end) return 0;
  const uint32_t x[6] = {W.v.x, W.v.y, W.v.z, W.v.w, n0, n1};
  // per byte, 0x80 flags: z = zero; the 4-byte word k of positions 4k..4k+3
  // keeps a position whose mode byte is in 1..63 and whose bytes +4 (top
  // byte of n) and +8 (top byte of plen) are zero
  uint32_t z[6];
#pragma unroll
  for (int k = 0; k < 6; k++) z[k] = bytes_within<0>(x[k]);
  uint32_t m = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint32_t f = bytes_within<0x3F>(x[k]) & ~z[k] & z[k + 1] & z[k + 2];  // bits 7, 15, 23, 31
    m |= (((f >> 7) & 1u) | ((f >> 14) & 2u) | ((f >> 21) & 4u) | ((f >> 28) & 8u)) << (4 * k);
  }
  if (!m) return 0;
  const uint32_t lo = a < L.fstart ? (uint32_t)(L.fstart - a) : 0u;  // first position in range
  const uint64_t last = end - 9;
  const uint32_t hi = a + 15 > last ? (uint32_t)(last - a) : 15u;   // last position in range
  m &= (0xFFFFu << lo) & ((2u << hi) - 1u);
  if (!m) return 0;
  return dp_check_survivors(s, L, a, m, x[0], x[1], x[2], x[3], x[4], x[5]);
}

__device__ __forceinline__ DpCand dp_cand_at(const uint8_t* __restrict__ s, uint64_t p) {
  DpCand c;
  c.pos = p;
  c.n = ld_u32(s + p + 1);
  c.plen_mode = (ld_u32(s + p + 5) << 8) | s[p];
  return c;
}

// The thread's candidate masks of its kDpSteps steps in chunk `chunk`, and
// where its candidates go in the chunk's position order: the step-k ones
// from at[k] (an exclusive scan over the CTA of four 16-bit counts at once).
// Returns the chunk's count.
constexpr uint32_t kDpSlots = 16;
__device__ inline uint64_t dp_chunk_cands(const uint8_t* __restrict__ s, uint64_t buf_len, const DpLane& L,
                                          uint64_t chunk, uint64_t* s_warp, uint32_t m[kDpSteps],
                                          uint64_t a[kDpSteps], uint64_t at[kDpSteps]) {
  const uint64_t base = dp_chunk_base(s, L) + chunk * kDpChunk + 16ull * threadIdx.x;
  DpWin w[kDpSteps];
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {  // every load in flight before any is used
    a[k] = base + (uint64_t)k * kDpStep;
    w[k] = dp_load(s, buf_len, a[k]);
  }
  uint64_t packed = 0;
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {
    m[k] = dp_thread_cands(s, L, a[k], w[k]);
    packed |= (uint64_t)__popc(m[k]) << (16 * k);
  }
  uint64_t tot;
  uint64_t x = block_excl_scan<ScanSum>(packed, s_warp, &tot);  // each field sums at most 16 * kDpThreads
  uint64_t before = 0;
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {
    at[k] = before + ((x >> (16 * k)) & 0xFFFF);
    before += (tot >> (16 * k)) & 0xFFFF;
  }
  return before;
}

// Per chunk: its candidate count, and its first kDpSlots candidates (in
// position order) in the chunk's slots.
__global__ void __launch_bounds__(kDpThreads) k_dp_cand_scan(const uint8_t* __restrict__ s, uint64_t buf_len,
                                                             const DpHead* __restrict__ H, int lane,
                                                             uint64_t* __restrict__ cnt, DpCand* __restrict__ slots) {
  __shared__ uint64_t s_warp[33];
  if (H->kind) {  // uniform over the CTA
    if (threadIdx.x == 0) cnt[blockIdx.x] = 0;
    return;
  }
  const DpLane& L = H->lanes[lane];
  uint32_t m[kDpSteps];
  uint64_t a[kDpSteps], at[kDpSteps];
  uint64_t tot = dp_chunk_cands(s, buf_len, L, blockIdx.x, s_warp, m, a, at);
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {
    uint32_t mk = m[k];
    uint64_t q = at[k];
    while (mk && q < kDpSlots) {
      uint32_t i = __ffs(mk) - 1;
      mk &= mk - 1;
      slots[(uint64_t)blockIdx.x * kDpSlots + q] = dp_cand_at(s, a[k] + i);
      q++;
    }
  }
  if (threadIdx.x == 0) cnt[blockIdx.x] = tot;
}

// Chunk j's candidates to cand[off[j] ..] (off = exclusive scan of the
// counts with one extra entry): from the slots, or by a second pass over a
// chunk with more candidates than slots.
__global__ void __launch_bounds__(kDpThreads) k_dp_cand_compact(const uint8_t* __restrict__ s, uint64_t buf_len,
                                                                const DpHead* __restrict__ H, int lane,
                                                                const uint64_t* __restrict__ off,
                                                                const DpCand* __restrict__ slots, uint64_t cap,
                                                                DpCand* __restrict__ cand) {
  __shared__ uint64_t s_warp[33];
  uint64_t base = off[blockIdx.x], c = off[blockIdx.x + 1] - base;
  if (c == 0 || H->kind) return;
  if (c <= kDpSlots) {
    if (threadIdx.x < c && base + threadIdx.x < cap)
      cand[base + threadIdx.x] = slots[(uint64_t)blockIdx.x * kDpSlots + threadIdx.x];
    return;
  }
  const DpLane& L = H->lanes[lane];
  uint32_t m[kDpSteps];
  uint64_t a[kDpSteps], at[kDpSteps];
  dp_chunk_cands(s, buf_len, L, blockIdx.x, s_warp, m, a, at);
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {
    uint32_t mk = m[k];
    uint64_t q = base + at[k];
    while (mk) {
      uint32_t i = __ffs(mk) - 1;
      mk &= mk - 1;
      if (q < cap) cand[q] = dp_cand_at(s, a[k] + i);
      q++;
    }
  }
}

// ---------------------------------------------------------------------------
// Chain resolution and item layout (one CTA per lane).
// ---------------------------------------------------------------------------
// ALP-RD header up to the rights tag (alp_rd.rs:208-250); false when it does
// not parse (the frame is then listed and the frame kernel reports it).
__device__ bool dp_alprd_tags(const uint8_t* p, uint64_t plen, uint64_t* nexc, uint32_t* ctag, uint32_t* rtag) {
  if (plen < 2 || p[1] > 8) return false;
  uint64_t pos = 2 + 8ull * p[1], clen = 0;
  if (pos > plen || rd_varint(p, plen, &pos, nexc) != E_OK) return false;
  for (uint64_t x = 0; x < *nexc; x++) {
    uint64_t pp;
    if (rd_varint(p, plen, &pos, &pp) != E_OK || plen - pos < 8) return false;
    pos += 8;
  }
  if (pos >= plen) return false;
  *ctag = p[pos++];
  if (rd_varint(p, plen, &pos, &clen) != E_OK || clen > plen - pos) return false;
  pos += clen;
  if (pos >= plen) return false;
  *rtag = p[pos];
  return true;
}

// Whether a listed frame may hold an entropy-coded part and so needs a
// device area (the host reader's entropy_frame_h, the same rules).
__device__ bool dp_entropy_frame(const uint8_t* p, uint64_t plen, uint32_t mode) {
  switch (mode) {
    case 11: case 7: case 20: case 45: case 0: case 25: case 29: case 4:
      return true;
    case 17:
      return plen < 2 || p[0] == 1;
    case 52: {
      uint64_t nexc = 0;
      uint32_t ct = 0, rt = 0;
      return !dp_alprd_tags(p, plen, &nexc, &ct, &rt) || ct == 1 || rt == 1;
    }
    case 19: {
      uint64_t pos = 0, card = 0, vlen = 0;
      if (rd_varint(p, plen, &pos, &card) != E_OK || pos >= plen) return true;
      uint32_t vtag = p[pos++];
      if (vtag == 2) return true;
      if (rd_varint(p, plen, &pos, &vlen) != E_OK || vlen > plen - pos) return true;
      pos += vlen;
      return pos >= plen || p[pos] == 1;
    }
    default:
      return false;
  }
}

struct FrameItems {
  uint32_t nmain, npre;
  bool list, scan, dict;
  uint64_t ent;
};

// The host reader's build_items for one frame.
__device__ FrameItems dp_frame_items(const uint8_t* p, uint64_t n, uint64_t plen, uint32_t mode, uint32_t plog2) {
  FrameItems r{0, 0, false, false, false, 0};
  uint32_t nv = (uint32_t)((n + 511) / 512);
  switch (mode) {
    case 5: case 1: case 2: case 50: case 9:
      r.nmain = nv;
      break;
    case 17:
      if (plen >= 2 && p[0] == 0) r.nmain = nv; else r.list = true;
      break;
    case 51:
      r.npre = r.nmain = nv;
      r.scan = true;
      break;
    case 3:
      r.npre = r.nmain = (uint32_t)((plen + kXorzItemBytes - 1) / kXorzItemBytes);
      r.scan = true;
      break;
    case 53: {
      uint64_t pos = 0, nr = 0;
      if (rd_varint(p, plen, &pos, &nr) != E_OK || nr > n) {
        r.list = true;
        break;
      }
      r.npre = (uint32_t)((nr + 1023) / 1024);
      r.nmain = nv;
      r.scan = true;
      break;
    }
    case 52: {  // one walk of the exception list gives both the items and the entropy rule
      uint64_t nexc = 1;
      uint32_t ct = 1, rt = 1;
      bool ok = dp_alprd_tags(p, plen, &nexc, &ct, &rt);
      r.dict = true;
      if (ok && nexc == 0 && ct == 0 && rt == 0) {
        r.nmain = nv;
      } else {
        r.list = true;
        if (!ok || ct == 1 || rt == 1) r.ent = ent_area_bytes(n, mode, plog2);
      }
      return r;
    }
    default:
      r.list = true;
      break;
  }
  r.dict = mode == 19 || mode == 53 || mode == 52;
  if (r.list && dp_entropy_frame(p, plen, mode)) r.ent = ent_area_bytes(n, mode, plog2);
  return r;
}

// Per candidate (one thread each): its successor, the candidate at
// pos + 9 + plen (binary search over the later candidates), or ~0.
__global__ void k_dp_succ(const DpHead* __restrict__ H, const DpCand* __restrict__ cand,
                          const uint64_t* __restrict__ d_ncand, uint64_t cap, DpNode* __restrict__ nodes) {
  uint64_t K = *d_ncand;
  if (H->kind || K > cap) return;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < K; i += (uint64_t)gridDim.x * blockDim.x) {
    DpCand c = cand[i];
    uint64_t target = c.pos + 9 + (c.plen_mode >> 8);
    uint64_t lo = i + 1, hi = K;
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if (cand[mid].pos < target) lo = mid + 1; else hi = mid;
    }
    nodes[i].succ = (lo < K && cand[lo].pos == target) ? (uint32_t)lo : kNone;
  }
}

// The lane's value count, or ~0 when the lane cannot be read here (a decimal
// limb whose count is not the column's valid count).
__device__ inline uint64_t dp_lane_total(const DpHead* H, const DpLane& L, const uint64_t* d_nvalid) {
  if (H->decimal) {
    uint64_t nv = H->has_validity ? *d_nvalid : H->n;
    return L.logical_n == nv ? nv : ~0ull;
  }
  return L.has_validity ? *d_nvalid : L.logical_n;
}

// One CTA: marks spread from the first frame (candidate 0, which must sit at
// the lane's first frame offset) along the successors by pointer doubling,
// then the marked candidates (the chain's frames, in position order) are
// listed in fidx.  ctl[0] = 0 when the lane cannot be read here, ctl[1] = the
// number of marked candidates.
__global__ void __launch_bounds__(kChainThreads) k_dp_marks(const DpHead* __restrict__ H, int lane,
                                                            const uint64_t* __restrict__ d_nvalid,
                                                            const DpCand* __restrict__ cand,
                                                            const DpNode* __restrict__ nodes,
                                                            const uint64_t* __restrict__ d_ncand, uint64_t cap,
                                                            uint32_t* __restrict__ gJ, uint8_t* __restrict__ marks,
                                                            uint64_t* __restrict__ ctl) {
  extern __shared__ __align__(16) uint8_t dsm[];
  __shared__ uint64_t s_warp[33];
  const int tid = threadIdx.x;
  if (H->kind) {
    if (tid == 0) ctl[0] = ctl[1] = 0;
    return;
  }
  const DpLane& L = H->lanes[lane];
  uint64_t K = *d_ncand, n_total = dp_lane_total(H, L, d_nvalid);
  // candidates start at the first frame offset, so the first frame is
  // candidate 0 or not a candidate at all
  bool good = n_total != ~0ull && (n_total == 0 || (K <= cap && K > 0 && cand[0].pos == L.fstart));
  if (!good || n_total == 0) {
    if (tid == 0) {
      ctl[0] = good;
      ctl[1] = 0;
    }
    return;
  }
  const uint32_t M = (uint32_t)K;
  // successor tables (two, for the doubling) and the marks: shared memory
  // when they fit
  uint32_t *J0, *J1;
  if ((uint64_t)M * 9 + 16 <= kDpChainSmem) {
    J0 = reinterpret_cast<uint32_t*>(dsm);
    J1 = J0 + M;
    marks = reinterpret_cast<uint8_t*>(J1 + M);
  } else {
    J0 = gJ;
    J1 = gJ + M;
  }
  for (uint32_t i = tid; i < M; i += kChainThreads) {
    J0[i] = nodes[i].succ;
    marks[i] = i == 0;
  }
  __syncthreads();
  // after round r every chain frame within 2^(r+1) - 1 jumps of the first is
  // marked (a mark set during a round may be used in the same round: it is a
  // chain frame too)
  uint32_t rounds = 1;
  while ((1ull << rounds) <= M) rounds++;
  for (uint32_t r = 0; r < rounds; r++) {
    for (uint32_t i = tid; i < M; i += kChainThreads) {
      uint32_t j = J0[i];
      if (j != kNone && marks[i]) marks[j] = 1;
      J1[i] = j == kNone ? kNone : J0[j];
    }
    __syncthreads();
    uint32_t* t = J0;
    J0 = J1;
    J1 = t;
  }
  // the marked candidates in order (gJ is free again: the doubling is done)
  uint64_t carry = 0;
  for (uint32_t t0 = 0; t0 < M; t0 += kChainThreads) {
    uint32_t i = t0 + tid;
    bool f = i < M && marks[i];
    uint64_t tot;
    uint64_t x = block_excl_scan<ScanSum>(f ? 1ull : 0ull, s_warp, &tot);
    if (f) gJ[carry + x] = i;
    carry += tot;
  }
  if (tid == 0) {
    ctl[0] = 1;
    ctl[1] = carry;
  }
}

// An ALP-RD frame's exception list (records of a varint position and an
// 8-byte left part) is walked record by record, each read depending on the
// one before; the warp first pulls the list's cache lines into L1 so that the
// walk's reads hit there.
__device__ __forceinline__ void dp_warp_prefetch_alprd(const uint8_t* p, uint64_t plen, uint32_t mode) {
  if (mode != 52 || plen < 2) return;
  const int l = threadIdx.x & 31;
  uint64_t pos = 2 + 8ull * p[1], nexc = 0;
  if (pos > plen || rd_varint(p, plen, &pos, &nexc) != E_OK) return;
  uint64_t end = nexc > plen ? plen : qmin(plen, pos + 18 * nexc + 32);
  for (uint64_t o = pos + 128ull * l; o < end; o += 128ull * 32)
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p + o));
}

// The warp items of every marked candidate (dp_frame_items), across the GPU:
// nodes[j] for the j-th marked candidate, its candidate index in .succ.  One
// warp per frame: the prefetch above, then lane 0 counts the items.
__global__ void k_dp_items(const uint8_t* __restrict__ s, const DpHead* __restrict__ H, int lane,
                           const DpCand* __restrict__ cand, const uint32_t* __restrict__ fidx,
                           const uint64_t* __restrict__ ctl, DpNode* __restrict__ nodes) {
  if (!ctl[0]) return;
  uint64_t F = ctl[1];
  uint32_t plog2 = H->lanes[lane].plog2;
  const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t j = w0; j < F; j += nw) {
    uint32_t i = fidx[j];
    DpCand c = cand[i];
    const uint8_t* p = s + c.pos + 9;
    dp_warp_prefetch_alprd(p, c.plen_mode >> 8, c.plen_mode & 0xFF);
    if ((threadIdx.x & 31) != 0) continue;
    FrameItems it = dp_frame_items(p, c.n, c.plen_mode >> 8, c.plen_mode & 0xFF, plog2);
    DpNode d;
    d.succ = i;
    d.nmain = it.nmain;
    d.npre = it.npre;
    d.flags = (it.list ? 1u : 0u) | (it.scan ? 2u : 0u) | (it.dict ? 4u : 0u);
    d.ent = it.ent;
    nodes[j] = d;
  }
}

// One CTA: the chain's frames (nodes[0 .. F), in position order) cut at the
// lane's value count and laid out as the block decoder's tables (the values
// before a frame only grow along the chain, so the kept frames, those
// starting below the count, are a prefix).
__global__ void __launch_bounds__(kChainThreads) k_dp_layout(const DpHead* __restrict__ H, int lane,
                                                             const uint64_t* __restrict__ d_nvalid,
                                                             const DpCand* __restrict__ cand,
                                                             const DpNode* __restrict__ nodes,
                                                             const uint64_t* __restrict__ d_ncand,
                                                             const uint64_t* __restrict__ ctl, DpTables T,
                                                             DpLaneOut* __restrict__ out) {
  __shared__ uint64_t s_warp[33];
  const int tid = threadIdx.x;
  DpLaneOut R;
  memset(&R, 0, sizeof(R));
  R.status = 1;
  R.ncand = *d_ncand;
  if (!ctl[0]) {
    if (tid == 0) *out = R;
    return;
  }
  const DpLane& L = H->lanes[lane];
  uint64_t n_total = dp_lane_total(H, L, d_nvalid);
  if (n_total == 0) {  // no frame is read (decoder.rs: the walk runs while counted < n)
    R.status = 0;
    if (tid == 0) {
      T.main_off[0] = 0;
      *out = R;
    }
    return;
  }
  const uint64_t F = ctl[1];
  uint64_t carry_f = 0, carry_v = 0, carry_main = 0, carry_pre = 0, carry_list = 0, carry_ent = 0;
  bool scan = false, dict = false, stop = false, fail = false;
  for (uint64_t t0 = 0; t0 < F && !stop; t0 += kChainThreads) {
    uint64_t j = t0 + tid;
    bool have = j < F;
    DpCand c;
    c.pos = 0;
    c.n = 0;
    c.plen_mode = 0;
    DpNode nd;
    memset(&nd, 0, sizeof(nd));
    if (have) {
      nd = nodes[j];
      c = cand[nd.succ];
    }
    uint64_t vx = block_excl_scan<ScanSum>(have ? (uint64_t)c.n : 0ull, s_warp, nullptr);
    uint64_t voff = carry_v + vx;
    bool keep = have && voff < n_total;
    bool list = keep && (nd.flags & 1);
    bool last = keep && voff + c.n >= n_total;
    stop = __syncthreads_or(last) != 0;
    // past the count: CorruptPayload, which the host reader reports
    fail = (__syncthreads_or(last && voff + c.n > n_total) != 0) || fail;
    uint64_t tf, tv, tp, tl, te;
    uint64_t fx = block_excl_scan<ScanSum>(keep ? 1ull : 0ull, s_warp, &tf);
    block_excl_scan<ScanSum>(keep ? (uint64_t)c.n : 0ull, s_warp, &tv);
    uint64_t packed = keep ? ((uint64_t)nd.npre << 32 | nd.nmain) : 0ull;
    uint64_t px = block_excl_scan<ScanSum>(packed, s_warp, &tp);
    uint64_t lx = block_excl_scan<ScanSum>(list ? 1ull : 0ull, s_warp, &tl);
    uint64_t ex = block_excl_scan<ScanSum>(keep ? nd.ent : 0ull, s_warp, &te);
    if (keep) {
      uint64_t f = carry_f + fx;
      FrameDesc d;
      d.payload_off = c.pos + 9;
      d.value_off = voff;
      d.n = c.n;
      d.plen = c.plen_mode >> 8;
      d.mode = c.plen_mode & 0xFF;
      d.aux = nd.ent ? (uint32_t)(1 + (carry_ent + ex) / 128) : 0u;
      T.frames[f] = d;
      T.frame_pre[f] = make_uint2((uint32_t)(carry_pre + (px >> 32)), nd.npre);
      T.main_off[f] = carry_main + (px & 0xFFFFFFFFull);
      if (list) T.list[carry_list + lx] = (uint32_t)f;
    }
    scan = (__syncthreads_or(keep && (nd.flags & 2)) != 0) || scan;
    dict = (__syncthreads_or(keep && (nd.flags & 4)) != 0) || dict;
    carry_f += tf;
    carry_v += tv;
    carry_main += tp & 0xFFFFFFFFull;
    carry_pre += tp >> 32;
    carry_list += tl;
    carry_ent += te;
  }
  if (tid == 0) {
    R.status = (fail || !stop || carry_v != n_total) ? 1u : 0u;
    R.nframes = (uint32_t)carry_f;
    R.nmain = (uint32_t)carry_main;
    R.npre = (uint32_t)carry_pre;
    R.nlist = (uint32_t)carry_list;
    R.need_scan = scan;
    R.any_dict = dict;
    R.ent_bytes = carry_ent;
    T.main_off[carry_f] = carry_main;
    *out = R;
  }
}

// Warp items of every frame: main items (frame, k) for k < its count, and the
// prepass items likewise (launch_decode_items' tables).
__global__ void k_dp_expand(const DpLaneOut* __restrict__ out, DpTables T) {
  uint32_t nf = out->status ? 0u : out->nframes;
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t f = warp; f < nf; f += nwarps) {
    uint64_t m0 = T.main_off[f], m1 = T.main_off[f + 1];
    for (uint64_t k = m0 + lane; k < m1; k += 32) T.main_items[k] = ItemRef{f, (uint32_t)(k - m0)};
    uint2 fp = T.frame_pre[f];
    for (uint32_t k = lane; k < fp.y; k += 32) T.pre_items[fp.x + k] = ItemRef{f, k};
  }
}

std::atomic<unsigned long long> g_chain_attr{0};

}  // namespace

void launch_dp_head(const uint8_t* s, uint64_t len, DpHead* H, cudaStream_t st) {
  k_dp_head<<<1, 32, 0, st>>>(s, len, H);
  count_launches(1);
}

void launch_dp_bitmap(const uint8_t* s, const DpHead* H, uint64_t n, uint8_t* bm, uint64_t* cnt, cudaStream_t st) {
  uint64_t nw = (n + 31) / 32 + 1;
  unsigned g = (unsigned)qmin((nw + 255) / 256, 148ull * 16);
  k_dp_bitmap<<<g, 256, 0, st>>>(s, H, reinterpret_cast<uint32_t*>(bm), cnt);
  count_launches(1);
}

void launch_dp_bitmap_rle(const uint8_t* s, DpHead* H, uint64_t n, uint64_t* ends, uint64_t* nruns, uint8_t* bm,
                          uint64_t* cnt, cudaStream_t st) {
  k_dp_rle_runs<<<1, kRleThreads, 0, st>>>(s, H, n, ends, nruns);
  uint64_t nw = (n + 31) / 32 + 1;
  unsigned g = (unsigned)qmin((nw + 255) / 256, 148ull * 8);
  k_dp_rle_fill<<<g, 256, 0, st>>>(H, n, ends, nruns, reinterpret_cast<uint32_t*>(bm), cnt);
  count_launches(2);
}

uint64_t dp_chunks(uint64_t lane_frames_bytes) {
  return lane_frames_bytes ? (lane_frames_bytes + 15 + kDpChunk - 1) / kDpChunk : 0;  // chunks start up to 15 bytes early
}
uint64_t dp_slot_bytes(uint64_t lane_frames_bytes) { return dp_chunks(lane_frames_bytes) * kDpSlots * sizeof(DpCand); }

void launch_dp_candidates(const uint8_t* s, uint64_t buf_len, const DpHead* H, int lane, uint64_t lane_frames_bytes,
                          uint64_t* cnt, DpCand* slots, uint64_t* tile_tmp, uint64_t* d_ncand, DpCand* cand,
                          uint64_t cap, cudaStream_t st) {
  // cnt has nchunks + 1 entries: the counts, then 0, so that after the
  // exclusive scan cnt[j + 1] - cnt[j] is chunk j's count
  uint64_t nchunks = dp_chunks(lane_frames_bytes);
  if (nchunks) k_dp_cand_scan<<<(unsigned)nchunks, kDpThreads, 0, st>>>(s, buf_len, H, lane, cnt, slots);
  cudaMemsetAsync(cnt + nchunks, 0, 8, st);
  launch_scan_sum(cnt, cnt, nchunks + 1, tile_tmp, d_ncand, st);
  if (nchunks)
    k_dp_cand_compact<<<(unsigned)nchunks, kDpThreads, 0, st>>>(s, buf_len, H, lane, cnt, slots, cap, cand);
  count_launches(nchunks ? 2 : 0);
}

void launch_dp_chain(const uint8_t* s, const DpHead* H, int lane, const uint64_t* d_nvalid, const DpCand* cand,
                     const uint64_t* d_ncand, uint64_t cap, DpNode* nodes, uint32_t* gJ, uint8_t* gmarks,
                     uint64_t* d_ctl, const DpTables& T, DpLaneOut* out, cudaStream_t st) {
  once_per_device(g_chain_attr, [] {
    cudaFuncSetAttribute(k_dp_marks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDpChainSmem);
  });
  unsigned g = (unsigned)qmin((cap + 255) / 256, 148ull * 4);
  k_dp_succ<<<g, 256, 0, st>>>(H, cand, d_ncand, cap, nodes);
  k_dp_marks<<<1, kChainThreads, kDpChainSmem, st>>>(H, lane, d_nvalid, cand, nodes, d_ncand, cap, gJ, gmarks, d_ctl);
  k_dp_items<<<g, 256, 0, st>>>(s, H, lane, cand, gJ, d_ctl, nodes);
  k_dp_layout<<<1, kChainThreads, 0, st>>>(H, lane, d_nvalid, cand, nodes, d_ncand, d_ctl, T, out);
  k_dp_expand<<<148 * 2, 256, 0, st>>>(out, T);
  count_launches(5);
}


// ===========================================================================
// Batches: every column of a batch read by one launch per kernel class.  A
// column's work items (bitmap words, candidate chunks, candidates) are found
// from its place in the batch's arrays by binary search over the columns'
// offsets, and the per-column steps (the chain doubling, the layout) take one
// CTA per column.  The same device functions as the single-column reader.
// ===========================================================================
namespace {

// The lane owning position `x` of an array laid out by the nondecreasing
// offsets first[0 .. n] (first[n] = the total): the last i with first[i] <= x.
__device__ inline int dp_owner(const uint64_t* first, int n, uint64_t x) {
  int lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (first[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void k_dpb_heads(const uint8_t* const* __restrict__ srcs, const uint64_t* __restrict__ lens, int n,
                            DpHead* __restrict__ H) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  DpHead h;
  dp_parse_head(srcs[i], lens[i], h);
  H[i] = h;
}

// The run ends of every lane with an RLE validity blob: one CTA each
// (rle_cols lists them).  A blob the sequential reader rejects marks the
// lane (status 1), which the single-column path then reads.
__global__ void __launch_bounds__(kRleThreads) k_dpb_rle_runs(DpBatch B) {
  __shared__ uint64_t s_warp[33];
  int c = (int)B.rle_cols[blockIdx.x];
  const DpBLane& Ln = B.lanes[c];
  bool ok = dp_rle_runs(Ln.s + Ln.vblob_off, Ln.vblob_len, Ln.bm_n, B.rle_ends + Ln.rle_off, B.rle_nruns + c,
                        s_warp);
  if (threadIdx.x == 0 && !ok) {
    B.out[c].status = 1;
    B.rle_nruns[c] = 0;
  }
}

// Bitmap words of every column with a bitmap (k_dp_bitmap's and
// k_dp_rle_fill's work), their popcounts, and the caller's bitmap bytes.
// word_first[c] = lanes[c].word0.
__global__ void k_dpb_bitmap(DpBatch B, const uint64_t* __restrict__ word_first) {
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < B.words;
       w += (uint64_t)gridDim.x * blockDim.x) {
    int c = dp_owner(word_first, B.nlanes, w);
    const DpBLane& Ln = B.lanes[c];
    uint64_t k = w - Ln.word0;
    uint32_t bits = 0;
    if (Ln.has_bm && k < Ln.nw && Ln.vtag == 1) {
      uint64_t n = Ln.bm_n, nb = (n + 7) / 8, b0 = 4 * k;
      bits = dp_rle_word(B.rle_ends + Ln.rle_off, B.rle_nruns[c], n, k);
      if (Ln.valid_out)
        for (uint64_t q = 0; q < 4 && b0 + q < nb; q++) Ln.valid_out[b0 + q] = (uint8_t)(bits >> (8 * q));
    } else if (Ln.has_bm && k < Ln.nw) {
      const uint8_t* src = Ln.s + Ln.vblob_off;
      uint64_t n = Ln.bm_n, nb = (n + 7) / 8, b0 = 4 * k;
      if (b0 + 4 <= nb) {
        bits = ld_u32(src + b0);
      } else {
        for (uint64_t q = 0; q < 4 && b0 + q < nb; q++) bits |= (uint32_t)src[b0 + q] << (8 * q);
      }
      uint64_t rem = n - 32 * k;
      if (rem < 32) bits &= (1u << rem) - 1u;
      if (Ln.valid_out)
        for (uint64_t q = 0; q < 4 && b0 + q < nb; q++) Ln.valid_out[b0 + q] = (uint8_t)(bits >> (8 * q));
    }
    B.bm32[w] = bits;
    B.ranks[w] = (uint64_t)__popc(bits);
  }
}

// Per column: its valid count and the global rank at its first word.
__global__ void k_dpb_lane_base(DpBatch B) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= B.nlanes) return;
  const DpBLane& Ln = B.lanes[c];
  uint64_t base = B.ranks[Ln.word0];
  B.rbase[c] = base;
  B.out[c].nvalid = Ln.has_bm ? B.ranks[Ln.word0 + Ln.nw] - base : Ln.bm_n;
}

// Column-relative ranks, then the select tables (k_select_table per column).
__global__ void k_dpb_ranks(DpBatch B, const uint64_t* __restrict__ word_first) {
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < B.words;
       w += (uint64_t)gridDim.x * blockDim.x) {
    int c = dp_owner(word_first, B.nlanes, w);
    B.ranks[w] -= B.rbase[c];
  }
}
__global__ void k_dpb_select(DpBatch B, const uint64_t* __restrict__ word_first) {
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < B.words;
       w += (uint64_t)gridDim.x * blockDim.x) {
    int c = dp_owner(word_first, B.nlanes, w);
    const DpBLane& Ln = B.lanes[c];
    uint64_t k = w - Ln.word0;
    if (!Ln.has_bm || Ln.decimal || k >= Ln.nw) continue;
    uint32_t bits = B.bm32[w];
    uint64_t r = B.ranks[w], cnt = (uint64_t)__popc(bits);
    uint64_t m = (r + 511) / 512 * 512;
    if (m < r + cnt) {
      uint32_t x = bits;
      for (uint64_t q = m - r; q; q--) x &= x - 1u;
      B.sel[Ln.sel0 + m / 512] = k * 32 + (uint64_t)(__ffs(x) - 1);
    }
  }
}

__global__ void __launch_bounds__(kDpThreads) k_dpb_cand_scan(DpBatch B) {
  __shared__ uint64_t s_warp[33];
  __shared__ int s_c;
  if (threadIdx.x == 0) s_c = dp_owner(B.chunk0, B.nlanes, blockIdx.x);
  __syncthreads();
  const DpBLane& Ln = B.lanes[s_c];
  uint64_t chunk = blockIdx.x - Ln.chunk0;
  uint32_t m[kDpSteps];
  uint64_t a[kDpSteps], at[kDpSteps];
  uint64_t tot = dp_chunk_cands(Ln.s, Ln.buf_len, Ln.L, chunk, s_warp, m, a, at);
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {
    uint32_t mk = m[k];
    uint64_t q = at[k];
    while (mk && q < kDpSlots) {
      uint32_t i = __ffs(mk) - 1;
      mk &= mk - 1;
      B.slots[(uint64_t)blockIdx.x * kDpSlots + q] = dp_cand_at(Ln.s, a[k] + i);
      q++;
    }
  }
  if (threadIdx.x == 0) B.cnt[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(kDpThreads) k_dpb_cand_compact(DpBatch B) {
  __shared__ uint64_t s_warp[33];
  __shared__ int s_c;
  uint64_t base = B.cnt[blockIdx.x], c = B.cnt[blockIdx.x + 1] - base;
  if (c == 0) return;
  if (threadIdx.x == 0) s_c = dp_owner(B.chunk0, B.nlanes, blockIdx.x);
  __syncthreads();
  const int lane = s_c;
  if (c <= kDpSlots) {
    if (threadIdx.x < c && base + threadIdx.x < B.cap) {
      B.cand[base + threadIdx.x] = B.slots[(uint64_t)blockIdx.x * kDpSlots + threadIdx.x];
      B.cand_lane[base + threadIdx.x] = (uint32_t)lane;
    }
    return;
  }
  const DpBLane& Ln = B.lanes[lane];
  uint32_t m[kDpSteps];
  uint64_t a[kDpSteps], at[kDpSteps];
  dp_chunk_cands(Ln.s, Ln.buf_len, Ln.L, blockIdx.x - Ln.chunk0, s_warp, m, a, at);
#pragma unroll
  for (int k = 0; k < kDpSteps; k++) {
    uint32_t mk = m[k];
    uint64_t q = base + at[k];
    while (mk) {
      uint32_t i = __ffs(mk) - 1;
      mk &= mk - 1;
      if (q < B.cap) {
        B.cand[q] = dp_cand_at(Ln.s, a[k] + i);
        B.cand_lane[q] = (uint32_t)lane;
      }
      q++;
    }
  }
}

// The candidate range [lo, hi) of column c (the exclusive scan of the chunk
// counts, read at the column's first chunks).
__device__ inline void dpb_range(const DpBatch& B, int c, uint64_t* lo, uint64_t* hi) {
  *lo = B.cnt[B.chunk0[c]];
  *hi = B.cnt[B.chunk0[c + 1]];
}

__global__ void k_dpb_succ(DpBatch B) {
  uint64_t K = B.cnt[B.chunks];
  if (K > B.cap) return;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < K; i += (uint64_t)gridDim.x * blockDim.x) {
    int c = (int)B.cand_lane[i];
    uint64_t lo, hi;
    dpb_range(B, c, &lo, &hi);
    DpCand cd = B.cand[i];
    uint64_t target = cd.pos + 9 + (cd.plen_mode >> 8);
    uint64_t a = i + 1, z = hi;
    while (a < z) {
      uint64_t mid = (a + z) >> 1;
      if (B.cand[mid].pos < target) a = mid + 1; else z = mid;
    }
    B.nodes[i].succ = (a < hi && B.cand[a].pos == target) ? (uint32_t)(a - lo) : kNone;  // column-relative
  }
}

// The values a column's frames hold (its valid count or n).
// (~0 for a decimal limb lane whose count is not the container's valid
// count: the single-column path reports it.)
__device__ inline uint64_t dpb_total(const DpBatch& B, int c) {
  const DpBLane& Ln = B.lanes[c];
  if (Ln.decimal) {
    uint64_t nv = B.out[Ln.vlane].nvalid;
    return Ln.L.logical_n == nv ? nv : ~0ull;
  }
  return Ln.has_bm ? B.out[c].nvalid : Ln.L.logical_n;
}

// One CTA per column: k_dp_marks over the column's candidates.  nmarked = 0
// and status 1 when the chain cannot be resolved; status 3 for a column with
// no valid value (left to the single-column path, which zero-fills it).
__global__ void __launch_bounds__(kChainThreads) k_dpb_marks(DpBatch B) {
  extern __shared__ __align__(16) uint8_t dsm[];
  __shared__ uint64_t s_warp[33];
  const int c = blockIdx.x, tid = threadIdx.x;
  const DpBLane& Ln = B.lanes[c];
  uint64_t Ktot = B.cnt[B.chunks];
  uint64_t lo, hi;
  dpb_range(B, c, &lo, &hi);
  uint64_t n_total = dpb_total(B, c);
  bool good = Ktot <= B.cap && n_total > 0 && n_total != ~0ull && hi > lo && B.cand[lo].pos == Ln.L.fstart &&
              B.out[c].status == 0;
  if (!good) {
    __syncthreads();  // every thread has read the status
    if (tid == 0) {
      B.out[c].nmarked = 0;
      if (B.out[c].status == 0) B.out[c].status = n_total == 0 && Ktot <= B.cap ? 3u : 1u;  // 3: no value
    }
    return;
  }
  const uint32_t M = (uint32_t)(hi - lo);
  uint32_t *J0, *J1;
  uint8_t* marks;
  if ((uint64_t)M * 9 + 16 <= kDpChainSmem) {
    J0 = reinterpret_cast<uint32_t*>(dsm);
    J1 = J0 + M;
    marks = reinterpret_cast<uint8_t*>(J1 + M);
  } else {
    J0 = B.gJ + 2 * lo;
    J1 = J0 + M;
    marks = B.gmarks + lo;
  }
  for (uint32_t i = tid; i < M; i += kChainThreads) {
    J0[i] = B.nodes[lo + i].succ;
    marks[i] = i == 0;
  }
  __syncthreads();
  uint32_t rounds = 1;
  while ((1ull << rounds) <= M) rounds++;
  for (uint32_t r = 0; r < rounds; r++) {
    for (uint32_t i = tid; i < M; i += kChainThreads) {
      uint32_t j = J0[i];
      if (j != kNone && marks[i]) marks[j] = 1;
      J1[i] = j == kNone ? kNone : J0[j];
    }
    __syncthreads();
    uint32_t* t = J0;
    J0 = J1;
    J1 = t;
  }
  uint64_t carry = 0;
  for (uint32_t t0 = 0; t0 < M; t0 += kChainThreads) {
    uint32_t i = t0 + tid;
    bool f = i < M && marks[i];
    uint64_t tot;
    uint64_t x = block_excl_scan<ScanSum>(f ? 1ull : 0ull, s_warp, &tot);
    if (f) B.flist[lo + carry + x] = i;  // the chain's candidates (column-relative), in order
    carry += tot;
  }
  if (tid == 0) {
    B.out[c].nmarked = carry;
    B.out[c].status = 0;
  }
}

// One CTA: exclusive scans over the columns (mode 0: frame bases from the
// chain lengths; mode 1: item, prepass and list bases from the layouts).
__global__ void __launch_bounds__(1024) k_dpb_lane_scan(DpBatch B, int mode) {
  __shared__ uint64_t s_warp[33];
  uint64_t c0 = 0, c1 = 0, c2 = 0, any = 0;
  for (int b = 0; b < B.nlanes; b += 1024) {
    int c = b + threadIdx.x;
    bool in = c < B.nlanes;
    DpBLaneOut o;
    memset(&o, 0, sizeof(o));
    if (in) o = B.out[c];
    if (mode == 0) {
      uint64_t t;
      uint64_t x = block_excl_scan<ScanSum>(in ? o.nmarked : 0ull, s_warp, &t);
      if (in) B.out[c].fbase = c0 + x;
      c0 += t;
    } else {
      bool ok = in && o.status == 0;
      uint64_t t0, t1, t2;
      uint64_t x0 = block_excl_scan<ScanSum>(ok ? (uint64_t)o.nmain : 0ull, s_warp, &t0);
      uint64_t x1 = block_excl_scan<ScanSum>(ok ? (uint64_t)o.npre : 0ull, s_warp, &t1);
      uint64_t x2 = block_excl_scan<ScanSum>(ok ? (uint64_t)o.nlist : 0ull, s_warp, &t2);
      if (in) {
        B.out[c].main_base = c0 + x0;
        B.out[c].pre_base = c1 + x1;
        B.out[c].list_base = c2 + x2;
      }
      any |= (uint64_t)__syncthreads_or(ok && o.need_scan);
      c0 += t0;
      c1 += t1;
      c2 += t2;
    }
  }
  if (threadIdx.x == 0) {
    if (mode == 0) {
      B.tot->nframes = c0;
    } else {
      B.tot->nmain = c0;
      B.tot->npre = c1;
      B.tot->nlist = c2;
      B.tot->need_scan = (uint32_t)any;
    }
  }
}

// Warp items of every chain frame (dp_frame_items), across the GPU: slot j of
// column c's candidate range holds its j-th chain frame.
__global__ void k_dpb_items(DpBatch B) {
  uint64_t K = B.cnt[B.chunks];
  if (K > B.cap) return;
  const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t j = w0; j < K; j += nw) {  // one warp per slot, as k_dp_items
    int c = (int)B.cand_lane[j];
    uint64_t lo = B.cnt[B.chunk0[c]];
    if (j - lo >= B.out[c].nmarked) continue;
    const DpBLane& Ln = B.lanes[c];
    uint64_t i = lo + B.flist[j];
    DpCand cd = B.cand[i];
    dp_warp_prefetch_alprd(Ln.s + cd.pos + 9, cd.plen_mode >> 8, cd.plen_mode & 0xFF);
    if ((threadIdx.x & 31) != 0) continue;
    FrameItems it = dp_frame_items(Ln.s + cd.pos + 9, cd.n, cd.plen_mode >> 8, cd.plen_mode & 0xFF, Ln.L.plog2);
    DpNode d;
    d.succ = (uint32_t)(i - lo);
    d.nmain = it.nmain;
    d.npre = it.npre;
    d.flags = (it.list ? 1u : 0u) | (it.scan ? 2u : 0u) | (it.dict ? 4u : 0u);
    d.ent = it.ent;
    B.nodes[j] = d;
  }
}

// One CTA per column: k_dp_layout into the batch's frame table (dense, at the
// column's frame base; payload offsets absolute).  A column that fails, or
// whose frames need entropy areas (status 2: the single-column path decodes
// it), keeps its frame slots as empty RAW frames.
__global__ void __launch_bounds__(kChainThreads) k_dpb_layout(DpBatch B) {
  __shared__ uint64_t s_warp[33];
  const int c = blockIdx.x, tid = threadIdx.x;
  const DpBLane& Ln = B.lanes[c];
  DpBLaneOut& O = B.out[c];
  const uint64_t F = O.nmarked, fb = O.fbase;
  uint64_t lo = B.cnt[B.chunk0[c]];
  const uint64_t n_total = dpb_total(B, c);
  uint64_t carry_f = 0, carry_v = 0, carry_main = 0, carry_pre = 0, carry_list = 0, carry_ent = 0;
  bool scan = false, dict = false, stop = false, fail = O.status != 0;
  for (uint64_t t0 = 0; t0 < F && !stop && !fail; t0 += kChainThreads) {
    uint64_t j = t0 + tid;
    bool have = j < F;
    DpCand cd;
    cd.pos = 0;
    cd.n = 0;
    cd.plen_mode = 0;
    DpNode nd;
    memset(&nd, 0, sizeof(nd));
    if (have) {
      nd = B.nodes[lo + j];
      cd = B.cand[lo + nd.succ];
    }
    uint64_t vx = block_excl_scan<ScanSum>(have ? (uint64_t)cd.n : 0ull, s_warp, nullptr);
    uint64_t voff = carry_v + vx;
    bool keep = have && voff < n_total;
    bool list = keep && (nd.flags & 1);
    bool last = keep && voff + cd.n >= n_total;
    stop = __syncthreads_or(last) != 0;
    fail = (__syncthreads_or(last && voff + cd.n > n_total) != 0) || fail;
    uint64_t tf, tv, tp, tl, te;
    uint64_t fx = block_excl_scan<ScanSum>(keep ? 1ull : 0ull, s_warp, &tf);
    block_excl_scan<ScanSum>(keep ? (uint64_t)cd.n : 0ull, s_warp, &tv);
    uint64_t packed = keep ? ((uint64_t)nd.npre << 32 | nd.nmain) : 0ull;
    uint64_t px = block_excl_scan<ScanSum>(packed, s_warp, &tp);
    uint64_t lx = block_excl_scan<ScanSum>(list ? 1ull : 0ull, s_warp, &tl);
    uint64_t ex = block_excl_scan<ScanSum>(keep ? nd.ent : 0ull, s_warp, &te);
    if (keep) {
      uint64_t f = carry_f + fx;
      FrameDesc d;
      d.payload_off = (uint64_t)(uintptr_t)(Ln.s + cd.pos + 9);
      d.value_off = voff;
      d.n = cd.n;
      d.plen = cd.plen_mode >> 8;
      d.mode = cd.plen_mode & 0xFF;
      d.aux = 0;
      B.frames[fb + f] = d;
      B.frame_col[fb + f] = (uint32_t)c;
      B.ftmp[lo + f] = make_uint4((uint32_t)(carry_pre + (px >> 32)), nd.npre,
                                  (uint32_t)(carry_main + (px & 0xFFFFFFFFull)), nd.nmain);
      B.flist[lo + f] = list ? (uint32_t)(carry_list + lx) : kNone;
    }
    scan = (__syncthreads_or(keep && (nd.flags & 2)) != 0) || scan;
    dict = (__syncthreads_or(keep && (nd.flags & 4)) != 0) || dict;
    carry_f += tf;
    carry_v += tv;
    carry_main += tp & 0xFFFFFFFFull;
    carry_pre += tp >> 32;
    carry_list += tl;
    carry_ent += te;
  }
  uint32_t status = O.status;
  if (status == 0 && (fail || !stop || carry_v != n_total)) status = 1;
  if (status == 0 && carry_ent) status = 2;
  const uint64_t kept = status == 0 ? carry_f : 0;
  // the slots past the kept frames (all of them for a column left out) hold
  // empty frames
  for (uint64_t f = kept + tid; f < F; f += kChainThreads) {
    FrameDesc d;
    d.payload_off = (uint64_t)(uintptr_t)Ln.s;
    d.value_off = 0;
    d.n = 0;
    d.plen = 0;
    d.mode = M_RAW;
    d.aux = 0;
    B.frames[fb + f] = d;
    B.frame_col[fb + f] = (uint32_t)c;
    B.frame_pre[fb + f] = make_uint2(0, 0);
  }
  if (tid == 0) {
    O.status = status;
    O.nframes = (uint32_t)kept;
    O.nmain = status == 0 ? (uint32_t)carry_main : 0u;
    O.npre = status == 0 ? (uint32_t)carry_pre : 0u;
    O.nlist = status == 0 ? (uint32_t)carry_list : 0u;
    O.need_scan = scan;
    O.any_dict = dict;
    O.ent = carry_ent;
  }
}

// Item lists of the batch: one warp per kept chain frame.
__global__ void k_dpb_expand(DpBatch B) {
  uint64_t K = B.cnt[B.chunks];
  if (K > B.cap) return;
  uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  int l = threadIdx.x & 31;
  for (uint64_t j = warp; j < K; j += nwarps) {
    int c = (int)B.cand_lane[j];
    const DpBLaneOut& O = B.out[c];
    uint64_t lo = B.cnt[B.chunk0[c]], f = j - lo;
    if (O.status != 0 || f >= O.nframes) continue;
    uint64_t gf = O.fbase + f;
    uint4 t = B.ftmp[j];
    uint64_t pre0 = O.pre_base + t.x, main0 = O.main_base + t.z;
    if (l == 0) {
      B.frame_pre[gf] = make_uint2((uint32_t)pre0, t.y);
      uint32_t li = B.flist[j];
      if (li != kNone) B.list[O.list_base + li] = (uint32_t)gf;
    }
    for (uint32_t k = l; k < t.w; k += 32) B.main_items[main0 + k] = ItemRef{(uint32_t)gf, k};
    for (uint32_t k = l; k < t.y; k += 32) B.pre_items[pre0 + k] = ItemRef{(uint32_t)gf, k};
  }
}

std::atomic<unsigned long long> g_bmarks_attr{0};

}  // namespace

uint64_t dp_batch_slot_bytes(uint64_t chunks) { return chunks * kDpSlots * sizeof(DpCand); }

void launch_dp_batch_heads(const uint8_t* const* srcs, const uint64_t* lens, int n, DpHead* H, cudaStream_t st) {
  if (n <= 0) return;
  k_dpb_heads<<<(n + 127) / 128, 128, 0, st>>>(srcs, lens, n, H);
  count_launches(1);
}

void launch_dp_batch_read(const DpBatch& B, uint64_t* tile_tmp, cudaStream_t st) {
  once_per_device(g_bmarks_attr, [] {
    cudaFuncSetAttribute(k_dpb_marks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDpChainSmem);
  });
  unsigned gw = (unsigned)qmin((B.words + 255) / 256, 148ull * 8);
  if (gw == 0) gw = 1;
  if (B.nrle) k_dpb_rle_runs<<<B.nrle, kRleThreads, 0, st>>>(B);
  k_dpb_bitmap<<<gw, 256, 0, st>>>(B, B.word0);
  cudaMemsetAsync(B.ranks + B.words, 0, 8, st);
  launch_scan_sum(B.ranks, B.ranks, B.words + 1, tile_tmp, nullptr, st);
  k_dpb_lane_base<<<(B.nlanes + 127) / 128, 128, 0, st>>>(B);
  k_dpb_ranks<<<gw, 256, 0, st>>>(B, B.word0);
  k_dpb_select<<<gw, 256, 0, st>>>(B, B.word0);
  if (B.chunks) k_dpb_cand_scan<<<(unsigned)B.chunks, kDpThreads, 0, st>>>(B);
  cudaMemsetAsync(B.cnt + B.chunks, 0, 8, st);
  launch_scan_sum(B.cnt, B.cnt, B.chunks + 1, tile_tmp, nullptr, st);
  if (B.chunks) k_dpb_cand_compact<<<(unsigned)B.chunks, kDpThreads, 0, st>>>(B);
  unsigned gc = (unsigned)qmin((B.cap + 255) / 256, 148ull * 8);
  k_dpb_succ<<<gc, 256, 0, st>>>(B);
  k_dpb_marks<<<B.nlanes, kChainThreads, kDpChainSmem, st>>>(B);
  k_dpb_lane_scan<<<1, 1024, 0, st>>>(B, 0);
  k_dpb_items<<<gc, 256, 0, st>>>(B);
  k_dpb_layout<<<B.nlanes, kChainThreads, 0, st>>>(B);
  k_dpb_lane_scan<<<1, 1024, 0, st>>>(B, 1);
  k_dpb_expand<<<gc, 256, 0, st>>>(B);
  count_launches(14);
}
}  // namespace qb
