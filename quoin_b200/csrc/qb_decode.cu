// Block decoder (reference src/decoder.rs:145-190 and the per-codec decode
// functions).  Two kernels:
//  * k_walk_frames — one thread per frame: validates the frame's payload
//    structure in the reference's check order and records the byte offsets of
//    its FastLanes sub-blocks (the sub-block sizes are data-dependent, so this
//    is a short dependent walk; every frame walks concurrently);
//  * k_decode_frames — one CTA per frame, one warp per 1024-value sub-block:
//    coalesced unpack of the lane-transposed words, delta / RLE prefix sums
//    across sub-blocks, ALP / FLOAT_MULT reconstruction, exception patching,
//    and a byte-parallel LEB128 + prefix-XOR decoder for XORZ.
// Every payload read is bounded by the frame's plen; malformed frames set an
// error word instead of faulting.
#include "qb_common.cuh"
#include "qb_kernels.h"
#include "qb_layout.h"

namespace qb {

constexpr int kDecThreads = 256;
constexpr int kDecWarps = kDecThreads / 32;
constexpr int kMaxSubs = kMaxBlock / kSub;  // 128
constexpr int kDictSmem = 2048;
constexpr int kXorzChunk = kDecThreads * 8;  // payload bytes per XORZ step
constexpr int kXorzRing = 4096;              // decoded XORZ values awaiting their store

// Per-frame results of the walk (device memory, one per frame).
struct FrameAux {
  uint32_t err;
  uint32_t pad;
  uint64_t a, b, c, d;  // mode-specific scalars
  uint64_t dict8[8];    // ALP-RD dictionary
  uint32_t offs[2][kMaxSubs + 1];  // chain 0 / chain 1 sub-block header offsets (payload-relative)
};

// ---------------------------------------------------------------------------
// FoR sub-block chain (reference codecs/for_bitpack.rs:108-157), walked over
// p[pos .. bound): varint(n) then sub-blocks [width u8][min u64][128*width B].
// ---------------------------------------------------------------------------
__device__ uint32_t for_walk(const uint8_t* p, uint64_t bound, uint64_t pos, uint64_t n_values, uint32_t* offs) {
  uint64_t n64;
  uint32_t e = rd_varint(p, bound, &pos, &n64);
  if (e) return e;
  if (n64 != n_values) return E_CORRUPT;
  uint32_t nsub = (uint32_t)((n_values + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    if (pos >= bound) return E_TRUNCATED;
    uint32_t w = p[pos];
    if (w > 64) return E_CORRUPT;
    if (bound - pos - 1 < 8) return E_TRUNCATED;
    uint64_t need = 128ull * w;
    if (bound - pos - 9 < need) return E_TRUNCATED;
    offs[k] = (uint32_t)pos;
    pos += 9 + need;
  }
  offs[nsub] = (uint32_t)pos;
  return E_OK;
}

// ALP sub-block chain (reference codecs/alp.rs:168-248).
__device__ uint32_t alp_walk(const uint8_t* p, uint64_t plen, uint64_t n, uint32_t* offs) {
  uint64_t pos = 0, n64;
  uint32_t e = rd_varint(p, plen, &pos, &n64);
  if (e) return e;
  if (n64 != n) return E_CORRUPT;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    uint64_t count = qmin(kSub, n - (uint64_t)k * kSub);
    if (pos >= plen) return E_TRUNCATED;
    uint32_t ee = p[pos];
    if (pos + 1 >= plen) return E_TRUNCATED;
    uint32_t ff = p[pos + 1];
    if (ee > 18 || ff > ee) return E_CORRUPT;
    if (plen < pos + 4) return E_TRUNCATED;
    uint32_t exc = ld_u16(p + pos + 2);
    if (plen < pos + 12 || pos + 12 >= plen) return E_TRUNCATED;
    uint32_t w = p[pos + 12];
    if (w > 32) return E_CORRUPT;
    offs[k] = (uint32_t)pos;
    uint64_t q = pos + 13;
    if (plen - q < 128ull * w) return E_TRUNCATED;
    q += 128ull * w;
    for (uint32_t x = 0; x < exc; x++) {
      if (plen < q + 2 || plen < q + 10) return E_TRUNCATED;
      if (ld_u16(p + q) >= count) return E_CORRUPT;
      q += 10;
    }
    pos = q;
  }
  return E_OK;
}

// One thread per frame.
__global__ void k_walk_frames(const uint8_t* __restrict__ stream, const FrameDesc* __restrict__ frames, int nf,
                              int dtype, FrameAux* __restrict__ aux, unsigned long long* __restrict__ err) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  FrameDesc d = frames[f];
  const uint8_t* p = stream + d.payload_off;
  uint64_t plen = d.plen, n = d.n;
  FrameAux& A = aux[f];
  uint32_t e = E_OK;
  switch (d.mode) {
    case M_RAW:
      if (plen != n * lane_bytes(dtype)) e = E_CORRUPT;
      break;
    case M_CONST:
      if (plen != 8) e = E_CORRUPT;
      break;
    case M_STRIDE:
      if (plen != 16) e = E_CORRUPT;
      break;
    case M_XORZ:
      break;  // validated by the parallel decoder
    case M_FOR_BITPACK:
      e = for_walk(p, plen, 0, n, A.offs[0]);
      break;
    case M_DELTA_BITPACK:  // delta_bitpack.rs:48-64
      if (plen < 8) { e = E_TRUNCATED; break; }
      e = for_walk(p, plen, 8, n, A.offs[0]);
      break;
    case M_FLOAT_MULT: {  // float_mult.rs:100-133
      if (plen < 1 || plen < 2) { e = E_TRUNCATED; break; }
      uint32_t tag = p[0], si = p[1];
      if (si >= 7) { e = E_CORRUPT; break; }
      if (tag == 1) { e = E_UNSUPPORTED; break; }
      if (tag != 0) { e = E_CORRUPT; break; }
      A.a = si;
      e = for_walk(p, plen, 2, n, A.offs[0]);
      break;
    }
    case M_ALP:
      e = alp_walk(p, plen, n, A.offs[0]);
      break;
    case M_ALP_RD: {  // alp_rd.rs:208-285
      uint64_t pos = 0;
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t lbw = p[pos++];
      if (lbw < 1 || lbw > 63) { e = E_CORRUPT; break; }
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t dsz = p[pos++];
      if (dsz > 8) { e = E_CORRUPT; break; }
      for (uint32_t j = 0; j < dsz; j++) {
        if (plen < pos + 8) { e = E_TRUNCATED; break; }
        A.dict8[j] = ld_u64(p + pos);
        pos += 8;
      }
      if (e) break;
      uint64_t nexc;
      e = rd_varint(p, plen, &pos, &nexc);
      if (e) break;
      if (nexc > n) { e = E_CORRUPT; break; }
      uint64_t exc_start = pos;
      for (uint64_t x = 0; x < nexc && !e; x++) {
        uint64_t pp;
        e = rd_varint(p, plen, &pos, &pp);
        if (e) break;
        if (plen < pos + 8) { e = E_TRUNCATED; break; }
        pos += 8;
        if (pp >= n) e = E_CORRUPT;
      }
      if (e) break;
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t ctag = p[pos++];
      uint64_t clen;
      e = rd_varint(p, plen, &pos, &clen);
      if (e) break;
      if (clen > plen - pos) { e = E_TRUNCATED; break; }
      uint64_t cpos = pos;
      pos += clen;
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t rtag = p[pos++];
      uint64_t rpos = pos;
      if (ctag == 1) { e = E_UNSUPPORTED; break; }
      if (ctag != 0) { e = E_CORRUPT; break; }
      e = for_walk(p, cpos + clen, cpos, n, A.offs[0]);
      if (e) break;
      if (rtag == 1) { e = E_UNSUPPORTED; break; }
      if (rtag != 0) { e = E_CORRUPT; break; }
      e = for_walk(p, plen, rpos, n, A.offs[1]);
      A.a = lbw;
      A.b = dsz;
      A.c = exc_start;
      A.d = nexc;
      break;
    }
    case M_DICT: {  // dict.rs:154-207
      uint64_t pos = 0, card, vlen;
      e = rd_varint(p, plen, &pos, &card);
      if (e) break;
      if (card > n) { e = E_CORRUPT; break; }
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t vtag = p[pos++];
      e = rd_varint(p, plen, &pos, &vlen);
      if (e) break;
      if (vlen > plen - pos) { e = E_TRUNCATED; break; }
      uint64_t vpos = pos;
      if (vtag == 0) {
        if (vlen != card * 8) { e = E_CORRUPT; break; }
      } else if (vtag == 1) {
        if (vlen < 8) { e = E_TRUNCATED; break; }
        e = for_walk(p, vpos + vlen, vpos + 8, card, A.offs[1]);
        if (e) break;
      } else if (vtag == 2) {
        e = E_UNSUPPORTED;
        break;
      } else {
        e = E_CORRUPT;
        break;
      }
      pos += vlen;
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t ctag = p[pos++];
      if (ctag == 1) { e = E_UNSUPPORTED; break; }
      if (ctag != 0) { e = E_CORRUPT; break; }
      e = for_walk(p, plen, pos, n, A.offs[0]);
      A.a = card;
      A.b = vtag;
      A.c = vpos;
      break;
    }
    case M_RLE: {  // rle.rs:44-75
      uint64_t pos = 0, nr;
      e = rd_varint(p, plen, &pos, &nr);
      if (e) break;
      if (nr > n) { e = E_CORRUPT; break; }
      if (plen - pos < nr * 8) { e = E_TRUNCATED; break; }
      uint64_t vpos = pos;
      pos += nr * 8;
      e = for_walk(p, plen, pos, nr, A.offs[0]);
      A.a = nr;
      A.b = vpos;
      break;
    }
    default:
      e = E_UNSUPPORTED;
      break;
  }
  A.err = e;
  if (e) atomicMin(err, ((unsigned long long)f << 8) | e);
}

// ---------------------------------------------------------------------------
// Warp-level FastLanes unpack of one sub-block: calls f(i, min + residual) for
// every value index i < count.  For widths <= 32 lane l decodes FastLanes lane
// l (rows 0..31); above 32 lane l decodes 64-bit lane l % 16, rows 32*(l/16)
// .. +31.  Each row's words are consecutive across the warp.
// ---------------------------------------------------------------------------
template <class F>
__device__ inline void warp_unpack(const uint8_t* p, uint32_t off, uint32_t count, F f) {
  int l = threadIdx.x & 31;
  uint32_t w = p[off];
  uint64_t mn = ld_u64(p + off + 1);
  const uint8_t* words = p + off + 9;
  if (w == 0) {
    for (uint32_t i = l; i < count; i += 32) f(i, mn);
  } else if (w <= 32) {
    uint32_t mask = w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u);
#pragma unroll 8
    for (uint32_t r = 0; r < 32; r++) {
      uint32_t idx = r * 32 + l;
      uint32_t bit = r * w, word = bit >> 5, sh = bit & 31;
      uint32_t v = ld_u32(words + 4u * (word * 32u + l)) >> sh;
      if (sh + w > 32) v |= ld_u32(words + 4u * ((word + 1) * 32u + l)) << (32 - sh);
      v &= mask;
      if (idx < count) f(idx, mn + (uint64_t)v);
    }
  } else {
    uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1ull);
    uint32_t fl = l & 15, r0 = (l >> 4) * 32;
#pragma unroll 8
    for (uint32_t r = r0; r < r0 + 32; r++) {
      uint32_t idx = r * 16 + fl;
      uint32_t bit = r * w, word = bit >> 6, sh = bit & 63;
      uint64_t v = ld_u64(words + 8u * (word * 16u + fl)) >> sh;
      if (sh + w > 64) v |= ld_u64(words + 8u * ((word + 1) * 16u + fl)) << (64 - sh);
      v &= mask;
      if (idx < count) f(idx, mn + v);
    }
  }
}

// Warp inclusive prefix over buf[0..count) (u64, wrapping), starting from
// `carry`; writes via out(i, v).
template <class W>
__device__ inline void warp_prefix_smem(const uint64_t* buf, uint32_t count, uint64_t carry, W out) {
  int l = threadIdx.x & 31;
  uint64_t run = carry;
  for (uint32_t base = 0; base < count; base += 32) {
    uint32_t i = base + l;
    uint64_t v = i < count ? buf[i] : 0ull;
    uint64_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
      if (l >= o) inc += u;
    }
    if (i < count) out(i, run + inc);
    run += __shfl_sync(0xffffffffu, inc, 31);
  }
}

struct DecSmem {
  uint64_t subsum[kMaxSubs + 1];
  uint64_t subcarry[kMaxSubs + 1];
  uint32_t flag;
  uint32_t wcnt[kDecWarps];
  int64_t wmax[kDecWarps];
  uint64_t wxor[kDecWarps];
  uint64_t sc[4];
  unsigned long long nth;
  union {
    uint64_t wbuf[kDecWarps][kSub];  // per-warp sub-block staging (64 KB)
    struct {
      uint64_t dict[kDictSmem];      // dictionary values (16 KB)
      uint64_t stage[4][kSub];       // staging for the dictionary prefix pass
    } d;
    struct {
      uint64_t xbuf[kXorzChunk];     // XORZ chunk values (16 KB)
      uint64_t ring[kXorzRing];      // decoded values not yet stored (32 KB)
    } x;
  } u;
};

// ---------------------------------------------------------------------------
// Output stores.  Every decoded run of values [c0, c0 + cnt) (c0 = lane index
// of the first value) is written straight to its final place: the lane (u64),
// or the typed column, narrowed to the native width and scattered through the
// validity bitmap with nulls as 0 (reference lib.rs:492-506, validity.rs:130-146).
// With a bitmap, c0 is a multiple of 1024 and c0 + cnt is too, or the end of
// the lane; the run then owns the positions [sel(c0), sel(c0 + cnt)), where
// sel(c) is the position of the c-th valid value (0 for c = 0, n at the end),
// so the nulls between runs are written exactly once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void put_out(const DecodeOut& O, uint64_t pos, uint64_t v) {
  if (O.dtype == DT_I32 || O.dtype == DT_U32) {
    reinterpret_cast<uint32_t*>(O.out)[pos] = (uint32_t)v;
  } else if (O.dtype == DT_F32) {
    reinterpret_cast<uint32_t*>(O.out)[pos] = v ? f64bits_to_f32bits(v) : 0u;
  } else {
    reinterpret_cast<uint64_t*>(O.out)[pos] = v;
  }
}

__device__ __forceinline__ void run_positions(const DecodeOut& O, uint64_t c0, uint64_t c1, uint64_t* p0,
                                              uint64_t* p1) {
  *p0 = c0 == 0 ? 0 : O.sel[c0 >> 10];
  *p1 = c1 >= O.nvalid ? O.n : O.sel[c1 >> 10];
}

// Positions [32*w0, 32*w1) of the run [p0, p1) by one warp, relative ranks
// counted from `rel` (the number of the run's values before position 32*w0).
// The bitmap words are fetched 32 at a time, one per lane, and broadcast.
template <class V>
__device__ __forceinline__ void warp_store_words(const DecodeOut& O, uint64_t w0, uint64_t w1, uint64_t p0,
                                                 uint64_t p1, uint32_t rel, V& val) {
  int l = threadIdx.x & 31;
  uint32_t below = (1u << l) - 1u;
  for (uint64_t wb = w0; wb < w1; wb += 32) {
    uint32_t mine = wb + l < w1 ? O.bm32[wb + l] : 0u;
    uint32_t nw = (uint32_t)qmin(32, w1 - wb);
    for (uint32_t j = 0; j < nw; j++) {
      uint32_t bits = __shfl_sync(0xffffffffu, mine, j);
      uint64_t base = (wb + j) << 5;
      uint32_t in = 0xFFFFFFFFu;  // positions of this word inside [p0, p1)
      if (base < p0) in &= 0xFFFFFFFFu << (uint32_t)(p0 - base);
      if (base + 32 > p1) in &= 0xFFFFFFFFu >> (uint32_t)(base + 32 - p1);
      bits &= in;
      if ((in >> l) & 1u) {
        uint64_t v = 0;
        if ((bits >> l) & 1u) v = val(rel + __popc(bits & below));
        put_out(O, base + l, v);
      }
      rel += __popc(bits);
    }
  }
}

// One warp stores one run; val(q) is called with increasing q per lane.
template <class V>
__device__ void warp_store(const DecodeOut& O, uint64_t c0, uint32_t cnt, V val) {
  int l = threadIdx.x & 31;
  if (!O.bm32) {
    for (uint32_t q = l; q < cnt; q += 32) put_out(O, c0 + q, val(q));
    return;
  }
  uint64_t p0, p1;
  run_positions(O, c0, c0 + cnt, &p0, &p1);
  if (p1 > p0) warp_store_words(O, p0 >> 5, (p1 + 31) >> 5, p0, p1, 0u, val);
}

// All warps of the CTA store one run: warp w takes the w-th contiguous slice of
// the run's bitmap words and starts from the word's global rank.
template <class V>
__device__ void cta_store(const DecodeOut& O, uint64_t c0, uint32_t cnt, V val) {
  int warp = threadIdx.x >> 5;
  if (!O.bm32) {
    for (uint32_t q = threadIdx.x; q < cnt; q += kDecThreads) put_out(O, c0 + q, val(q));
    return;
  }
  uint64_t p0, p1;
  run_positions(O, c0, c0 + cnt, &p0, &p1);
  if (p1 <= p0) return;
  uint64_t wb = p0 >> 5, we = (p1 + 31) >> 5;
  uint64_t per = (we - wb + kDecWarps - 1) / kDecWarps;
  uint64_t w0 = wb + (uint64_t)warp * per, w1 = qmin(w0 + per, we);
  if (w0 >= w1) return;
  uint32_t rel = w0 == wb ? 0u : (uint32_t)(O.wrank[w0] - c0);
  warp_store_words(O, w0, w1, p0, p1, rel, val);
}

// Sum of one sub-block's values after a per-value map g (warp-uniform result).
template <class G>
__device__ inline uint64_t warp_sub_sum(const uint8_t* p, uint32_t off, uint32_t count, G g) {
  uint64_t s = 0;
  warp_unpack(p, off, count, [&](uint32_t, uint64_t v) { s += g(v); });
  return warp_sum(s);
}

// Two-phase prefix-sum decode of a FoR chain whose values are summed in index
// order (DeltaBitpack deltas, dictionary deltas): per-sub-block sums, a carry
// scan, then each warp stages its sub-block in smem, turns it into running
// values in place and hands it to done(k, buf, cnt).  `nstage` warps take part
// in the second phase (one staging buffer each).
template <class G, class D>
__device__ void chain_prefix(DecSmem& S, const uint8_t* p, const uint32_t* offs, uint64_t n, uint64_t base_carry,
                             uint64_t* stage, int nstage, G g, D done) {
  int l = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = warp; k < nsub; k += kDecWarps) {
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    uint64_t s = warp_sub_sum(p, offs[k], cnt, g);
    if (l == 0) S.subsum[k] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t c = base_carry;
    for (uint32_t k = 0; k < nsub; k++) {
      S.subcarry[k] = c;
      c += S.subsum[k];
    }
  }
  __syncthreads();
  if (warp < nstage) {
    uint64_t* buf = stage + (size_t)warp * kSub;
    for (uint32_t k = warp; k < nsub; k += nstage) {
      uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
      warp_unpack(p, offs[k], cnt, [&](uint32_t i, uint64_t v) { buf[i] = g(v); });
      __syncwarp();
      warp_prefix_smem(buf, cnt, S.subcarry[k], [&](uint32_t i, uint64_t v) { buf[i] = v; });
      __syncwarp();
      done(k, buf, cnt);
      __syncwarp();
    }
  }
  __syncthreads();
}

// XORZ (reference codecs/xorz.rs:18-32): LEB128 of v_i ^ v_{i-1}.  Byte-parallel:
// terminator bytes (bit 7 clear) end values; block scans number them and find
// each value's first byte, the terminator's thread assembles the value, and a
// block XOR-scan rebuilds v.  Values collect in a ring and leave it in runs of
// 1024 (the last run shorter).  Error kinds follow the sequential reader.
__device__ uint32_t dec_xorz(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, const DecodeOut& O,
                             uint64_t c0) {
  int t = threadIdx.x, l = t & 31, warp = t >> 5;
  if (n == 0) return plen ? E_CORRUPT : E_OK;
  uint64_t* ring = S.u.x.ring;
  uint64_t vbase = 0;         // values completed before this chunk
  uint64_t flushed = 0;       // values already stored
  uint64_t xcarry = 0;        // XOR of all values so far
  int64_t last_term = -1;     // position of the last terminator before the chunk
  bool saw_nth = false;
  uint64_t nth_pos = 0;
  if (t == 0) {
    S.flag = 0;
    S.nth = ~0ull;
  }
  __syncthreads();
  for (uint64_t base = 0; base < plen && vbase < n; base += kXorzChunk) {
    uint64_t b0 = base + (uint64_t)t * 8;
    uint32_t tm = 0;  // terminator mask of this thread's 8 bytes
#pragma unroll
    for (int j = 0; j < 8; j++)
      if (b0 + j < plen && !(p[b0 + j] & 0x80)) tm |= 1u << j;
    uint32_t cnt = __popc(tm);
    int64_t mylast = tm ? (int64_t)(b0 + 31 - __clz(tm)) : -1;
    uint32_t inc = cnt;
    int64_t mx = mylast;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
      int64_t um = __shfl_up_sync(0xffffffffu, mx, o);
      if (l >= o) {
        inc += u;
        mx = um > mx ? um : mx;
      }
    }
    if (l == 31) {
      S.wcnt[warp] = inc;
      S.wmax[warp] = mx;
    }
    __syncthreads();
    uint32_t woff = 0, total = 0;
    int64_t wprev = last_term, chunk_last = last_term;
    for (int w2 = 0; w2 < kDecWarps; w2++) {
      if (w2 < warp) {
        woff += S.wcnt[w2];
        wprev = S.wmax[w2] > wprev ? S.wmax[w2] : wprev;
      }
      total += S.wcnt[w2];
      chunk_last = S.wmax[w2] > chunk_last ? S.wmax[w2] : chunk_last;
    }
    int64_t mx_ex = __shfl_up_sync(0xffffffffu, mx, 1);
    if (l == 0) mx_ex = -1;
    int64_t prev = mx_ex > wprev ? mx_ex : wprev;  // last terminator before this thread's bytes
    uint32_t k = woff + inc - cnt;
    uint32_t m = tm;
    while (m) {
      int j = __ffs(m) - 1;
      m &= m - 1;
      uint64_t pos = b0 + j;
      uint64_t start = (uint64_t)(prev + 1);
      uint64_t len = pos - start + 1;
      uint64_t vi = vbase + k;
      if (vi < n) {
        if (len > 10) {
          S.flag = 1;
        } else {
          uint64_t x = 0;
          for (uint64_t q = 0; q < len; q++) x |= (uint64_t)(p[start + q] & 0x7f) << (7 * q);
          S.u.x.xbuf[k] = x;
        }
        if (vi == n - 1) {
          saw_nth = true;
          nth_pos = pos;
        }
      }
      prev = (int64_t)pos;
      k++;
    }
    __syncthreads();
    uint32_t cv = (uint32_t)qmin(total, n - vbase);
    uint32_t i0 = (uint32_t)t * 8;
    uint64_t vals[8], xs = 0;
    for (int j = 0; j < 8; j++) {
      vals[j] = (i0 + j < cv) ? S.u.x.xbuf[i0 + j] : 0ull;
      xs ^= vals[j];
    }
    uint64_t xi = xs;
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, xi, o);
      if (l >= o) xi ^= u;
    }
    if (l == 31) S.wxor[warp] = xi;
    __syncthreads();
    uint64_t wx = 0, tx = 0;
    for (int w2 = 0; w2 < kDecWarps; w2++) {
      if (w2 < warp) wx ^= S.wxor[w2];
      tx ^= S.wxor[w2];
    }
    uint64_t run = xcarry ^ wx ^ xi ^ xs;
    for (int j = 0; j < 8; j++) {
      run ^= vals[j];
      if (i0 + j < cv) ring[(vbase + i0 + j) & (kXorzRing - 1)] = run;
    }
    xcarry ^= tx;
    vbase += total;
    last_term = chunk_last;
    __syncthreads();
    uint64_t have = qmin(vbase, n);
    bool stored = false;
    while (flushed + kSub <= have) {  // at most 3071 values wait in the ring
      uint64_t f0 = flushed;
      cta_store(O, c0 + f0, kSub, [&](uint32_t q) { return ring[(f0 + q) & (kXorzRing - 1)]; });
      flushed += kSub;
      stored = true;
    }
    if (stored) __syncthreads();
  }
  if (flushed < qmin(vbase, n)) {
    uint64_t f0 = flushed;
    cta_store(O, c0 + f0, (uint32_t)(qmin(vbase, n) - f0), [&](uint32_t q) { return ring[(f0 + q) & (kXorzRing - 1)]; });
  }
  if (saw_nth) atomicMin(&S.nth, (unsigned long long)nth_pos);
  __syncthreads();
  uint32_t e = E_OK;
  if (S.flag) e = E_CORRUPT;
  else if (vbase < n) e = (plen - (uint64_t)(last_term + 1) >= 10) ? E_CORRUPT : E_TRUNCATED;
  else if (S.nth != plen - 1) e = E_CORRUPT;
  __syncthreads();
  return e;
}

// ---------------------------------------------------------------------------
// The decode kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kDecThreads) k_decode_frames(const uint8_t* __restrict__ stream,
                                                              const FrameDesc* __restrict__ frames, int nf,
                                                              int dtype, const FrameAux* __restrict__ aux,
                                                              DecodeOut O, uint64_t* __restrict__ scratch,
                                                              unsigned long long* __restrict__ err) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  DecSmem& S = *reinterpret_cast<DecSmem*>(smem_raw);
  int f = blockIdx.x;
  if (f >= nf) return;
  const FrameAux& A = aux[f];
  if (A.err) return;
  FrameDesc d = frames[f];
  const uint8_t* p = stream + d.payload_off;
  uint64_t plen = d.plen, n = d.n;
  uint64_t c0 = d.value_off;
  int t = threadIdx.x, l = t & 31, warp = t >> 5;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  uint64_t* stg = &S.u.wbuf[warp][0];
  uint32_t e = E_OK;
  if (t == 0) S.flag = 0;
  __syncthreads();
  switch (d.mode) {
    case M_RAW: {
      uint32_t lb = lane_bytes(dtype);
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        const uint8_t* q0 = p + (uint64_t)k * kSub * lb;
        if (dtype == DT_F32) {
          warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return f32bits_to_f64bits(ld_u32(q0 + 4 * q)); });
        } else if (lb == 4) {
          warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return (uint64_t)ld_u32(q0 + 4 * q); });
        } else {
          warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return ld_u64(q0 + 8 * q); });
        }
      }
      break;
    }
    case M_CONST: {
      uint64_t v = ld_u64(p);
      for (uint32_t k = warp; k < nsub; k += kDecWarps)
        warp_store(O, c0 + (uint64_t)k * kSub, (uint32_t)qmin(kSub, n - (uint64_t)k * kSub), [&](uint32_t) { return v; });
      break;
    }
    case M_STRIDE: {
      uint64_t first = ld_u64(p), stride = ld_u64(p + 8);
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint64_t i0 = (uint64_t)k * kSub;
        warp_store(O, c0 + i0, (uint32_t)qmin(kSub, n - i0), [&](uint32_t q) { return first + (i0 + q) * stride; });
      }
      break;
    }
    case M_XORZ:
      e = dec_xorz(S, p, plen, n, O, c0);
      break;
    case M_FOR_BITPACK:
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t v) { stg[i] = v; });
        __syncwarp();
        warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return stg[q]; });
        __syncwarp();
      }
      break;
    case M_DELTA_BITPACK:
      chain_prefix(S, p, A.offs[0], n, ld_u64(p), &S.u.wbuf[0][0], kDecWarps,
                   [](uint64_t v) { return unzigzag64(v); },
                   [&](uint32_t k, const uint64_t* buf, uint32_t cnt) {
                     warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return buf[q]; });
                   });
      break;
    case M_FLOAT_MULT: {
      double scale = kFmScales[A.a];
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t v) {
          stg[i] = f64_bits(__ddiv_rn(__ll2double_rn((long long)v), scale));
        });
        __syncwarp();
        warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return stg[q]; });
        __syncwarp();
      }
      break;
    }
    case M_ALP:
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t off = A.offs[0][k];
        int ee = p[off], ff = p[off + 1];
        uint32_t exc = ld_u16(p + off + 2);
        int64_t mn = (int64_t)ld_u64(p + off + 4);
        uint32_t w = p[off + 12];
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        const uint8_t* words = p + off + 13;
        if (w == 0) {
          uint64_t v = f64_bits(alp_decode_value(mn, ee, ff));
          for (uint32_t i = l; i < cnt; i += 32) stg[i] = v;
        } else {
          uint32_t mask = w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u);
          for (uint32_t r = 0; r < 32; r++) {
            uint32_t idx = r * 32 + l;
            uint32_t bit = r * w, word = bit >> 5, sh = bit & 31;
            uint32_t v = ld_u32(words + 4u * (word * 32u + l)) >> sh;
            if (sh + w > 32) v |= ld_u32(words + 4u * ((word + 1) * 32u + l)) << (32 - sh);
            v &= mask;
            if (idx < cnt) stg[idx] = f64_bits(alp_decode_value((int64_t)((uint64_t)mn + v), ee, ff));
          }
        }
        __syncwarp();
        if (exc && l == 0) {  // in order, so a repeated position keeps the last exception
          const uint8_t* xp = words + 128u * w;
          for (uint32_t x = 0; x < exc; x++) stg[ld_u16(xp + 10 * x)] = ld_u64(xp + 10 * x + 2);
        }
        __syncwarp();
        warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return stg[q]; });
        __syncwarp();
      }
      break;
    case M_ALP_RD: {
      uint32_t lbw = (uint32_t)A.a, dsz = (uint32_t)A.b, rbw = 64 - lbw;
      // With exceptions the values are assembled in the frame's scratch range
      // first (the exception list is one sequential stream over the frame).
      uint64_t* fo = A.d ? scratch + d.value_off : nullptr;
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t v) { stg[i] = v; });
        __syncwarp();
        uint64_t* o = fo ? fo + (size_t)k * kSub : stg;
        warp_unpack(p, A.offs[1][k], cnt, [&](uint32_t i, uint64_t r) {
          uint64_t c = stg[i];
          if (c >= dsz) S.flag = 1;
          else o[i] = (A.dict8[c] << rbw) | r;
        });
        __syncwarp();
        if (!fo) warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return stg[q]; });
        __syncwarp();
      }
      __syncthreads();
      if (S.flag) {
        e = E_CORRUPT;
        break;
      }
      if (fo) {
        if (t == 0) {  // exceptions in order (alp_rd.rs:281-283)
          uint64_t pos = A.c, rmask = (1ull << rbw) - 1ull;
          for (uint64_t x = 0; x < A.d; x++) {
            uint64_t pp = 0;
            rd_varint(p, plen, &pos, &pp);
            uint64_t lv = ld_u64(p + pos);
            pos += 8;
            fo[pp] = (lv << rbw) | (fo[pp] & rmask);
          }
        }
        __syncthreads();
        cta_store(O, c0, (uint32_t)n, [&](uint32_t q) { return fo[q]; });
      }
      break;
    }
    case M_DICT: {
      uint64_t card = A.a;
      const uint8_t* vb = p + A.c;
      const uint64_t* dict = nullptr;
      if (A.b == 1) {  // delta-coded sorted dictionary -> smem or scratch
        // scratch holds one u64 per lane value; a frame's dictionary (card <= n)
        // uses the frame's own range
        uint64_t* dd = card <= kDictSmem ? S.u.d.dict : (scratch ? scratch + d.value_off : nullptr);
        if (!dd) {
          e = E_UNSUPPORTED;
          break;
        }
        chain_prefix(S, p, A.offs[1], card, ld_u64(vb), &S.u.d.stage[0][0], 4,
                     [](uint64_t v) { return unzigzag64(v); },
                     [&](uint32_t k, const uint64_t* buf, uint32_t cnt) {
                       for (uint32_t q = l; q < cnt; q += 32) dd[(uint64_t)k * kSub + q] = buf[q];
                     });
        dict = dd;
      } else if (card <= kDictSmem) {
        for (uint64_t i = t; i < card; i += kDecThreads) S.u.d.dict[i] = ld_u64(vb + 8 * i);
        __syncthreads();
        dict = S.u.d.dict;
      }
      // codes -> values, per warp and sub-block: with the dictionary in smem the
      // codes are staged as u16 beside it, else the values in the warp's buffer
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        if (dict == S.u.d.dict) {
          uint16_t* cb = reinterpret_cast<uint16_t*>(&S.u.d.stage[0][0]) + (size_t)warp * kSub;
          warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t c) {
            if (c >= card) {
              S.flag = 1;
              c = 0;
            }
            cb[i] = (uint16_t)c;
          });
          __syncwarp();
          warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return dict[cb[q]]; });
        } else {
          warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t c) {
            if (c >= card) S.flag = 1;
            else stg[i] = dict ? dict[c] : ld_u64(vb + 8 * c);
          });
          __syncwarp();
          warp_store(O, c0 + (uint64_t)k * kSub, cnt, [&](uint32_t q) { return stg[q]; });
        }
        __syncwarp();
      }
      __syncthreads();
      if (S.flag) e = E_CORRUPT;
      break;
    }
    case M_RLE: {
      uint64_t nr = A.a;
      const uint8_t* rv = p + A.b;
      uint32_t nrs = (uint32_t)((nr + kSub - 1) / kSub);
      // phase 1: run-length sums per chunk (saturating at n+1 to catch overruns)
      for (uint32_t k = warp; k < nrs; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, nr - (uint64_t)k * kSub);
        uint64_t s = 0;
        warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t, uint64_t v) { s = qmin(s + qmin(v, n + 1), n + 1); });
        for (int o = 16; o; o >>= 1) s = qmin(s + __shfl_xor_sync(0xffffffffu, s, o), n + 1);
        if (l == 0) S.subsum[k] = s;
      }
      __syncthreads();
      if (t == 0) {
        uint64_t c = 0;
        uint32_t bad = 0;
        for (uint32_t k = 0; k < nrs; k++) {
          S.subcarry[k] = c;
          c += S.subsum[k];
          if (c > n) bad = 1;
        }
        S.sc[0] = bad ? 1ull : (c != n ? 2ull : 0ull);
      }
      __syncthreads();
      if (S.sc[0] == 1) { e = E_CORRUPT; break; }
      if (S.sc[0] == 2) { e = E_LENGTH_MISMATCH; break; }
      if (!scratch) { e = E_UNSUPPORTED; break; }
      // phase 2: run ends (u32, the frame's scratch range) ...
      uint32_t* ends = reinterpret_cast<uint32_t*>(scratch + d.value_off);
      for (uint32_t k = warp; k < nrs; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, nr - (uint64_t)k * kSub);
        warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t v) { stg[i] = v; });
        __syncwarp();
        warp_prefix_smem(stg, cnt, S.subcarry[k], [&](uint32_t i, uint64_t v) { ends[(uint64_t)k * kSub + i] = (uint32_t)v; });
        __syncwarp();
      }
      __syncthreads();
      // ... phase 3: each warp expands whole output sub-blocks from a cursor
      // found by binary search over the run ends
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t lo = k * kSub, cnt = (uint32_t)qmin(kSub, n - lo);
        uint32_t a = 0, b = (uint32_t)nr;
        while (a < b) {
          uint32_t mid = (a + b) >> 1;
          if (ends[mid] > lo) b = mid; else a = mid + 1;
        }
        uint32_t cur = a;
        warp_store(O, c0 + lo, cnt, [&](uint32_t q) {
          uint32_t i = lo + q;
          while (ends[cur] <= i) cur++;
          return ld_u64(rv + 8ull * cur);
        });
      }
      break;
    }
    default:
      e = E_UNSUPPORTED;
      break;
  }
  if (e && t == 0) atomicMin(err, ((unsigned long long)f << 8) | e);
}

// ---------------------------------------------------------------------------
// Validity ranks and the final typed write.
// ---------------------------------------------------------------------------

// popcount of each 32-bit word of a bitmap of n bits (bytes beyond n ignored).
__global__ void k_word_popcount(const uint8_t* __restrict__ bm, uint64_t n, uint64_t* __restrict__ cnt) {
  uint64_t nw = (n + 31) / 32;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    uint64_t b0 = w * 4, nbytes = (n + 7) / 8;
    for (int k = 0; k < 4; k++)
      if (b0 + k < nbytes) bits |= (uint32_t)bm[b0 + k] << (8 * k);
    uint64_t rem = n - w * 32;
    if (rem < 32) bits &= (1u << rem) - 1u;
    cnt[w] = (uint64_t)__popc(bits);
  }
}

// sel[m] = position of the (1024*m)-th valid value: the owner of every 1024th
// rank is the one bitmap word whose rank range contains it.
__global__ void k_select_table(const uint8_t* __restrict__ bm, uint64_t n, const uint64_t* __restrict__ word_rank,
                               uint64_t nvalid, uint64_t* __restrict__ sel) {
  uint64_t nw = (n + 31) / 32, nbytes = (n + 7) / 8;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    for (int k = 0; k < 4; k++)
      if (w * 4 + k < nbytes) bits |= (uint32_t)bm[w * 4 + k] << (8 * k);
    uint64_t rem = n - w * 32;
    if (rem < 32) bits &= (1u << rem) - 1u;
    uint64_t r = word_rank[w], c = (uint64_t)__popc(bits);
    uint64_t m = (r + kSub - 1) / kSub * kSub;
    if (m < r + c && m < nvalid) {
      for (uint64_t k = m - r; k; k--) bits &= bits - 1u;  // drop the lower set bits
      sel[m / kSub] = w * 32 + (uint64_t)(__ffs(bits) - 1);
    }
  }
}

// Scatter the compacted lane through the validity bitmap (null -> 0) and
// narrow to the dtype's native width (reference lib.rs:492-506,
// validity.rs:130-146).  Warp w handles bitmap words; lane l position l.
__global__ void k_finalize(const uint64_t* __restrict__ lane, const uint8_t* __restrict__ bm,
                           const uint64_t* __restrict__ word_rank, uint64_t n, int dtype, void* __restrict__ out) {
  uint64_t nw = (n + 31) / 32, nbytes = (n + 7) / 8;
  int l = threadIdx.x & 31;
  uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = warp; w < nw; w += nwarps) {
    uint64_t i = w * 32 + l;
    uint64_t v = 0;
    if (bm) {
      uint32_t byte = (w * 4 + (l >> 3) < nbytes) ? bm[w * 4 + (l >> 3)] : 0u;
      uint32_t bits = 0;
      for (int k = 0; k < 4; k++) bits |= __shfl_sync(0xffffffffu, byte, k * 8) << (8 * k);
      if (i < n && ((bits >> l) & 1u)) v = lane[word_rank[w] + __popc(bits & ((1u << l) - 1u))];
    } else if (i < n) {
      v = lane[i];
    }
    if (i >= n) continue;
    if (dtype == DT_I32 || dtype == DT_U32) {
      reinterpret_cast<uint32_t*>(out)[i] = (uint32_t)v;
    } else if (dtype == DT_F32) {
      reinterpret_cast<uint32_t*>(out)[i] = v ? f64bits_to_f32bits(v) : 0u;
    } else {
      reinterpret_cast<uint64_t*>(out)[i] = v;
    }
  }
}

// Decimal recombine (reference decimal.rs:218-246, 379-408): value = vmin +
// (limb0 | limb1 << 64 | ...) with carries, scattered through the bitmap.
__global__ void k_decimal_combine(const uint64_t* __restrict__ limbs, uint64_t limb_stride, int nlimbs,
                                  const uint64_t* __restrict__ vmin, const uint8_t* __restrict__ bm,
                                  const uint64_t* __restrict__ word_rank, uint64_t n, uint8_t* __restrict__ out) {
  uint64_t nw = (n + 31) / 32, nbytes = (n + 7) / 8;
  int l = threadIdx.x & 31;
  uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint64_t vm[4];
  for (int k = 0; k < 4; k++) vm[k] = k < nlimbs ? vmin[k] : 0;
  for (uint64_t w = warp; w < nw; w += nwarps) {
    uint64_t i = w * 32 + l;
    bool valid = i < n;
    uint64_t j = i;
    if (bm) {
      uint32_t byte = (w * 4 + (l >> 3) < nbytes) ? bm[w * 4 + (l >> 3)] : 0u;
      uint32_t bits = 0;
      for (int k = 0; k < 4; k++) bits |= __shfl_sync(0xffffffffu, byte, k * 8) << (8 * k);
      valid = valid && ((bits >> l) & 1u);
      j = word_rank[w] + __popc(bits & ((1u << l) - 1u));
    }
    if (i >= n) continue;
    uint64_t* o = reinterpret_cast<uint64_t*>(out + i * 8ull * nlimbs);
    uint64_t carry = 0;
    for (int k = 0; k < nlimbs; k++) {
      uint64_t r = 0;
      if (valid) {
        uint64_t a = vm[k], b = limbs[k * limb_stride + j];
        uint64_t s = a + b;
        uint64_t c1 = s < a;
        r = s + carry;
        carry = c1 | (r < s);
      }
      o[k] = r;
    }
  }
}

// ---------------------------------------------------------------------------
// Host launchers.
// ---------------------------------------------------------------------------
uint64_t decode_aux_bytes(int nf) { return (uint64_t)(nf > 0 ? nf : 1) * sizeof(FrameAux); }

void launch_decode_frames(const uint8_t* stream, const FrameDesc* frames, int nf, int dtype, const DecodeOut& out,
                          uint64_t* scratch, void* aux, unsigned long long* err, cudaStream_t st) {
  if (nf <= 0) return;
  FrameAux* A = reinterpret_cast<FrameAux*>(aux);
  k_walk_frames<<<(nf + 127) / 128, 128, 0, st>>>(stream, frames, nf, dtype, A, err);
  cudaFuncSetAttribute(k_decode_frames, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DecSmem));
  k_decode_frames<<<nf, kDecThreads, sizeof(DecSmem), st>>>(stream, frames, nf, dtype, A, out, scratch, err);
  count_launches(2);
}

void launch_select_table(const uint8_t* bm, uint64_t n, const uint64_t* word_rank, uint64_t nvalid, uint64_t* sel,
                         cudaStream_t st) {
  uint64_t nw = (n + 31) / 32;
  if (nw == 0) return;
  unsigned g = (unsigned)qmin((nw + 255) / 256, 148ull * 16);
  k_select_table<<<g, 256, 0, st>>>(bm, n, word_rank, nvalid, sel);
  count_launches(1);
}

void launch_word_popcount(const uint8_t* bm, uint64_t n, uint64_t* cnt, cudaStream_t st) {
  uint64_t nw = (n + 31) / 32;
  unsigned g = (unsigned)qmin((nw + 255) / 256, 148ull * 16);
  if (g == 0) g = 1;
  k_word_popcount<<<g, 256, 0, st>>>(bm, n, cnt);
  count_launches(1);
}

void launch_finalize(const uint64_t* lane, const uint8_t* bm, const uint64_t* word_rank, uint64_t n, int dtype,
                     void* out, cudaStream_t st) {
  uint64_t nw = (n + 31) / 32;
  unsigned g = (unsigned)qmin((nw + 7) / 8, 148ull * 32);
  if (g == 0) g = 1;
  k_finalize<<<g, 256, 0, st>>>(lane, bm, word_rank, n, dtype, out);
  count_launches(1);
}

void launch_decimal_combine(const uint64_t* limbs, uint64_t limb_stride, int nlimbs, const uint64_t* vmin,
                            const uint8_t* bm, const uint64_t* word_rank, uint64_t n, uint8_t* out,
                            cudaStream_t st) {
  uint64_t nw = (n + 31) / 32;
  unsigned g = (unsigned)qmin((nw + 7) / 8, 148ull * 32);
  if (g == 0) g = 1;
  k_decimal_combine<<<g, 256, 0, st>>>(limbs, limb_stride, nlimbs, vmin, bm, word_rank, n, out);
  count_launches(1);
}

}  // namespace qb
