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
constexpr uint64_t kSelStep = 512;           // select-table granularity (valid values)

// Per-frame results of the walk (device memory, one per frame).
struct FrameAux {
  uint32_t err;
  uint32_t ent;         // 1: an entropy-coded part is decoded by the frame kernel
  uint64_t a, b, c, d;  // mode-specific scalars
  uint64_t e0, e1, e2;  // entropy-coded parts: payload positions
  uint32_t t0, t1;      // and their tags
  uint32_t defer;       // 1: an ALP-RD exception list left to the frame kernel's walk
  uint32_t pad_;
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

// ALP-RD payload after the exception list (alp_rd.rs:208-285): codes tag,
// varint(codes_len), codes, rights tag, rights.  Bit-packed parts get their
// FoR sub-block offsets; an entropy-coded part (tag 1) leaves the rest to the
// frame kernel's entropy path.
__device__ uint32_t alprd_walk_tail(const uint8_t* p, uint64_t plen, uint64_t n, uint64_t pos, FrameAux& A) {
  if (pos >= plen) return E_TRUNCATED;
  uint32_t ctag = p[pos++];
  uint64_t clen;
  uint32_t e = rd_varint(p, plen, &pos, &clen);
  if (e) return e;
  if (clen > plen - pos) return E_TRUNCATED;
  uint64_t cpos = pos;
  pos += clen;
  if (pos >= plen) return E_TRUNCATED;
  uint32_t rtag = p[pos++];
  A.e0 = cpos;
  A.e1 = clen;
  A.e2 = pos;
  A.t0 = ctag;
  A.t1 = rtag;
  if (ctag == 1) {  // codes entropy-coded: the frame kernel decodes the rest in order
    A.ent = 1;
    return E_OK;
  }
  if (ctag != 0) return E_CORRUPT;
  e = for_walk(p, cpos + clen, cpos, n, A.offs[0]);
  if (e) return e;
  if (rtag == 1) {  // rights entropy-coded (bit-packed rights bytes)
    A.ent = 1;
    return E_OK;
  }
  if (rtag != 0) return E_CORRUPT;
  return for_walk(p, plen, pos, n, A.offs[1]);
}

// One thread per frame.
__global__ void k_walk_frames(const uint8_t* __restrict__ stream, const FrameDesc* __restrict__ frames, int nf,
                              int dtype, FrameAux* __restrict__ aux, unsigned long long* __restrict__ err,
                              BatchView bv) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  FrameDesc d = frames[f];
  if (bv.cols) dtype = bv.cols[bv.frame_col[f]].dtype;
  const uint8_t* p = stream + d.payload_off;
  uint64_t plen = d.plen, n = d.n;
  FrameAux& A = aux[f];
  A.ent = 0;
  A.defer = 0;
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
    case M_BYTE_TRANSPOSE:  // transpose.rs:10-32: the whole payload is entropy-coded
    case M_ORDERED_DELTA:   // linear.rs: entropy-coded residual bytes (decoder.rs:162-171)
    case M_DELTA2:
    case M_DELTA_DP:
    case M_PRED:            // pred.rs: a predictor table in the frame's area (decoder.rs:150-157)
    case M_PRED_RC:
    case M_PRED2:
    case M_LZ:              // lz.rs: entropy-coded LZ tokens (decoder.rs:172-175)
      A.ent = 1;
      break;
    case M_FLOAT_MULT: {  // float_mult.rs:100-133
      if (plen < 1 || plen < 2) { e = E_TRUNCATED; break; }
      uint32_t tag = p[0], si = p[1];
      if (si >= 7) { e = E_CORRUPT; break; }
      if (tag == 1) {  // FM_ENTROPY: rANS over LEB128 zigzag deltas of k
        A.a = si;
        A.ent = 1;
        break;
      }
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
      A.a = lbw;
      A.b = dsz;
      A.c = pos;
      A.d = nexc;
      if (nexc) {  // the list and the rest of the walk: alprd_list_walk + alprd_walk_tail in the frame kernel
        A.defer = 1;
        break;
      }
      e = alprd_walk_tail(p, plen, n, pos, A);
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
      } else if (vtag == 2) {  // TRANSPOSE values: the frame kernel decodes the rest in order
        A.a = card;
        A.b = vtag;
        A.c = vpos;
        A.d = vlen;
        A.ent = 1;
        break;
      } else {
        e = E_CORRUPT;
        break;
      }
      pos += vlen;
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t ctag = p[pos++];
      A.a = card;
      A.b = vtag;
      A.c = vpos;
      A.d = vlen;
      if (ctag == 1) {  // CODES_ENTROPY byte planes
        A.e0 = pos;
        A.ent = 1;
        break;
      }
      if (ctag != 0) { e = E_CORRUPT; break; }
      e = for_walk(p, plen, pos, n, A.offs[0]);
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

// One value of a FastLanes sub-block (the same layout as warp_unpack): value
// index i sits in lane i % 32, row i / 32 for widths <= 32, and in 64-bit lane
// i % 16, row i / 16 above.
__device__ inline uint64_t for_value_at(const uint8_t* p, uint32_t off, uint32_t i) {
  uint32_t w = p[off];
  uint64_t mn = ld_u64(p + off + 1);
  const uint8_t* words = p + off + 9;
  if (w == 0) return mn;
  if (w <= 32) {
    uint32_t l = i & 31, r = i >> 5, bit = r * w, word = bit >> 5, sh = bit & 31;
    uint32_t v = ld_u32(words + 4u * (word * 32u + l)) >> sh;
    if (sh + w > 32) v |= ld_u32(words + 4u * ((word + 1) * 32u + l)) << (32 - sh);
    return mn + (uint64_t)(v & (w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u)));
  }
  uint32_t fl = i & 15, r = i >> 4, bit = r * w, word = bit >> 6, sh = bit & 63;
  uint64_t v = ld_u64(words + 8u * (word * 16u + fl)) >> sh;
  if (sh + w > 64) v |= ld_u64(words + 8u * ((word + 1) * 16u + fl)) << (64 - sh);
  return mn + (v & (w == 64 ? ~0ull : ((1ull << w) - 1ull)));
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
  uint16_t* rcm;                     // range-coder model (256 x 256) of the frame, in its entropy area
  uint8_t* lzs;                      // the LZ cascade's scratch (ent_lz_cap bytes), in the same area
  uint64_t lzs_cap;
  uint32_t eoffs[kMaxSubs + 1];      // FoR chain sub-block offsets found by the frame kernel
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
    struct {                         // rANS tables (rans.rs:110-175)
      uint32_t freq[256];
      uint32_t cum[257];
      uint8_t sym[4096];
      uint64_t sc[4];
    } r;
  } u;
};

// ---------------------------------------------------------------------------
// Output stores.  Every decoded run of values [c0, c0 + cnt) (c0 = lane index
// of the first value) is written straight to its final place: the lane (u64),
// or the typed column, narrowed to the native width and scattered through the
// validity bitmap with nulls as 0 (reference lib.rs:492-506, validity.rs:130-146).
// With a bitmap the run owns the positions [sel(c0), sel(c0 + cnt)), where
// sel(c) is the position of the c-th valid value (0 for c = 0, n at the end),
// so the nulls between runs are written exactly once.  Every lane of the
// warp takes part (run_positions is warp-cooperative).
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

// Position of the k-th set bit of x (k < popcount(x)): halving by popcounts.
__device__ __forceinline__ uint32_t select_in_word(uint32_t x, uint32_t k) {
  uint32_t pos = 0, c = __popc(x & 0xFFFFu);
  if (k >= c) { k -= c; pos += 16; x >>= 16; }
  c = __popc(x & 0xFFu);
  if (k >= c) { k -= c; pos += 8; x >>= 8; }
  c = __popc(x & 0xFu);
  if (k >= c) { k -= c; pos += 4; x >>= 4; }
  c = __popc(x & 0x3u);
  if (k >= c) { k -= c; pos += 2; x >>= 2; }
  return pos + ((k >= (x & 1u)) ? 1u : 0u);
}

// Position of the c-th valid value (c < nvalid): from the 512-granular table,
// the owning bitmap word is found 32 words at a time.
__device__ uint64_t warp_select(const DecodeOut& O, uint64_t c) {
  if (!O.bm32) return c;
  if (c >= O.nvalid) return O.n;
  uint64_t s = O.sel[c >> 9];
  if ((c & 511) == 0) return s;
  int l = threadIdx.x & 31;
  uint64_t nw = (O.n + 31) >> 5;
  uint32_t tail = (uint32_t)(O.n & 31);
  for (uint64_t w0 = s >> 5; w0 < nw; w0 += 32) {
    uint64_t w = w0 + l;
    uint32_t bits = 0;
    uint64_t r = 0;
    bool hit = false;
    if (w < nw) {
      bits = O.bm32[w];
      if (w == nw - 1 && tail) bits &= (1u << tail) - 1u;
      r = O.wrank[w];
      hit = r <= c && c < r + (uint64_t)__popc(bits);
    }
    uint32_t m = __ballot_sync(0xffffffffu, hit);
    if (m) {
      int src = __ffs(m) - 1;
      bits = __shfl_sync(0xffffffffu, bits, src);
      r = __shfl_sync(0xffffffffu, r, src);
      return ((w0 + (uint64_t)src) << 5) + (uint64_t)select_in_word(bits, (uint32_t)(c - r));
    }
  }
  return O.n;
}

__device__ __forceinline__ void run_positions(const DecodeOut& O, uint64_t c0, uint64_t c1, uint64_t* p0,
                                              uint64_t* p1) {
  *p0 = c0 == 0 ? 0 : warp_select(O, c0);
  *p1 = c1 >= O.nvalid ? O.n : warp_select(O, c1);
}

// Output element writers: 0 = u64 lane value, 1 = low 32 bits (i32 / u32),
// 2 = f64 bits narrowed to f32 (nulls stay 0).
template <int KIND>
__device__ __forceinline__ void put_kind(void* base, uint64_t i, uint64_t v) {
  if (KIND == 0) reinterpret_cast<uint64_t*>(base)[i] = v;
  else if (KIND == 1) reinterpret_cast<uint32_t*>(base)[i] = (uint32_t)v;
  else reinterpret_cast<uint32_t*>(base)[i] = v ? f64bits_to_f32bits(v) : 0u;
}
__device__ __forceinline__ int out_kind(int dtype) {
  return (dtype == DT_I32 || dtype == DT_U32) ? 1 : dtype == DT_F32 ? 2 : 0;
}

// Positions [32*w0, 32*w1) of the run [p0, p1) by one warp, relative ranks
// counted from `rel` (the number of the run's values before position 32*w0).
// The bitmap words are fetched 32 at a time, one per lane, and broadcast; the
// lanes of a word write 32 consecutive positions.
template <int KIND, class V>
__device__ __forceinline__ void store_words_k(const DecodeOut& O, uint64_t w0, uint64_t nwords, uint32_t first_in,
                                              uint32_t last_in, uint32_t rel, V& val) {
  int l = threadIdx.x & 31;
  uint32_t below = (1u << l) - 1u;
  uint8_t* ow = reinterpret_cast<uint8_t*>(O.out) + (w0 << 5) * (KIND == 0 ? 8u : 4u);
  const uint32_t* bw = O.bm32 + w0;
  for (uint64_t wb = 0; wb < nwords; wb += 32) {
    uint32_t mine = wb + l < nwords ? bw[wb + l] : 0u;
    uint32_t nw = (uint32_t)qmin(32, nwords - wb);
    for (uint32_t j = 0; j < nw; j++) {
      uint32_t in = (wb + j == 0 ? first_in : 0xFFFFFFFFu) & (wb + j + 1 == nwords ? last_in : 0xFFFFFFFFu);
      uint32_t bits = __shfl_sync(0xffffffffu, mine, j) & in;
      if ((in >> l) & 1u) {
        uint64_t v = 0;
        if ((bits >> l) & 1u) v = val(rel + __popc(bits & below));
        put_kind<KIND>(ow, (uint64_t)l, v);
      }
      rel += __popc(bits);
      ow += 32u * (KIND == 0 ? 8u : 4u);
    }
  }
}

template <class V>
__device__ __forceinline__ void warp_store_words(const DecodeOut& O, uint64_t w0, uint64_t w1, uint64_t p0,
                                                 uint64_t p1, uint32_t rel, V& val) {
  uint64_t lo = w0 << 5, hi = w1 << 5;
  uint32_t first_in = p0 > lo ? (0xFFFFFFFFu << (uint32_t)(p0 - lo)) : 0xFFFFFFFFu;
  uint32_t last_in = p1 < hi ? (0xFFFFFFFFu >> (uint32_t)(hi - p1)) : 0xFFFFFFFFu;
  switch (out_kind(O.dtype)) {
    case 1: store_words_k<1>(O, w0, w1 - w0, first_in, last_in, rel, val); break;
    case 2: store_words_k<2>(O, w0, w1 - w0, first_in, last_in, rel, val); break;
    default: store_words_k<0>(O, w0, w1 - w0, first_in, last_in, rel, val); break;
  }
}

// Lanes store values c0 .. c0+cnt-1 of a run without a bitmap.
template <class V>
__device__ __forceinline__ void warp_store_dense(const DecodeOut& O, uint64_t c0, uint32_t cnt, V& val) {
  int l = threadIdx.x & 31;
  switch (out_kind(O.dtype)) {
    case 1:
      for (uint32_t q = l; q < cnt; q += 32) put_kind<1>(O.out, c0 + q, val(q));
      break;
    case 2:
      for (uint32_t q = l; q < cnt; q += 32) put_kind<2>(O.out, c0 + q, val(q));
      break;
    default:
      for (uint32_t q = l; q < cnt; q += 32) put_kind<0>(O.out, c0 + q, val(q));
      break;
  }
}

// One warp stores one run; val(q) is called with increasing q per lane.
template <class V>
__device__ void warp_store(const DecodeOut& O, uint64_t c0, uint32_t cnt, V val) {
  if (!O.bm32) {
    warp_store_dense(O, c0, cnt, val);
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

// A whole frame's values f(0 .. n-1), typically reads of a global buffer,
// stored by the CTA one 1024-value sub-block per warp: the warp reads its
// sub-block into its staging buffer (eight reads in flight per lane) and
// stores it as one run.  Uses the per-warp staging area.
template <class F>
__device__ void cta_store_staged(DecSmem& S, const DecodeOut& O, uint64_t c0, uint32_t n, F f) {
  int l = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t* stg = &S.u.wbuf[warp][0];
  uint32_t nsub = (n + kSub - 1) / kSub;
  __syncthreads();  // the staging area is free
  for (uint32_t k = warp; k < nsub; k += kDecWarps) {
    uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
    for (uint32_t j0 = 0; j0 < 32; j0 += 8) {
      uint64_t r[8];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        uint32_t i = (j0 + j) * 32 + l;
        r[j] = i < cnt ? f(base + i) : 0ull;
      }
#pragma unroll
      for (int j = 0; j < 8; j++) stg[(j0 + j) * 32 + l] = r[j];
    }
    __syncwarp();
    warp_store(O, c0 + base, cnt, [&](uint32_t q) { return stg[q]; });
    __syncwarp();
  }
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
// ALP-RD exception lists (alp_rd.rs:208-285): nexc records of (varint
// position, u64 left part).  Records have variable length, so the start of
// each depends on the previous one's varint.  The list is staged through
// shared memory (at most 16 KB, and at most 18 bytes per remaining record, a
// round) with a bitmap of its varint terminator bytes (high bit clear); the
// CTA computes, for every staged offset, where a record starting there would
// end (the first terminator within 10 bytes, then 8 bytes), and one thread
// follows the chain through that table: one shared load per record.  The
// records of a round are then decoded, checked and applied by the whole CTA.
// ---------------------------------------------------------------------------
constexpr uint32_t kExcStage = 16384;  // staged list bytes per round
constexpr uint32_t kExcRecs = 2048;    // records per round (a stage holds at most 16384 / 9 + 1)
constexpr uint32_t kExcWords = (kExcStage + 32) / 32 + 7;  // 520: two words past the last staged byte
constexpr uint16_t kNxBadVarint = 0xFFFF, kNxShort = 0xFFFE;

struct ExcStage {
  uint8_t* bytes;   // bytes[j] = the byte at the 16-byte aligned address below the round's position + j
  uint16_t* nx;     // nx[j]: stage offset after a record starting at j, or kNxBadVarint / kNxShort
  uint32_t* epos;   // record positions (over nx, once the chain has been followed)
  uint64_t* left;   // record left parts (likewise)
  uint32_t* term;   // terminator bitmap over the stage (bit j: byte j staged, high bit clear)
  uint16_t* start;  // record starts (stage offsets)
};

// Carves the stage out of the per-warp staging area (64 KB): 16 KB + 32 of
// bytes, the next-record table (its space reused for positions and left
// parts), 520 bitmap words and the starts (55 KB).
__device__ inline ExcStage exc_stage(DecSmem& S) {
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(&S.u.wbuf[0][0]) + 15) & ~(uintptr_t)15);
  ExcStage X;
  X.bytes = base;
  X.nx = reinterpret_cast<uint16_t*>(base + kExcStage + 32);
  X.left = reinterpret_cast<uint64_t*>(X.nx);
  X.epos = reinterpret_cast<uint32_t*>(X.left + kExcRecs);
  X.term = reinterpret_cast<uint32_t*>(X.nx + kExcStage + 32);
  X.start = reinterpret_cast<uint16_t*>(X.term + kExcWords);
  return X;
}
static_assert(8 * kExcRecs + 4 * kExcRecs <= 2 * (kExcStage + 32), "positions and left parts fit the table");
static_assert(3 * (kExcStage + 32) + 4 * kExcWords + 2 * kExcRecs + 15 <= sizeof(uint64_t) * kDecWarps * kSub,
              "exception stage fits the per-warp staging area");

// The 4 bytes at byte offset o of a 4-byte aligned shared buffer (o + 8 within it).
__device__ inline uint32_t lds_u32(const uint8_t* b, uint32_t o) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(b);
  return __funnelshift_r(w[o >> 2], w[(o >> 2) + 1], (o & 3) * 8);
}

// Bits of the 10 bytes from stage offset o in the terminator bitmap.
__device__ inline uint32_t term10(const uint32_t* term, uint32_t o) {
  uint64_t win = ((uint64_t)term[o >> 5] | ((uint64_t)term[(o >> 5) + 1] << 32)) >> (o & 31);
  return (uint32_t)win & 0x3FFu;
}

// Payload bytes [pos, send) into the stage by the whole CTA (16-byte loads for
// the aligned middle, bytes at the edges; nothing outside the range is read),
// the terminator bitmap and the next-record table (bounded by plen as the
// record reads are).  Returns the stage offset of byte pos.
__device__ uint32_t stage_list(const ExcStage& X, const uint8_t* p, uint64_t pos, uint64_t send, uint64_t plen) {
  uintptr_t g0 = reinterpret_cast<uintptr_t>(p + pos), g1 = reinterpret_cast<uintptr_t>(p + send);
  uintptr_t a0 = g0 & ~(uintptr_t)15, c0 = (g0 + 15) & ~(uintptr_t)15, a1 = g1 & ~(uintptr_t)15;
  uint32_t head = (uint32_t)(g0 - a0), end = head + (uint32_t)(send - pos);
  for (uintptr_t c = c0 + 16u * threadIdx.x; c < a1; c += 16u * blockDim.x)
    *reinterpret_cast<uint4*>(X.bytes + (c - a0)) = __ldg(reinterpret_cast<const uint4*>(c));
  uintptr_t e0 = c0 < g1 ? c0 : g1, t0 = a1 > c0 ? a1 : c0;
  for (uintptr_t c = g0 + threadIdx.x; c < e0; c += blockDim.x) X.bytes[c - a0] = *reinterpret_cast<const uint8_t*>(c);
  for (uintptr_t c = t0 + threadIdx.x; c < g1; c += blockDim.x) X.bytes[c - a0] = *reinterpret_cast<const uint8_t*>(c);
  __syncthreads();
  for (uint32_t w = threadIdx.x; w < kExcWords; w += blockDim.x) {
    uint32_t bits = 0;
    uint32_t j0 = 32 * w;
    if (j0 < end && j0 + 32 > head) {
      const uint32_t* q = reinterpret_cast<const uint32_t*>(X.bytes + j0);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        uint32_t m = ~q[i] & 0x80808080u;
        bits |= (((m >> 7) & 1u) | ((m >> 14) & 2u) | ((m >> 21) & 4u) | ((m >> 28) & 8u)) << (4 * i);
      }
      if (head > j0) bits &= ~0u << (head - j0);
      if (end < j0 + 32) bits &= (1u << (end - j0)) - 1u;
    }
    X.term[w] = bits;
  }
  __syncthreads();
  for (uint32_t j = head + threadIdx.x; j < end; j += blockDim.x) {
    uint32_t m10 = term10(X.term, j);
    uint16_t v = kNxBadVarint;
    if (m10) {
      uint32_t vl = (uint32_t)__ffs(m10);
      v = plen - (pos + (j - head) + vl) < 8 ? kNxShort : (uint16_t)(j + vl + 8);
    }
    X.nx[j] = v;
  }
  __syncthreads();
  return head;
}

__device__ __forceinline__ uint32_t lds_u16(const uint16_t* p) {
  uint16_t v;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"((uint32_t)__cvta_generic_to_shared(p)));
  return v;
}
__device__ __forceinline__ void sts_u16(uint16_t* p, uint32_t v) {
  asm volatile("st.shared.u16 [%0], %1;" ::"r"((uint32_t)__cvta_generic_to_shared(p)), "h"((uint16_t)v));
}

// Thread 0: the chain of records from stage offset `head` (list position
// gpos) while records remain (at most kExcRecs) and each is wholly staged (its
// start + 18 within the stage, or the stage reaching plen).  Fills X.start;
// stops at the first record whose varint runs past 10 bytes (E_CORRUPT, as
// rd_varint) or past plen, or whose 8-byte left part does not fit
// (E_TRUNCATED).  Returns the records found; *err and *next describe the stop.
__device__ __forceinline__ uint32_t exc_chain(const ExcStage& X, uint32_t head, uint32_t end, uint64_t gpos,
                                              uint64_t plen, bool staged_to_plen, uint64_t want, uint32_t* err,
                                              uint64_t* next) {
  uint32_t k = 0, e = E_OK, o = head;
  uint32_t lim = (uint32_t)qmin(want, (uint64_t)kExcRecs);
  uint32_t last = staged_to_plen ? end : (end >= 18 ? end - 18 : 0);  // records may start at o <= last
  while (k < lim && o <= last) {
    if (!staged_to_plen || o < end) {
      uint32_t nxt = lds_u16(X.nx + o);
      if (nxt < kNxShort) {
        sts_u16(X.start + k, o);
        k++;
        o = nxt;
        continue;
      }
      e = nxt == kNxShort ? E_TRUNCATED : (plen - (gpos + (o - head)) >= 10 ? E_CORRUPT : E_TRUNCATED);
    } else {
      e = E_TRUNCATED;  // the list runs past plen
    }
    break;
  }
  *err = e;
  *next = gpos + (o - head);
  return k;
}

// Record r of the stage: its position and left part (rd_varint's value).
__device__ inline void exc_decode(const ExcStage& X, uint32_t r, uint64_t* pp, uint64_t* lv) {
  uint32_t o = X.start[r];
  uint32_t vl = (uint32_t)__ffs(term10(X.term, o));
  uint64_t v = 0;
  for (uint32_t i = 0; i < vl; i++) v |= (uint64_t)(X.bytes[o + i] & 0x7Fu) << (7 * i);
  *pp = v;
  *lv = (uint64_t)lds_u32(X.bytes, o + vl) | ((uint64_t)lds_u32(X.bytes, o + vl + 4) << 32);
}

// The frame walk's pass over an exception list (alp_rd.rs:230-245): in list
// order, each record's varint (rd_varint's errors), its 8 bytes (E_TRUNCATED),
// then position < n (E_CORRUPT); the first failing record decides.  All
// threads call it.  Returns the error and sets *end past the list.
__device__ uint32_t alprd_list_walk(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t pos,
                                    uint64_t nexc, uint64_t* end) {
  ExcStage X = exc_stage(S);
  uint64_t x = 0;
  uint32_t e = E_OK;
  while (x < nexc) {
    uint64_t send = pos + qmin(qmin((uint64_t)kExcStage, plen - pos), 18 * (nexc - x));
    __syncthreads();  // the previous round's reads are done
    uint32_t head = stage_list(X, p, pos, send, plen);
    if (threadIdx.x == 0) {
      uint32_t ee;
      uint64_t q;
      uint32_t k = exc_chain(X, head, head + (uint32_t)(send - pos), pos, plen, send == plen, nexc - x, &ee, &q);
      S.sc[0] = q;
      S.sc[1] = k;
      S.flag = ee;
    }
    __syncthreads();
    uint32_t k = (uint32_t)S.sc[1];
    bool bad = false;
    for (uint32_t r = threadIdx.x; r < k; r += blockDim.x) {
      uint64_t pp, lv;
      exc_decode(X, r, &pp, &lv);
      bad |= pp >= n;
    }
    if (__syncthreads_or(bad)) {  // a record before any structural stop
      e = E_CORRUPT;
      break;
    }
    pos = S.sc[0];
    x += k;
    e = S.flag;
    if (e || k == 0) break;  // k == 0 without an error is not reached: a stage holds a record
  }
  *end = pos;
  return e;
}

// ALP-RD exceptions (alp_rd.rs:281-283): vals[p] = (left << rbw) | rights[p]
// for each record, in list order.  A round whose positions strictly increase
// (every list the encoder writes) is applied by the whole CTA, whose random
// reads of the rights overlap; otherwise thread 0 applies it in order, so a
// repeated position keeps its last record.  The list was validated by
// alprd_list_walk (positions < n, no truncation).
__device__ void alprd_exceptions(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t pos, uint64_t nexc,
                                 const uint8_t* rsrc, const uint32_t* roffs, uint32_t rbw, uint64_t* vals) {
  ExcStage X = exc_stage(S);
  int t = threadIdx.x;
  uint64_t x = 0;
  while (x < nexc) {
    uint64_t send = pos + qmin(qmin((uint64_t)kExcStage, plen - pos), 18 * (nexc - x));
    __syncthreads();  // every thread has left the staging area (and read S.flag)
    uint32_t head = stage_list(X, p, pos, send, plen);
    if (t == 0) {
      uint32_t ee;
      uint64_t q;
      uint32_t k = exc_chain(X, head, head + (uint32_t)(send - pos), pos, plen, send == plen, nexc - x, &ee, &q);
      S.sc[0] = q;
      S.sc[1] = k;
    }
    __syncthreads();
    uint32_t k = (uint32_t)S.sc[1];
    uint64_t q = S.sc[0];
    for (uint32_t r = t; r < k; r += blockDim.x) {
      uint64_t pp, lv;
      exc_decode(X, r, &pp, &lv);
      X.epos[r] = (uint32_t)pp;
      X.left[r] = lv;
    }
    __syncthreads();
    bool dis = false;
    for (uint32_t r = t + 1; r < k; r += blockDim.x) dis |= X.epos[r] <= X.epos[r - 1];
    bool inc = !__syncthreads_or(dis);
    auto apply = [&](uint32_t r) {
      uint32_t pp = X.epos[r];
      vals[pp] = (X.left[r] << rbw) | for_value_at(rsrc, roffs[pp / kSub], pp % kSub);
    };
    if (inc) {
      for (uint32_t r = t; r < k; r += blockDim.x) apply(r);
    } else if (t == 0) {
      for (uint32_t r = 0; r < k; r++) apply(r);
    }
    if (k == 0) break;  // not reached for a walked list
    x += k;
    pos = q;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Entropy-coded parts (Balanced and above): the 4-state rANS blocks of
// rans.rs:110-175 behind the entropy tag of entropy/mod.rs:152-178.
// ---------------------------------------------------------------------------

// One rANS block decoded by the CTA: thread 0 reads the header and runs the
// decoder (four states share one byte stream, so it is sequential); all
// threads build the slot -> symbol table.  Writes the first min(len, cap)
// symbols to out and the decoded length to *len_out.  Error kinds and their
// order follow rans.rs.
__device__ __noinline__ uint32_t rans_decode_cta(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t max_len, uint8_t* out,
                                   uint64_t cap, uint64_t* len_out) {
  int t = threadIdx.x;
  for (int i = t; i < 256; i += blockDim.x) S.u.r.freq[i] = 0;
  for (int i = t; i < 4096; i += blockDim.x) S.u.r.sym[i] = 0;
  __syncthreads();
  if (t == 0) {
    uint32_t e = E_OK;
    uint64_t pos = 0, n64 = 0, ns = 0;
    do {
      e = rd_varint(p, plen, &pos, &n64);
      if (e) break;
      if (n64 > max_len) { e = E_CORRUPT; break; }
      e = rd_varint(p, plen, &pos, &ns);
      if (e) break;
      if (ns == 0 || ns > 256) { e = E_CORRUPT; break; }
      uint32_t sum = 0;
      for (uint64_t k = 0; k < ns; k++) {
        if (pos >= plen) { e = E_TRUNCATED; break; }
        uint32_t sy = p[pos++];
        uint64_t f64v;
        e = rd_varint(p, plen, &pos, &f64v);
        if (e) break;
        uint32_t f = (uint32_t)f64v;  // the reference reads the frequency as a u32 (`as u32`)
        if (f == 0 || f > 4096) { e = E_CORRUPT; break; }
        S.u.r.freq[sy] = f;
        sum += f;
      }
      if (e) break;
      if (sum != 4096) { e = E_CORRUPT; break; }
      uint32_t c = 0;
      for (int sy = 0; sy < 256; sy++) {
        S.u.r.cum[sy] = c;
        c += S.u.r.freq[sy];
      }
      S.u.r.cum[256] = c;
    } while (false);
    S.u.r.sc[0] = e;
    S.u.r.sc[1] = pos;
    S.u.r.sc[2] = n64;
  }
  __syncthreads();
  uint32_t e = (uint32_t)S.u.r.sc[0];
  if (e) {
    *len_out = 0;
    __syncthreads();
    return e;
  }
  for (int sy = t; sy < 256; sy += blockDim.x)
    for (uint32_t slot = S.u.r.cum[sy]; slot < S.u.r.cum[sy + 1] && slot < 4096; slot++) S.u.r.sym[slot] = (uint8_t)sy;
  __syncthreads();
  if (t == 0) {
    uint64_t pos = S.u.r.sc[1], n64 = S.u.r.sc[2];
    uint32_t x[4] = {0, 0, 0, 0};
    uint32_t ee = E_OK;
    for (int k = 0; k < 4 && !ee; k++) {
      if (plen < pos + 4) {
        ee = E_TRUNCATED;
      } else {
        x[k] = ld_u32(p + pos);
        pos += 4;
      }
    }
    for (uint64_t i = 0; i < n64 && !ee; i++) {
      uint32_t idx = (uint32_t)(i & 3), xi = x[idx], slot = xi & 4095u;
      uint32_t sy = S.u.r.sym[slot];
      if (i < cap) out[i] = (uint8_t)sy;
      uint32_t xn = S.u.r.freq[sy] * (xi >> 12) + slot - S.u.r.cum[sy];
      while (xn < (1u << 23)) {
        if (pos >= plen) {
          ee = E_TRUNCATED;
          break;
        }
        xn = (xn << 8) | p[pos++];
      }
      x[idx] = xn;
    }
    S.u.r.sc[0] = ee;
  }
  __syncthreads();
  e = (uint32_t)S.u.r.sc[0];
  *len_out = S.u.r.sc[2];
  __syncthreads();
  return e;
}

// entropy/mod.rs:152-178: a tag byte, then rANS (the range coder, legacy tANS
// and the LZ cascade tags are outside the pool).
// Thread 0 computes a status, every thread gets it.
__device__ __forceinline__ uint32_t cta_bcast(DecSmem& S, uint32_t v) {
  if (threadIdx.x == 0) S.sc[3] = v;
  __syncthreads();
  uint32_t r = (uint32_t)S.sc[3];
  __syncthreads();
  return r;
}

// The range coder (rc.rs:86-225): an LZMA-style binary decoder, 11-bit
// probabilities adapted by shift 5, under an order-1 byte model (the previous
// byte picks one of 256 bit trees of 256 nodes).  The bits are one dependent
// chain, so thread 0 decodes; the CTA resets the 128 KB model (in the frame's
// entropy area) first.  Reads past the end give 0, as in the reference, so
// only the declared length can fail (E_CORRUPT above max_len).  Every
// renormalisation loop ends: a probability stays in [1, 2047], so after a
// bit the range is at least 2^13 and two byte shifts bring it back above 2^24.
__device__ __noinline__ uint32_t rc_decode_cta(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t max_len,
                                               uint8_t* out, uint64_t cap, uint64_t* len_out) {
  uint16_t* probs = S.rcm;
  if (!probs) return E_NO_ENTROPY_AREA;
  for (uint32_t i = threadIdx.x; i < 65536u; i += blockDim.x) probs[i] = 1024;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t pos = 0, len = 0;
    uint32_t e = rd_varint(p, plen, &pos, &len);
    if (!e && (len > max_len || len > cap)) e = E_CORRUPT;
    if (!e) {
      const uint8_t* in = p + pos;
      uint64_t inlen = plen - pos, ip = 0;
      auto next = [&]() -> uint32_t {
        uint32_t b = ip < inlen ? in[ip] : 0u;
        ip++;
        return b;
      };
      uint32_t code = 0, range = 0xFFFFFFFFu;
      next();  // the encoder's leading cache byte
      for (int k = 0; k < 4; k++) code = (code << 8) | next();
      uint32_t ctx = 0;
      for (uint64_t i = 0; i < len; i++) {
        uint16_t* pr = probs + ctx * 256;
        uint32_t node = 1;
        for (int k = 0; k < 8; k++) {
          uint32_t pv = pr[node];
          uint32_t bound = (range >> 11) * pv;
          if (code >= bound) {
            code -= bound;
            range -= bound;
            pr[node] = (uint16_t)(pv - (pv >> 5));
            node = (node << 1) | 1u;
          } else {
            range = bound;
            pr[node] = (uint16_t)(pv + ((2048u - pv) >> 5));
            node <<= 1;
          }
          while (range < (1u << 24)) {
            range <<= 8;
            code = (code << 8) | next();
          }
        }
        uint8_t b = (uint8_t)(node & 0xFF);
        out[i] = b;
        ctx = b;
      }
    }
    S.sc[2] = e ? 0 : len;
    S.flag = e;
  }
  __syncthreads();
  uint32_t e = S.flag;
  *len_out = S.sc[2];
  __syncthreads();
  return e;
}

// tANS (tans.rs:193-283, entropy tag 1, still decoded by the reference):
// varint(len) ++ u8(distinct - 1) ++ symbols ++ u16 LE weights (each >= 1,
// symbols distinct, sum 1024) ++ u32 LE state in [1024, 2048) ++ MSB-first
// renormalisation bits (reads past the end give 0).  Symbol s of weight w
// takes w of the 1,024 table slots, visited with the odd stride 615; the k-th
// slot of s continues from x = w + k and reads the bits that bring x << bits
// into [1024, 2048).  A legacy tag, so thread 0 builds the table (in the
// frame's range-coder model area) and decodes; every loop is bounded by 1024
// or by the declared length.
__device__ __noinline__ uint32_t tans_decode_cta(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t max_len,
                                                 uint8_t* out, uint64_t cap, uint64_t* len_out) {
  if (!S.rcm) return E_NO_ENTROPY_AREA;
  if (threadIdx.x == 0) {
    uint32_t* node = reinterpret_cast<uint32_t*>(S.rcm);  // base | bits << 16 | symbol << 24
    uint8_t* table = reinterpret_cast<uint8_t*>(node + 1024);
    uint32_t* x = reinterpret_cast<uint32_t*>(table + 1024);  // per symbol
    uint64_t pos = 0, len = 0;
    uint32_t e = rd_varint(p, plen, &pos, &len);
    if (!e && (len > max_len || len > cap)) e = E_CORRUPT;
    uint32_t num = 0, state = 0;
    uint64_t syms = 0, wts = 0;
    if (!e) {
      if (pos >= plen) e = E_TRUNCATED;
      else num = p[pos++] + 1u;
    }
    if (!e) {
      if (plen - pos < num) e = E_TRUNCATED;
      syms = pos;
      pos += num;
    }
    if (!e) {
      if (plen - pos < 2ull * num) e = E_TRUNCATED;
      wts = pos;
      pos += 2ull * num;
    }
    if (!e) {
      if (plen - pos < 4) e = E_TRUNCATED;
      else state = ld_u32(p + pos);
      pos += 4;
    }
    if (!e && (state < 1024u || state >= 2048u)) e = E_CORRUPT;
    if (!e) {
      uint32_t seen[8] = {0, 0, 0, 0, 0, 0, 0, 0}, wsum = 0;
      for (uint32_t s = 0; s < num && !e; s++) {
        uint32_t sym = p[syms + s], w = p[wts + 2 * s] | ((uint32_t)p[wts + 2 * s + 1] << 8);
        if (w == 0 || ((seen[sym >> 5] >> (sym & 31)) & 1u)) e = E_CORRUPT;
        seen[sym >> 5] |= 1u << (sym & 31);
        wsum += w;
      }
      if (!e && wsum != 1024u) e = E_CORRUPT;
    }
    if (!e) {
      uint32_t step = 0;
      for (uint32_t s = 0; s < num; s++) {
        uint32_t sym = p[syms + s], w = p[wts + 2 * s] | ((uint32_t)p[wts + 2 * s + 1] << 8);
        x[sym] = w;
        for (uint32_t k = 0; k < w; k++, step++) table[(615u * step) & 1023u] = (uint8_t)sym;
      }
      for (uint32_t i = 0; i < 1024u; i++) {
        uint32_t sym = table[i], b = x[sym]++;
        uint32_t bits = (uint32_t)(__clz(b) - __clz(1024u));
        node[i] = ((b << bits) - 1024u) | (bits << 16) | (sym << 24);
      }
      const uint8_t* in = p + pos;
      uint64_t inlen = plen - pos, ip = 0, acc = 0;
      uint32_t have = 0;
      for (uint64_t k = 0; k < len; k++) {
        uint32_t nd = node[state - 1024u];
        uint32_t bits = (nd >> 16) & 0xFFu, extra = 0;
        if (bits) {
          while (have < bits) {
            acc = (acc << 8) | (ip < inlen ? in[ip] : 0u);
            ip++;
            have += 8;
          }
          have -= bits;
          extra = (uint32_t)(acc >> have) & ((1u << bits) - 1u);
          acc &= (1ull << have) - 1ull;
        }
        out[k] = (uint8_t)(nd >> 24);
        state = 1024u + (nd & 0xFFFFu) + extra;  // < 2048 for a table built from valid weights
      }
    }
    S.sc[2] = e ? 0 : len;
    S.flag = e;
  }
  __syncthreads();
  uint32_t e = S.flag;
  *len_out = S.sc[2];
  __syncthreads();
  return e;
}

// LZ tokens (lz.rs:119-155): varint(length) (== expected, else E_CORRUPT),
// then groups of a control byte (8 flags, MSB first) and 8 tokens: a match
// (varint offset, varint length - 4; overlapping copies allowed) or a
// literal.  Thread 0; every loop is bounded by the expected length.
__device__ uint32_t lz_decode(const uint8_t* p, uint64_t len, uint64_t expected, uint8_t* out, uint64_t cap) {
  uint64_t pos = 0, n = 0, o = 0;
  uint32_t e = rd_varint(p, len, &pos, &n);
  if (e) return e;
  if (n != expected || n > cap) return E_CORRUPT;
  while (o < n) {
    if (pos >= len) return E_TRUNCATED;
    uint32_t ctrl = p[pos++];
    for (int k = 0; k < 8 && o < n; k++) {
      if ((ctrl >> (7 - k)) & 1u) {
        uint64_t off, ml;
        if ((e = rd_varint(p, len, &pos, &off))) return e;
        if ((e = rd_varint(p, len, &pos, &ml))) return e;
        ml += 4;
        if (off == 0 || off > o) return E_CORRUPT;
        if (ml > n - o) return E_CORRUPT;  // o + ml > n, without wrapping (o <= n)
        for (uint64_t j = 0; j < ml; j++, o++) out[o] = out[o - off];
      } else {
        if (pos >= len) return E_TRUNCATED;
        out[o++] = p[pos++];
      }
    }
  }
  return E_OK;
}

// entropy/mod.rs:152-163: tag 2 rANS, tag 0 the range coder, tag 1 tANS.
__device__ uint32_t entropy_only_cta(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t max_len, uint8_t* out,
                                     uint64_t cap, uint64_t* len_out) {
  *len_out = 0;
  if (plen == 0) return E_TRUNCATED;
  uint32_t tag = p[0];
  if (tag == 2) return rans_decode_cta(S, p + 1, plen - 1, max_len, out, cap, len_out);
  if (tag == 0) return rc_decode_cta(S, p + 1, plen - 1, max_len, out, cap, len_out);
  if (tag == 1) return tans_decode_cta(S, p + 1, plen - 1, max_len, out, cap, len_out);
  return E_CORRUPT;
}

// entropy/mod.rs:165-178: tag 3 is the LZ cascade (Max): varint(residual
// length, at most max_len) ++ an entropy-coded LZ stream of at most twice that
// + 64 bytes, decoded into the area's cascade scratch, then expanded.
__device__ uint32_t residuals_cta(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t max_len, uint8_t* out,
                                 uint64_t cap, uint64_t* len_out) {
  *len_out = 0;
  if (plen == 0 || p[0] != 3) return entropy_only_cta(S, p, plen, max_len, out, cap, len_out);
  uint64_t pos = 1, orig = 0, lzl = 0;
  uint32_t e = rd_varint(p, plen, &pos, &orig);
  if (e) return e;
  if (orig > max_len || orig > cap) return E_CORRUPT;
  if (!S.lzs || 2 * orig + 64 > S.lzs_cap) return E_NO_ENTROPY_AREA;
  e = entropy_only_cta(S, p + pos, plen - pos, 2 * orig + 64, S.lzs, S.lzs_cap, &lzl);
  if (e) return e;
  e = cta_bcast(S, threadIdx.x == 0 ? lz_decode(S.lzs, lzl, orig, out, cap) : 0u);
  if (!e) *len_out = orig;
  return e;
}

// ---------------------------------------------------------------------------
// Linear recurrences (linear.rs, High / Max): thread 0 runs them over the
// decoded residual bytes (each value depends on the previous ones).  The f64
// arithmetic is the reference's, with no contraction; NaN operands propagate
// as x86 SSE does in source order (the first NaN operand, quieted; an invalid
// operation gives the default NaN), so encode and decode stay in lock-step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double nan_op(double a, double b, double r) {
  if (isnan(a)) return as_f64(f64_bits(a) | 0x0008000000000000ull);
  if (isnan(b)) return as_f64(f64_bits(b) | 0x0008000000000000ull);
  if (isnan(r)) return as_f64(0xFFF8000000000000ull);
  return r;
}
__device__ __forceinline__ double x_mul(double a, double b) { return nan_op(a, b, __dmul_rn(a, b)); }
__device__ __forceinline__ double x_add(double a, double b) { return nan_op(a, b, __dadd_rn(a, b)); }

// linear.rs:75-100: the order-min(order, avail) Newton extrapolation from the
// history h (most recent first): 0.0 + c0*h0 + c1*h1 + ...
__device__ inline double lin_predict(const double* h, uint32_t avail, uint32_t order) {
  uint32_t eff = order < avail ? order : avail;
  double pred = 0.0;
  if (eff == 1) {
    pred = x_add(pred, x_mul(1.0, h[0]));
  } else if (eff == 2) {
    pred = x_add(pred, x_mul(2.0, h[0]));
    pred = x_add(pred, x_mul(-1.0, h[1]));
  } else if (eff == 3) {
    pred = x_add(pred, x_mul(3.0, h[0]));
    pred = x_add(pred, x_mul(-3.0, h[1]));
    pred = x_add(pred, x_mul(1.0, h[2]));
  } else if (eff == 4) {
    pred = x_add(pred, x_mul(4.0, h[0]));
    pred = x_add(pred, x_mul(-6.0, h[1]));
    pred = x_add(pred, x_mul(4.0, h[2]));
    pred = x_add(pred, x_mul(-1.0, h[3]));
  }
  return pred;
}

// The predictor hash (hash.rs:18-31): CRC32C, reflected polynomial
// 0x82F63B78, over the 8 bytes of v, by slicing: eight 256-entry tables
// (t[k][b] = the CRC of byte b followed by k zero bytes) in shared memory.
__device__ void crc_tables(uint32_t (*t)[256]) {
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x) {
    uint32_t c = i;
    for (int k = 0; k < 8; k++) c = (c >> 1) ^ (0x82F63B78u & (0u - (c & 1u)));
    t[0][i] = c;
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < 256; i += blockDim.x)
    for (int k = 1; k < 8; k++) t[k][i] = (t[k - 1][i] >> 8) ^ t[0][t[k - 1][i] & 0xFF];
  __syncthreads();
}
__device__ __forceinline__ uint32_t crc32c_u64(const uint32_t (*t)[256], uint32_t crc, uint64_t v) {
  uint32_t x = crc ^ (uint32_t)v, hi = (uint32_t)(v >> 32);
  return t[7][x & 0xFF] ^ t[6][(x >> 8) & 0xFF] ^ t[5][(x >> 16) & 0xFF] ^ t[4][x >> 24] ^ t[3][hi & 0xFF] ^
         t[2][(hi >> 8) & 0xFF] ^ t[1][(hi >> 16) & 0xFF] ^ t[0][hi >> 24];
}

// FCM (pred.rs:37-58) or DFCM (pred.rs:78-98) values from LEB128 residuals
// r[0 .. len) with a zeroed 2^plog2 table.  Thread 0 only.
__device__ uint32_t pred_values(bool dfcm, const uint8_t* r, uint64_t len, uint64_t n, uint32_t plog2,
                                const uint32_t (*crc)[256], uint64_t* table, uint64_t* vals) {
  const uint32_t seed = 0x9e3779b9u, mask = (1u << plog2) - 1u;
  uint64_t pos = 0, last = 0;
  uint32_t ctx = 0;
  for (uint64_t i = 0; i < n; i++) {
    uint64_t z;
    uint32_t e = rd_varint(r, len, &pos, &z);
    if (e) return e;
    if (!dfcm) {
      uint64_t v = z ^ table[ctx];
      vals[i] = v;
      table[ctx] = v;
      ctx = crc32c_u64(crc, seed, v) & mask;
    } else {
      uint64_t v = z ^ (last + table[ctx]);
      vals[i] = v;
      uint64_t delta = v - last;
      table[ctx] = delta;
      ctx = crc32c_u64(crc, seed, delta) & mask;
      last = v;
    }
  }
  return pos == len ? E_OK : E_CORRUPT;
}

// One linear-mode frame's values from its residual bytes r[0 .. len):
// ORDERED_DELTA (linear.rs:47-66), DELTA2 (159-179), DELTA_DP (215-237).
// Thread 0 only; returns the error kind.
__device__ uint32_t linear_values(uint32_t mode, const uint8_t* r, uint64_t len, uint64_t n, uint64_t* vals) {
  uint64_t pos = 0;
  if (mode == M_ORDERED_DELTA) {
    uint64_t p1 = 0, p2 = 0;
    for (uint64_t i = 0; i < n; i++) {
      uint64_t pred = i == 0 ? 0 : i == 1 ? p1 : p1 * 2 - p2, z;
      uint32_t e = rd_varint(r, len, &pos, &z);
      if (e) return e;
      uint64_t v = pred + unzigzag64(z);
      vals[i] = v;
      p2 = p1;
      p1 = v;
    }
    return pos == len ? E_OK : E_CORRUPT;
  }
  if (len == 0) return E_TRUNCATED;
  uint32_t order = r[0];
  if (order < 1 || order > 4) return E_CORRUPT;
  pos = 1;
  double h[4] = {0.0, 0.0, 0.0, 0.0};
  uint64_t prev = 0;
  for (uint64_t i = 0; i < n; i++) {
    double pred = lin_predict(h, i < 4 ? (uint32_t)i : 4u, order);
    uint64_t z;
    uint32_t e = rd_varint(r, len, &pos, &z);
    if (e) return e;
    double x;
    if (mode == M_DELTA2) {
      vals[i] = z ^ f64_bits(pred);
      x = as_f64(vals[i]);
    } else {
      uint64_t rb = z ^ prev;
      x = x_add(pred, as_f64(rb));
      vals[i] = f64_bits(x);
      prev = rb;
    }
    h[3] = h[2];
    h[2] = h[1];
    h[1] = h[0];
    h[0] = x;
  }
  return pos == len ? E_OK : E_CORRUPT;
}


// A frame with an entropy-coded part, decoded whole by the CTA into the
// frame's entropy area (24 bytes per value + 128, then the range coder's
// 128 KB model) and stored.  Without an
// area the frame is not decoded (E_NO_ENTROPY_AREA).
__device__ __noinline__ uint32_t decode_entropy_frame(DecSmem& S, const FrameDesc& d, const FrameAux& A, const uint8_t* p,
                                         uint8_t* ent, const DecodeOut& O) {
  int t = threadIdx.x, l = t & 31, warp = t >> 5;
  uint64_t plen = d.plen, n = d.n, c0 = d.value_off, len = 0;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  uint32_t e = E_OK;
  if (!ent) return E_NO_ENTROPY_AREA;
  if (t == 0) {
    S.rcm = reinterpret_cast<uint16_t*>(ent + ent_rc_off(n));
    S.lzs = ent + ent_lz_off(n, d.mode, O.plog2);
    S.lzs_cap = ent_lz_cap(n);
  }
  __syncthreads();
  switch (d.mode) {
    case M_LZ: {  // decoder.rs:172-175: LZ tokens (bound 16n + 1,024) over the block's bytes (lz.rs:165-172)
      uint8_t* tok = ent;
      uint64_t* vals = reinterpret_cast<uint64_t*>(ent + ((n * 16 + 1024 + 15) & ~15ull));  // 8n
      e = residuals_cta(S, p, plen, n * 16 + 1024, tok, n * 16 + 1024, &len);
      if (e) return e;
      e = cta_bcast(S, t == 0 ? lz_decode(tok, len, n * 8, reinterpret_cast<uint8_t*>(vals), n * 8) : 0u);
      if (e) return e;
      cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) { return vals[q]; });
      return E_OK;
    }
    case M_PRED:
    case M_PRED_RC:
    case M_PRED2: {  // decoder.rs:150-157: PRED's payload is the LEB128 residuals
      uint8_t* res = ent;                                                               // <= 10n + 16 bytes
      uint64_t* vals = reinterpret_cast<uint64_t*>(ent + ((n * 10 + 16 + 15) & ~15ull));  // 8n
      uint64_t* table = reinterpret_cast<uint64_t*>(ent + ent_table_off(n));
      const uint8_t* r = p;
      len = plen;
      if (d.mode != M_PRED) {
        e = residuals_cta(S, p, plen, n * 10 + 16, res, n * 10 + 16, &len);
        if (e) return e;
        r = res;
      }
      uint32_t plog2 = O.plog2 < 10 ? 10u : O.plog2 > 16 ? 16u : O.plog2;
      for (uint32_t i = t; i < (1u << plog2); i += blockDim.x) table[i] = 0;
      auto crc = reinterpret_cast<uint32_t(*)[256]>(&S.u.wbuf[0][0]);  // 8 KB of the staging area
      crc_tables(crc);
      e = cta_bcast(S, t == 0 ? pred_values(d.mode == M_PRED2, r, len, n, plog2, crc, table, vals) : 0u);
      if (e) return e;
      cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) { return vals[q]; });
      return E_OK;
    }
    case M_ORDERED_DELTA:
    case M_DELTA2:
    case M_DELTA_DP: {  // decoder.rs:162-171: residuals (bound 10n + 16), then the recurrence
      uint8_t* res = ent;                                               // <= 10n + 16 bytes
      uint64_t* vals = reinterpret_cast<uint64_t*>(ent + ((n * 10 + 16 + 15) & ~15ull));  // 8n
      e = residuals_cta(S, p, plen, n * 10 + 16, res, n * 10 + 16, &len);
      if (e) return e;
      e = cta_bcast(S, t == 0 ? linear_values(d.mode, res, len, n, vals) : 0u);
      if (e) return e;
      cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) { return vals[q]; });
      return E_OK;
    }
    case M_BYTE_TRANSPOSE: {  // transpose.rs:10-32, transform.rs:24-47
      uint8_t* bt = ent;
      e = residuals_cta(S, p, plen, n * 8 + 16, bt, n * 8 + 16, &len);
      if (e) return e;
      if (len != n * 8) return E_CORRUPT;
      cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) {
        uint64_t w = 0;
        for (int pl = 0; pl < 8; pl++) w |= (uint64_t)bt[(uint64_t)pl * n + q] << (8 * pl);
        return w;
      });
      return E_OK;
    }
    case M_FLOAT_MULT: {  // float_mult.rs:100-133, FM_ENTROPY
      uint64_t cap = n * 10 + 16;
      uint8_t* res = ent;
      e = residuals_cta(S, p + 2, plen - 2, cap, res, cap, &len);
      if (e) return e;
      uint64_t* vals = reinterpret_cast<uint64_t*>(ent + ((cap + 15) & ~15ull));
      uint32_t ee = E_OK;
      if (t == 0) {
        uint64_t pos = 0;
        int64_t prev = 0;
        for (uint64_t i = 0; i < n && !ee; i++) {
          uint64_t z = 0;
          ee = rd_varint(res, len, &pos, &z);
          if (ee) break;
          prev = (int64_t)((uint64_t)prev + unzigzag64(z));
          vals[i] = (uint64_t)prev;
        }
        if (!ee && pos != len) ee = E_CORRUPT;
      }
      e = cta_bcast(S, ee);
      if (e) return e;
      double scale = kFmScales[A.a];
      cta_store_staged(S, O, c0, (uint32_t)n,
                       [&](uint32_t q) { return f64_bits(__ddiv_rn(__ll2double_rn((long long)vals[q]), scale)); });
      return E_OK;
    }
    case M_ALP_RD: {  // alp_rd.rs:208-285 with entropy-coded codes and/or rights
      uint32_t lbw = (uint32_t)A.a, dsz = (uint32_t)A.b, rbw = 64 - lbw;
      uint8_t* codes = ent;                                   // n bytes
      uint8_t* rb = ent + ((n + 15) & ~15ull);                // rights bytes, <= 8n + 64
      uint64_t* vals = reinterpret_cast<uint64_t*>(rb + ((n * 8 + 64 + 15) & ~15ull));
      if (A.t0 == 1) {
        e = residuals_cta(S, p + A.e0, A.e1, n, codes, n, &len);
        if (e) return e;
        if (len != n) return E_CORRUPT;
      }
      const uint8_t* rsrc = p;
      uint32_t ee = E_OK;
      if (A.t1 == 0) {
        if (t == 0) ee = for_walk(p, plen, A.e2, n, S.eoffs);
      } else if (A.t1 == 1) {
        e = residuals_cta(S, p + A.e2, plen - A.e2, n * 8 + 64, rb, n * 8 + 64, &len);
        if (e) return e;
        rsrc = rb;
        if (t == 0) ee = for_walk(rb, len, 0, n, S.eoffs);
      } else {
        ee = E_CORRUPT;
      }
      e = cta_bcast(S, ee);
      if (e) return e;
      if (t == 0) S.flag = 0;
      __syncthreads();
      uint64_t* cbuf = &S.u.wbuf[warp][0];
      for (uint32_t k = warp; k < nsub; k += kDecWarps) {
        uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
        if (A.t0 == 1) {
          for (uint32_t i = l; i < cnt; i += 32) cbuf[i] = codes[(uint64_t)k * kSub + i];
        } else {
          warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t c) { cbuf[i] = c; });
        }
        __syncwarp();
        uint64_t* o = vals + (uint64_t)k * kSub;
        warp_unpack(rsrc, S.eoffs[k], cnt, [&](uint32_t i, uint64_t r) {
          uint64_t c = cbuf[i];
          if (c >= dsz) S.flag = 1;
          else o[i] = (A.dict8[c] << rbw) | r;
        });
        __syncwarp();
      }
      __syncthreads();
      if (S.flag) return E_CORRUPT;
      if (A.d) alprd_exceptions(S, p, plen, A.c, A.d, rsrc, S.eoffs, rbw, vals);
      cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) { return vals[q]; });
      return E_OK;
    }
    case M_DICT: {  // dict.rs:154-207 with TRANSPOSE values and/or CODES_ENTROPY
      uint64_t card = A.a, vtag = A.b, vpos = A.c, vlen = A.d;
      uint64_t* dv = reinterpret_cast<uint64_t*>(ent);                      // card values (card <= n)
      uint64_t* vals = reinterpret_cast<uint64_t*>(ent + 8 * n);            // also the byte-plane buffer
      uint16_t* codes = reinterpret_cast<uint16_t*>(ent + 16 * n);
      if (vtag == 0) {
        for (uint64_t i = t; i < card; i += kDecThreads) dv[i] = ld_u64(p + vpos + 8 * i);
      } else if (vtag == 1) {
        chain_prefix(S, p, A.offs[1], card, ld_u64(p + vpos), &S.u.d.stage[0][0], 4,
                     [](uint64_t v) { return unzigzag64(v); },
                     [&](uint32_t k, const uint64_t* buf, uint32_t cnt) {
                       for (uint32_t q = l; q < cnt; q += 32) dv[(uint64_t)k * kSub + q] = buf[q];
                     });
      } else {
        uint8_t* tb = reinterpret_cast<uint8_t*>(vals);
        e = residuals_cta(S, p + vpos, vlen, card * 8, tb, card * 8, &len);
        if (e) return e;
        if (len != card * 8) return E_CORRUPT;
        for (uint64_t i = t; i < card; i += kDecThreads) {
          uint64_t w = 0;
          for (int pl = 0; pl < 8; pl++) w |= (uint64_t)tb[(uint64_t)pl * card + i] << (8 * pl);
          dv[i] = w;
        }
      }
      __syncthreads();
      // codes: the tag byte follows the values (already read by the walk for
      // values tags 0 and 1, where only CODES_ENTROPY lands here)
      uint32_t ctag = 1;
      uint64_t pos = A.e0;
      if (vtag == 2) {
        uint32_t ee = E_OK;
        if (t == 0) {
          uint64_t q = vpos + vlen;
          if (q >= plen) {
            ee = E_TRUNCATED;
          } else {
            ctag = p[q];
            S.sc[2] = q + 1;
            if (ctag == 0) ee = for_walk(p, plen, q + 1, n, S.eoffs);
            else if (ctag != 1) ee = E_CORRUPT;
            S.sc[1] = ctag;
          }
        }
        e = cta_bcast(S, ee);
        if (e) return e;
        ctag = (uint32_t)S.sc[1];
        pos = S.sc[2];
        __syncthreads();
      }
      if (ctag == 0) {
        if (t == 0) S.flag = 0;
        __syncthreads();
        for (uint32_t k = warp; k < nsub; k += kDecWarps) {
          uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
          uint64_t* o = vals + (uint64_t)k * kSub;
          warp_unpack(p, S.eoffs[k], cnt, [&](uint32_t i, uint64_t c) {
            if (c >= card) S.flag = 1;
            else o[i] = dv[c];
          });
        }
        __syncthreads();
        if (S.flag) return E_CORRUPT;
      } else {
        for (uint64_t i = t; i < n; i += kDecThreads) codes[i] = 0;
        uint32_t ee = E_OK;
        uint64_t nb = 0;
        if (t == 0) {
          if (pos >= plen) {
            ee = E_TRUNCATED;
          } else {
            nb = p[pos++];
            if (nb < 1 || nb > 2) ee = E_CORRUPT;
          }
          S.sc[1] = nb;
          S.sc[2] = pos;
        }
        e = cta_bcast(S, ee);
        if (e) return e;
        nb = S.sc[1];
        pos = S.sc[2];
        __syncthreads();
        uint8_t* plane = reinterpret_cast<uint8_t*>(vals);
        for (uint64_t k = 0; k < nb; k++) {
          uint64_t ln = 0;
          ee = E_OK;
          if (t == 0) {
            ee = rd_varint(p, plen, &pos, &ln);
            if (!ee && ln > plen - pos) ee = E_TRUNCATED;
            S.sc[1] = ln;
            S.sc[2] = pos;
          }
          e = cta_bcast(S, ee);
          if (e) return e;
          ln = S.sc[1];
          pos = S.sc[2];
          __syncthreads();
          e = residuals_cta(S, p + pos, ln, n, plane, n, &len);
          if (e) return e;
          pos += ln;
          if (len != n) return E_CORRUPT;
          for (uint64_t i = t; i < n; i += kDecThreads) codes[i] |= (uint16_t)((uint32_t)plane[i] << (8 * k));
          __syncthreads();
        }
        if (t == 0) S.flag = 0;
        __syncthreads();
        for (uint64_t i = t; i < n; i += kDecThreads) {
          uint32_t c = codes[i];
          if (c >= card) S.flag = 1;
          else vals[i] = dv[c];
        }
        __syncthreads();
        if (S.flag) return E_CORRUPT;
      }
      cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) { return vals[q]; });
      return E_OK;
    }
    default:
      return E_UNSUPPORTED;
  }
}

// ---------------------------------------------------------------------------
// The decode kernel
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kDecThreads) k_decode_frames(const uint8_t* __restrict__ stream,
                                                              const FrameDesc* __restrict__ frames, int nf,
                                                              int dtype, FrameAux* aux,
                                                              DecodeOut O, uint64_t* __restrict__ scratch,
                                                              unsigned long long* __restrict__ err,
                                                              const uint32_t* __restrict__ list,
                                                              uint8_t* __restrict__ ent, BatchView bv) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  DecSmem& S = *reinterpret_cast<DecSmem*>(smem_raw);
  if ((int)blockIdx.x >= nf) return;
  int f = list ? (int)list[blockIdx.x] : (int)blockIdx.x;
  if (bv.cols) {  // a batch: the frame's column decides the output
    const BatchCol& C = bv.cols[bv.frame_col[f]];
    O = C.O;
    dtype = C.dtype;
    scratch = C.scratch;
  }
  FrameAux& A = aux[f];  // written here only by thread 0 of a deferred walk, read after a barrier
  if (A.err) return;
  FrameDesc d = frames[f];
  const uint8_t* p = stream + d.payload_off;
  if (A.defer) {  // an ALP-RD frame with exceptions: the rest of the frame walk
    uint64_t end = 0;
    uint32_t e = alprd_list_walk(S, p, d.plen, d.n, A.c, A.d, &end);
    if (!e) e = cta_bcast(S, threadIdx.x == 0 ? alprd_walk_tail(p, d.plen, d.n, end, A) : 0u);
    if (e) {
      if (threadIdx.x == 0) {
        A.err = e;
        atomicMin(err, ((unsigned long long)f << 8) | e);
      }
      return;
    }
  }
  if (A.ent) {  // entropy-coded parts, in the frame's area (FrameDesc::aux = 1 + offset / 128)
    uint8_t* area = ent && d.aux ? ent + 128ull * (d.aux - 1) : nullptr;
    uint32_t ee = decode_entropy_frame(S, d, A, p, area, O);
    if (ee && threadIdx.x == 0) atomicMin(err, ((unsigned long long)f << 8) | ee);
    return;
  }
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
        alprd_exceptions(S, p, plen, A.c, A.d, p, A.offs[1], rbw, fo);
        cta_store_staged(S, O, c0, (uint32_t)n, [&](uint32_t q) { return fo[q]; });
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

// ===========================================================================
// Warp-item decoder.  The frame table is cut into warp-sized items of at most
// 512 values (half a FastLanes sub-block) or 2048 XORZ payload bytes (four
// rounds of 512), so every
// warp of the grid has the same amount of work whatever the frame sizes.
// Modes whose values depend on everything before them in the frame carry
// state across items through a prepass:
//   DELTA  item sums of the deltas      -> carry = base + sums before
//   RLE    run-chunk (1024 runs) sums   -> start value of each chunk
//   XORZ   per item value count, XOR of the values ending in it, last
//          terminator, over-long flag   -> value base and XOR carry
// and a per-frame scan (one warp per frame) that also performs the frame-level
// checks in the sequential decoder's order.  DICT frames and ALP-RD frames
// with exceptions are decoded by k_decode_frames from a frame list.
// ===========================================================================
constexpr int kItemVals = 512;
constexpr int kItemBytes = 512;          // XORZ payload bytes per round of an item
constexpr int kXorzRounds = 4;           // rounds per XORZ item (kXorzItemBytes = 2048 payload bytes)
static_assert(kItemBytes * kXorzRounds == kXorzItemBytes, "XORZ item size shared with the readers");
constexpr int kItemStage = kItemVals + kItemVals / 16;  // u64 staging with one pad per 16
constexpr int kItemWarps = 8;
// Resident CTAs per SM the item kernel is compiled for (its register cap):
// 5 gives 48 registers a thread, and the kernel's 39 KB of shared memory
// holds five CTAs on an SM.
#ifndef QB_ITEM_MIN_BLOCKS
#define QB_ITEM_MIN_BLOCKS 5
#endif

struct PreRec {
  uint64_t a;     // DELTA/RLE: sum; XORZ: XOR of values ending in the item.  After the scan: carry / start / XOR carry
  uint64_t b;     // XORZ: value count.  After the scan: value base
  int64_t last;   // XORZ: last terminator (payload-relative), -1 if none
  uint32_t flag;  // XORZ: a value longer than 10 bytes ends in the item
  uint32_t pad;
};
static_assert(sizeof(PreRec) == 32, "PreRec layout");

__device__ __forceinline__ uint32_t skew(uint32_t i) { return i + (i >> 4); }

// Half h (values [512h, 512h+512) of a sub-block holding `count` values) of a
// FastLanes FoR sub-block; f(i, v) with i relative to the sub-block.
template <class F>
__device__ inline void warp_unpack_half(const uint8_t* p, uint32_t off, uint32_t h, uint32_t count, F f) {
  int l = threadIdx.x & 31;
  uint32_t w = p[off];
  uint64_t mn = ld_u64(p + off + 1);
  const uint8_t* words = p + off + 9;
  if (w == 0) {
    uint32_t e = min(count, (h + 1) * kItemVals);
    for (uint32_t i = h * kItemVals + l; i < e; i += 32) f(i, mn);
  } else if (w <= 32) {
    // lane l's bit stream: rows 16h .. 16h+15 start at bit 16h*w; words are
    // read once each into a 64-bit buffer
    uint32_t mask = w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u);
    uint32_t bit0 = h * 16 * w, wd = bit0 >> 5;
    const uint8_t* lw = words + 4u * l;
    uint64_t buf = ld_u32(lw + 128u * wd) >> (bit0 & 31);
    uint32_t nb = 32 - (bit0 & 31);
    wd++;
#pragma unroll 4
    for (uint32_t r = h * 16; r < h * 16 + 16; r++) {
      if (nb < w) {
        buf |= (uint64_t)ld_u32(lw + 128u * wd) << nb;
        wd++;
        nb += 32;
      }
      uint32_t v = (uint32_t)buf & mask;
      buf >>= w;
      nb -= w;
      uint32_t idx = r * 32 + l;
      if (idx < count) f(idx, mn + (uint64_t)v);
    }
  } else {
    uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1ull);
    uint32_t fl = l & 15, r0 = h * 32 + (l >> 4) * 16;
#pragma unroll 8
    for (uint32_t r = r0; r < r0 + 16; r++) {
      uint32_t idx = r * 16 + fl;
      uint32_t bit = r * w, word = bit >> 6, sh = bit & 63;
      uint64_t v = ld_u64(words + 8u * (word * 16u + fl)) >> sh;
      if (sh + w > 64) v |= ld_u64(words + 8u * ((word + 1) * 16u + fl)) << (64 - sh);
      v &= mask;
      if (idx < count) f(idx, mn + v);
    }
  }
}

// Store the run [c0, c0 + cnt) of lane values (any c0): it owns the positions
// from the c0-th valid value (0 for c0 = 0) to the (c0+cnt)-th (n at the end).
template <class V>
__device__ void warp_store_any(const DecodeOut& O, uint64_t c0, uint32_t cnt, V val) {
  if (cnt == 0) return;
  if (!O.bm32) {
    warp_store_dense(O, c0, cnt, val);
    return;
  }
  uint64_t p0, p1;
  run_positions(O, c0, c0 + cnt, &p0, &p1);
  if (p1 > p0) warp_store_words(O, p0 >> 5, (p1 + 31) >> 5, p0, p1, 0u, val);
}

// Half h of a FastLanes sub-block of width W <= 32 (rows 16h .. 16h+15 of
// every lane), with the width a compile-time constant: lane l's rows sit in
// bits [16hW, 16hW + 16W) of its word stream (word k of lane l at byte
// 4 * (32k + l) from `words`), so the words are loaded once into registers and
// every value is a fixed shift and mask of one or two of them.  A payload
// offset that is not a multiple of 4 is read with aligned loads: lane l's word
// is the funnel of its aligned word and lane l+1's (lane 31 takes lane 0's
// next one), so each word is one load.
template <int W, int H, class F>
__device__ __forceinline__ void unpack_half_w(const uint8_t* words, uint64_t mn, uint32_t count, F& f) {
  constexpr int B0 = 16 * H * W;           // first bit of the half in each lane's stream
  constexpr int K0 = B0 >> 5;              // its word
  constexpr int NW = ((B0 & 31) + 16 * W + 31) >> 5;  // words of the half
  const int l = threadIdx.x & 31;
  uint32_t wv[NW];
  const uintptr_t addr = reinterpret_cast<uintptr_t>(words);
  const uint32_t mis = (uint32_t)(addr & 3);
  const uint32_t* base = reinterpret_cast<const uint32_t*>(addr - mis);
  if (mis == 0) {
#pragma unroll
    for (int k = 0; k < NW; k++) wv[k] = __ldg(base + (K0 + k) * 32 + l);
  } else {
    uint32_t a[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) a[k] = __ldg(base + (K0 + k) * 32 + l);
    // lane 31's high part is lane 0's word of the next row
    uint32_t last = l == 0 ? __ldg(base + (K0 + NW) * 32) : 0u;
#pragma unroll
    for (int k = 0; k < NW; k++) {
      uint32_t nx = __shfl_down_sync(0xffffffffu, a[k], 1);
      uint32_t n0 = __shfl_sync(0xffffffffu, k + 1 < NW ? a[k + 1 < NW ? k + 1 : k] : last, 0);
      if (l == 31) nx = n0;
      wv[k] = __funnelshift_r(a[k], nx, mis * 8);
    }
  }
  constexpr uint32_t MASK = W == 32 ? 0xFFFFFFFFu : ((1u << W) - 1u);
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const int b = B0 + j * W - K0 * 32;  // bit within the loaded words
    const int k = b >> 5, sh = b & 31;
    uint32_t v = wv[k] >> sh;
    if (sh + W > 32) v |= wv[k + 1 < NW ? k + 1 : k] << (32 - sh);
    v &= MASK;
    uint32_t idx = (uint32_t)((16 * H + j) * 32 + l);
    if (idx < count) f(idx, mn + (uint64_t)v);
  }
}

template <int W, class F>
__device__ __forceinline__ void unpack_half_h(const uint8_t* words, uint32_t h, uint64_t mn, uint32_t count, F& f) {
  if (h) unpack_half_w<W, 1>(words, mn, count, f);
  else unpack_half_w<W, 0>(words, mn, count, f);
}

// warp_unpack_half with the widths up to 32 specialised.
template <class F>
__device__ inline void warp_unpack_half_fast(const uint8_t* p, uint32_t off, uint32_t h, uint32_t count, F f) {
  uint32_t w = p[off];
  if (w == 0 || w > 32) {
    warp_unpack_half(p, off, h, count, f);
    return;
  }
  uint64_t mn = ld_u64(p + off + 1);
  const uint8_t* words = p + off + 9;
  switch (w) {
#define QB_UNPACK_CASE(W) case W: unpack_half_h<W>(words, h, mn, count, f); break;
    QB_UNPACK_CASE(1) QB_UNPACK_CASE(2) QB_UNPACK_CASE(3) QB_UNPACK_CASE(4) QB_UNPACK_CASE(5) QB_UNPACK_CASE(6)
    QB_UNPACK_CASE(7) QB_UNPACK_CASE(8) QB_UNPACK_CASE(9) QB_UNPACK_CASE(10) QB_UNPACK_CASE(11) QB_UNPACK_CASE(12)
    QB_UNPACK_CASE(13) QB_UNPACK_CASE(14) QB_UNPACK_CASE(15) QB_UNPACK_CASE(16) QB_UNPACK_CASE(17)
    QB_UNPACK_CASE(18) QB_UNPACK_CASE(19) QB_UNPACK_CASE(20) QB_UNPACK_CASE(21) QB_UNPACK_CASE(22)
    QB_UNPACK_CASE(23) QB_UNPACK_CASE(24) QB_UNPACK_CASE(25) QB_UNPACK_CASE(26) QB_UNPACK_CASE(27)
    QB_UNPACK_CASE(28) QB_UNPACK_CASE(29) QB_UNPACK_CASE(30) QB_UNPACK_CASE(31) QB_UNPACK_CASE(32)
#undef QB_UNPACK_CASE
    default: break;
  }
}

// Store the run [c0, c0 + cnt) of lane values (any c0) like warp_store_any,
// with 16-byte stores: a lane writes 16 bytes of consecutive positions (two
// u64 or four u32 outputs) per step, so a warp's store covers 512
// consecutive bytes.  With a bitmap, the run's bitmap words (at most 32 per
// round) and their ranks relative to c0 are loaded once, one per lane, and
// each lane takes its position group's word from the lane holding it.
// Positions outside [p0, p1) (a partial group at either end) are written one
// by one; an output not 16-byte aligned goes through warp_store_any.
template <int KIND, class V>
__device__ __forceinline__ void store_group(const DecodeOut& O, uint64_t pos, uint64_t p0, uint64_t p1, uint32_t sub,
                                            uint32_t rank0, V& val) {
  constexpr uint32_t VW = KIND == 0 ? 2 : 4;
  // positions of the group inside [p0, p1); a valid one's value index is
  // rank0 + the valid positions before it in the group (those outside the
  // run count too: their values precede the run's)
  uint32_t inr = 0;
#pragma unroll
  for (uint32_t k = 0; k < VW; k++)
    if (pos + k >= p0 && pos + k < p1) inr |= 1u << k;
  uint64_t v[VW];
#pragma unroll
  for (uint32_t k = 0; k < VW; k++) {
    v[k] = 0;
    if ((sub & inr) >> k & 1u) v[k] = val(rank0 + __popc(sub & ((1u << k) - 1u)));
  }
  if (inr == (1u << VW) - 1u) {
    if (KIND == 0) {
      *reinterpret_cast<ulonglong2*>(reinterpret_cast<uint64_t*>(O.out) + pos) = make_ulonglong2(v[0], v[1]);
    } else {
      uint32_t u[VW];
#pragma unroll
      for (uint32_t k = 0; k < VW; k++) u[k] = KIND == 1 ? (uint32_t)v[k] : (v[k] ? f64bits_to_f32bits(v[k]) : 0u);
      *reinterpret_cast<uint4*>(reinterpret_cast<uint32_t*>(O.out) + pos) = make_uint4(u[0], u[1], u[VW > 2 ? 2 : 0],
                                                                                        u[VW > 3 ? 3 : 0]);
    }
  } else {
#pragma unroll
    for (uint32_t k = 0; k < VW; k++)
      if ((inr >> k) & 1u) put_kind<KIND>(O.out, pos + k, v[k]);
  }
}

template <int KIND, class V>
__device__ void warp_store_vec(const DecodeOut& O, uint64_t c0, uint32_t cnt, V& val, uint64_t* pchain) {
  constexpr uint32_t VW = KIND == 0 ? 2 : 4;
  const int l = threadIdx.x & 31;
  if (!O.bm32) {  // positions c0 .. c0 + cnt hold values 0 .. cnt
    uint64_t g0 = c0 / VW, g1 = (c0 + cnt + VW - 1) / VW;
    for (uint64_t g = g0 + l; g < g1; g += 32) {
      uint64_t pos = g * VW;
      // every position holds a value: value index = position - c0
      store_group<KIND>(O, pos, c0, c0 + cnt, (1u << VW) - 1u, (uint32_t)(pos - c0), val);
    }
    return;
  }
  uint64_t p0, p1;
  if (pchain && *pchain != ~0ull) {  // the previous run of the warp ended here
    p0 = *pchain;
    p1 = c0 + cnt >= O.nvalid ? O.n : warp_select(O, c0 + cnt);
  } else {
    run_positions(O, c0, c0 + cnt, &p0, &p1);
  }
  if (pchain) *pchain = p1;
  if (p1 <= p0) return;
  uint64_t wb = p0 >> 5, we = (p1 + 31) >> 5;
  const uint64_t nw_all = (O.n + 31) >> 5;
  for (uint64_t w0 = wb; w0 < we; w0 += 32) {
    uint32_t nwords = (uint32_t)qmin(32, we - w0);
    uint32_t mybits = 0, myrank = 0;
    if ((uint32_t)l < nwords && w0 + l < nw_all) {
      mybits = O.bm32[w0 + l];
      myrank = (uint32_t)(O.wrank[w0 + l] - c0);  // wraps below 0 for positions before the run: never used
    }
    const uint32_t ngroups = nwords * (32 / VW);
    for (uint32_t gb = 0; gb < ngroups; gb += 32) {
      uint32_t g = gb + (uint32_t)l;
      uint32_t j = (g * VW) >> 5, bo = (g * VW) & 31;
      uint32_t bits = __shfl_sync(0xffffffffu, mybits, j & 31);
      uint32_t r = __shfl_sync(0xffffffffu, myrank, j & 31);
      if (g < ngroups) {
        uint64_t pos = (w0 << 5) + (uint64_t)g * VW;
        uint32_t sub = (bits >> bo) & ((1u << VW) - 1u);
        store_group<KIND>(O, pos, p0, p1, sub, r + __popc(bits & ((1u << bo) - 1u)), val);
      }
    }
  }
}

// pchain (optional): in, the first position of this run when a previous run
// of the warp ended there (~0 when unknown); out, this run's end position.
template <class V>
__device__ void warp_store_item(const DecodeOut& O, uint64_t c0, uint32_t cnt, V val, uint64_t* pchain = nullptr) {
  if (cnt == 0) return;
  if (reinterpret_cast<uintptr_t>(O.out) & 15) {
    if (pchain) *pchain = ~0ull;
    warp_store_any(O, c0, cnt, val);
    return;
  }
  switch (out_kind(O.dtype)) {
    case 1: warp_store_vec<1>(O, c0, cnt, val, pchain); break;
    case 2: warp_store_vec<2>(O, c0, cnt, val, pchain); break;
    default: warp_store_vec<0>(O, c0, cnt, val, pchain); break;
  }
}

// In-place inclusive prefix sum (wrapping u64) of stg[skew(0 .. cnt)), cnt <=
// 512, starting from `carry`: each lane sums 16 consecutive entries.
__device__ inline void warp_prefix_skewed(uint64_t* stg, uint32_t cnt, uint64_t carry) {
  int l = threadIdx.x & 31;
  uint32_t b0 = (uint32_t)l * 16;
  uint64_t s = 0;
#pragma unroll
  for (int j = 0; j < 16; j++)
    if (b0 + j < cnt) s += stg[skew(b0 + j)];
  uint64_t inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if (l >= o) inc += u;
  }
  uint64_t run = carry + inc - s;
#pragma unroll
  for (int j = 0; j < 16; j++)
    if (b0 + j < cnt) {
      run += stg[skew(b0 + j)];
      stg[skew(b0 + j)] = run;
    }
  __syncwarp();
}

// XORZ rounds (reference codecs/xorz.rs:18-32: LEB128 of v_i ^ v_{i-1}).  A
// round is payload bytes [s0, s0 + 512) of a frame with plen bytes; lane l
// owns bytes [s0 + 16l, s0 + 16l + 16) and decodes the values whose
// terminator (a byte below 0x80) lies there, one value per step.  The round's
// bytes, with the 16 bytes before it, sit in a per-warp shared buffer, so a
// value that began in another lane or the previous round is read whole: its
// bytes, loaded as 8 (or 16) at its start, are masked to its length and
// their 7-bit groups packed together.  A value longer than 10 bytes is
// over-long (varint.rs limits); bytes 9 and 10 contribute 7 bits and 1 bit as
// the sequential reader's shifts by 56 and 63 leave them.
constexpr int kXorzBufWords = 68;  // 16 bytes before the round, 512 of it, 16 after

struct XLane {
  uint64_t b0;                  // lane's first payload byte
  uint32_t tm;                  // terminators among the lane's bytes (bit q: byte b0 + q)
  uint32_t cnt, before, total;  // lane values, values in lanes before, round values
  int64_t prev;                 // last terminator before b0 (-1: the frame's first byte starts a value)
  int64_t lastt;                // round's last terminator (-1 none)
};

__device__ __forceinline__ uint32_t term_mask8(uint64_t w) {
  uint64_t t = (~w & 0x8080808080808080ull) >> 7;
  return (uint32_t)((t * 0x0102040810204080ull) >> 56);
}

// Loads the round into xb and finds the lanes' terminators.
__device__ XLane xorz_round(const uint8_t* p, uint64_t plen, uint64_t s0, uint64_t* xb) {
  int l = threadIdx.x & 31;
  XLane X;
  X.b0 = s0 + (uint64_t)l * 16;
  uint32_t nb = X.b0 < plen ? (uint32_t)qmin(16, plen - X.b0) : 0u;
  uint64_t w0 = 0, w1 = 0;
  if (nb == 16) {
    w0 = ld_u64(p + X.b0);
    w1 = ld_u64(p + X.b0 + 8);
  } else {
    for (uint32_t q = 0; q < nb; q++) {
      uint64_t b = p[X.b0 + q];
      if (q < 8) w0 |= b << (8 * q); else w1 |= b << (8 * (q - 8));
    }
  }
  xb[2 + 2 * l] = w0;
  xb[3 + 2 * l] = w1;
  uint64_t pre = 0;  // lanes 0, 1: the 16 bytes before the round
  if (l < 2 && s0 >= 16) pre = ld_u64(p + s0 - 16 + 8 * l);
  if (l < 2) xb[l] = pre;
  if (l >= 2 && l < 4) xb[64 + l] = 0;
  uint32_t pm = l < 2 ? term_mask8(pre) << (8 * l) : 0u;
  pm |= __shfl_sync(0xffffffffu, pm, 1);
  pm = __shfl_sync(0xffffffffu, pm, 0);
  // no terminator among the 16 bytes before: the value in progress is over-long
  int64_t item_prev = s0 == 0 ? -1 : (pm ? (int64_t)s0 - 16 + (31 - __clz(pm)) : (int64_t)s0 - 17);
  uint32_t tm = term_mask8(w0) | (term_mask8(w1) << 8);
  if (nb < 16) tm &= (1u << nb) - 1u;
  X.tm = tm;
  X.cnt = __popc(tm);
  int64_t mylast = tm ? (int64_t)(X.b0 + 31 - __clz(tm)) : -1;
  uint32_t inc = X.cnt;
  int64_t mx = mylast;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
    int64_t um = __shfl_up_sync(0xffffffffu, mx, o);
    if (l >= o) {
      inc += u;
      mx = um > mx ? um : mx;
    }
  }
  X.before = inc - X.cnt;
  X.total = __shfl_sync(0xffffffffu, inc, 31);
  X.lastt = __shfl_sync(0xffffffffu, mx, 31);
  int64_t prev = __shfl_up_sync(0xffffffffu, mx, 1);  // last terminator in the lanes before
  X.prev = (l == 0 || prev < item_prev) ? item_prev : prev;
  __syncwarp();
  return X;
}

// The value whose bytes start at xb byte o and number len (1..10): up to 4
// bytes in 32-bit arithmetic, else from two (three) 64-bit words.
__device__ __forceinline__ uint64_t xorz_value(const uint64_t* xb, uint32_t o, uint32_t len) {
  if (len <= 4) {
    const uint32_t* x32 = reinterpret_cast<const uint32_t*>(xb);
    uint32_t w = __funnelshift_r(x32[o >> 2], x32[(o >> 2) + 1], (o & 3) * 8);
    if (len < 4) w &= (1u << (8 * len)) - 1u;
    w = (w & 0x007F007Fu) | ((w >> 1) & 0x3F803F80u);
    return (uint64_t)((w & 0x3FFFu) | ((w >> 2) & 0x0FFFC000u));
  }
  const uint32_t wi = o >> 3, sh = (o & 7) * 8;
  uint64_t a = xb[wi], b = xb[wi + 1];
  uint64_t w = sh ? (a >> sh) | (b << (64 - sh)) : a;
  if (len < 8) w &= (1ull << (8 * len)) - 1ull;
  w = (w & 0x007F007F007F007Full) | ((w >> 1) & 0x3F803F803F803F80ull);  // 14 bits per 16
  w = (w & 0x00003FFF00003FFFull) | ((w >> 2) & 0x0FFFC0000FFFC000ull);  // 28 bits per 32
  w = (w & 0x000000000FFFFFFFull) | ((w >> 4) & 0x00FFFFFFF0000000ull);  // 56 bits
  if (len > 8) {
    uint64_t c = xb[wi + 2];
    uint64_t hi = sh ? (b >> sh) | (c << (64 - sh)) : b;  // the value's bytes 9 and 10
    w |= (hi & 0x7Full) << 56;
    if (len > 9) w |= (hi >> 8) << 63;
  }
  return w;
}

// The lane's values in order: XOR-prefix from the lane's start, stored at
// stg[skew(before + k)] when STORE.  bad: an over-long value with index < n
// (every index when n = ~0), or (STORE) value n-1 not ending at the last
// payload byte.  Returns the XOR of the lane's values.  Positions are
// relative to s0 (the lane's last terminator before it is at least s0 - 17).
template <bool STORE>
__device__ __forceinline__ uint64_t xorz_lane_values(const XLane& X, const uint64_t* xb, uint64_t s0,
                                                     uint64_t* stg, uint64_t vbase, uint64_t n, uint64_t plen,
                                                     uint32_t& bad) {
  uint32_t m = X.tm, k = X.before;
  const int32_t b0 = (int32_t)(X.b0 - s0);
  int32_t prev = (int32_t)(X.prev - (int64_t)s0);
  // the round index of value n-1 and the payload's last byte, when in the round
  const int64_t kn = (int64_t)n - 1 - (int64_t)vbase;
  const uint32_t klast = (kn >= 0 && kn < 4096) ? (uint32_t)kn : ~0u;
  const int64_t el = (int64_t)plen - 1 - (int64_t)s0;
  const int32_t elast = (el >= 0 && el < 4096) ? (int32_t)el : -1000;
  const uint64_t lim = n > vbase ? n - vbase : 0;  // values with an index below n
  uint64_t acc = 0;
  while (m) {
    uint32_t q = __ffs(m) - 1;
    m &= m - 1u;
    int32_t end = b0 + (int32_t)q;
    int32_t len = end - prev;
    if (len <= 10) {
      acc ^= xorz_value(xb, (uint32_t)(prev + 17), (uint32_t)len);
    } else if (k < lim) {
      bad = 1;
    }
    if (STORE) {
      stg[skew(k)] = acc;
      if (k == klast && end != elast) bad = 1;
    }
    k++;
    prev = end;
  }
  return acc;
}

__device__ inline uint32_t warp_or_u32(uint32_t v) {
  for (int o = 16; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Prepass: one warp per prepass item.
__global__ void __launch_bounds__(kItemWarps * 32, 6) k_prepass(const uint8_t* __restrict__ stream,
                                                           const FrameDesc* __restrict__ frames,
                                                           const FrameAux* __restrict__ aux,
                                                           const ItemRef* __restrict__ items, uint32_t nitems,
                                                           PreRec* __restrict__ pre, uint64_t* __restrict__ scratch,
                                                           BatchView bv) {
  __shared__ __align__(16) uint32_t rle_stage[kItemWarps][kSub];  // XORZ: the round's byte buffer
  static_assert(kSub * 4 >= kXorzBufWords * 8, "the XORZ buffer fits a warp's stage");
  uint32_t g = blockIdx.x * kItemWarps + (threadIdx.x >> 5);
  int l = threadIdx.x & 31;
  if (g >= nitems) return;
  ItemRef it = items[g];
  const FrameAux& A = aux[it.frame];
  if (A.err) return;
  FrameDesc d = frames[it.frame];
  if (bv.cols) scratch = bv.cols[bv.frame_col[it.frame]].scratch;
  const uint8_t* p = stream + d.payload_off;
  uint64_t n = d.n;
  PreRec R;
  R.a = 0;
  R.b = 0;
  R.last = -1;
  R.flag = 0;
  R.pad = 0;
  if (d.mode == M_DELTA_BITPACK) {
    uint32_t k = it.local >> 1, h = it.local & 1;
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    uint64_t s = 0;
    warp_unpack_half_fast(p, A.offs[0][k], h, cnt, [&](uint32_t, uint64_t v) { s += unzigzag64(v); });
    R.a = warp_sum(s);
  } else if (d.mode == M_RLE) {
    // run chunk k: the saturating length sum (validation) and the chunk-local
    // run ends (u32, the frame's scratch range) for the output items
    uint64_t nr = A.a;
    uint32_t k = it.local;
    uint32_t cnt = (uint32_t)qmin(kSub, nr - (uint64_t)k * kSub);
    uint32_t* ends = reinterpret_cast<uint32_t*>(scratch + d.value_off) + (uint64_t)k * kSub;
    uint32_t* buf = rle_stage[threadIdx.x >> 5];
    uint64_t s = 0;
    warp_unpack(p, A.offs[0][k], cnt, [&](uint32_t i, uint64_t v) {
      s = qmin(s + qmin(v, n + 1), n + 1);
      buf[i] = (uint32_t)v;
    });
    __syncwarp();
    uint32_t run = 0;
    for (uint32_t base = 0; base < cnt; base += 32) {  // every lane takes every step
      uint32_t i = base + l;
      uint32_t inc = i < cnt ? buf[i] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
        if (l >= o) inc += u;
      }
      if (i < cnt) ends[i] = run + inc;
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
    for (int o = 16; o; o >>= 1) s = qmin(s + __shfl_xor_sync(0xffffffffu, s, o), n + 1);
    R.a = s;
  } else if (d.mode == M_XORZ) {
    // the item's rounds of 512 payload bytes: XOR of the values ending in
    // the item, value count, last terminator, over-long flag
    uint64_t* xb = reinterpret_cast<uint64_t*>(rle_stage[threadIdx.x >> 5]);
    uint64_t xo = 0;
    for (int r = 0; r < kXorzRounds; r++) {
      uint64_t s0 = (uint64_t)it.local * kXorzItemBytes + (uint64_t)r * kItemBytes;
      if (s0 >= d.plen) break;
      XLane X = xorz_round(p, d.plen, s0, xb);
      uint32_t bad = 0;
      xo ^= xorz_lane_values<false>(X, xb, s0, nullptr, 0, ~0ull, d.plen, bad);
      R.b += X.total;
      if (X.lastt > R.last) R.last = X.lastt;
      R.flag |= warp_or_u32(bad);
      __syncwarp();  // the buffer is reused by the next round
    }
    for (int o = 16; o; o >>= 1) xo ^= __shfl_xor_sync(0xffffffffu, xo, o);
    R.a = xo;
  }
  if (l == 0) pre[g] = R;
}

// Per frame (one warp): exclusive scan of its prepass records and the
// frame-level checks.  frame_pre[f] = (first prepass record, count).
__global__ void k_prepass_scan(const uint8_t* __restrict__ stream, const FrameDesc* __restrict__ frames, int nf,
                               FrameAux* __restrict__ aux, const uint2* __restrict__ frame_pre,
                               PreRec* __restrict__ pre, unsigned long long* __restrict__ err) {
  int f = blockIdx.x * kItemWarps + (threadIdx.x >> 5);
  int l = threadIdx.x & 31;
  if (f >= nf) return;
  FrameDesc d = frames[f];
  if (d.mode != M_DELTA_BITPACK && d.mode != M_RLE && d.mode != M_XORZ) return;
  if (aux[f].err) return;
  uint2 fp = frame_pre[f];
  PreRec* R = pre + fp.x;
  const uint8_t* p = stream + d.payload_off;
  uint64_t n = d.n;
  uint64_t carry_a = d.mode == M_DELTA_BITPACK ? ld_u64(p) : 0ull;
  uint64_t carry_b = 0;
  int64_t last = -1;
  uint32_t flag = 0;
  for (uint32_t b = 0; b < fp.y; b += 32) {
    uint32_t i = b + l;
    PreRec r;
    r.a = 0;
    r.b = 0;
    r.last = -1;
    r.flag = 0;
    if (i < fp.y) r = R[i];
    uint64_t ia = r.a, ib = r.b;
    int64_t im = r.last;
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t ua = __shfl_up_sync(0xffffffffu, ia, o);
      uint64_t ub = __shfl_up_sync(0xffffffffu, ib, o);
      int64_t um = __shfl_up_sync(0xffffffffu, im, o);
      if (l >= o) {
        ia = d.mode == M_XORZ ? (ia ^ ua) : (ia + ua);
        ib += ub;
        im = um > im ? um : im;
      }
    }
    if (i < fp.y) {
      R[i].a = d.mode == M_XORZ ? (carry_a ^ ia ^ r.a) : (carry_a + ia - r.a);
      R[i].b = carry_b + ib - r.b;
    }
    carry_a = d.mode == M_XORZ ? (carry_a ^ __shfl_sync(0xffffffffu, ia, 31)) : (carry_a + __shfl_sync(0xffffffffu, ia, 31));
    carry_b += __shfl_sync(0xffffffffu, ib, 31);
    int64_t bm = __shfl_sync(0xffffffffu, im, 31);
    last = bm > last ? bm : last;
    flag |= warp_or_u32(r.flag);
  }
  if (l != 0) return;
  uint32_t e = E_OK;
  if (d.mode == M_RLE) {  // rle.rs:58-71 (sums saturate at n + 1)
    if (carry_a > n) e = E_CORRUPT;
    else if (carry_a != n) e = E_LENGTH_MISMATCH;
  } else if (d.mode == M_XORZ) {  // xorz.rs:18-32 read sequentially
    if (n == 0) e = d.plen ? E_CORRUPT : E_OK;
    else if (carry_b < n) e = flag ? E_CORRUPT : ((d.plen - (uint64_t)(last + 1) >= 10) ? E_CORRUPT : E_TRUNCATED);
  }
  if (e) {
    aux[f].err = e;
    atomicMin(err, ((unsigned long long)f << 8) | e);
  }
}

// Main items: one warp per item.
__global__ void __launch_bounds__(kItemWarps * 32, QB_ITEM_MIN_BLOCKS) k_decode_items(const uint8_t* __restrict__ stream,
                                                                const FrameDesc* __restrict__ frames,
                                                                int dtype, const FrameAux* __restrict__ aux,
                                                                const ItemRef* __restrict__ items, uint32_t nitems,
                                                                const uint2* __restrict__ frame_pre,
                                                                const PreRec* __restrict__ pre, DecodeOut O,
                                                                const uint64_t* __restrict__ scratch,
                                                                unsigned long long* __restrict__ err, BatchView bv) {
  __shared__ __align__(16) uint64_t stage_all[kItemWarps][kItemStage];
  __shared__ __align__(16) uint64_t xbuf_all[kItemWarps][kXorzBufWords];  // XORZ rounds' bytes
  int warp = threadIdx.x >> 5, l = threadIdx.x & 31;
  uint32_t g = blockIdx.x * kItemWarps + warp;
  if (g >= nitems) return;
  ItemRef it = items[g];
  const FrameAux& A = aux[it.frame];
  if (A.err) return;
  FrameDesc d = frames[it.frame];
  if (bv.cols) {  // a batch: the frame's column decides the output
    const BatchCol& C = bv.cols[bv.frame_col[it.frame]];
    O = C.O;
    dtype = C.dtype;
    scratch = C.scratch;
  }
  const uint8_t* p = stream + d.payload_off;
  uint64_t n = d.n;
  uint64_t* stg = stage_all[warp];
  uint32_t e = E_OK;
  switch (d.mode) {
    case M_RAW: case M_CONST: case M_STRIDE: {
      uint64_t i0 = (uint64_t)it.local * kItemVals;
      uint32_t cnt = (uint32_t)qmin(kItemVals, n - i0);
      uint64_t c0 = d.value_off + i0;
      if (d.mode == M_CONST) {
        uint64_t v = ld_u64(p);
        warp_store_item(O, c0, cnt, [&](uint32_t) { return v; });
      } else if (d.mode == M_STRIDE) {
        uint64_t first = ld_u64(p), stride = ld_u64(p + 8);
        warp_store_item(O, c0, cnt, [&](uint32_t q) { return first + (i0 + q) * stride; });
      } else if (dtype == DT_F32) {
        warp_store_item(O, c0, cnt, [&](uint32_t q) { return f32bits_to_f64bits(ld_u32(p + 4 * (i0 + q))); });
      } else if (lane_bytes(dtype) == 4) {
        warp_store_item(O, c0, cnt, [&](uint32_t q) { return (uint64_t)ld_u32(p + 4 * (i0 + q)); });
      } else {
        warp_store_item(O, c0, cnt, [&](uint32_t q) { return ld_u64(p + 8 * (i0 + q)); });
      }
      break;
    }
    case M_FOR_BITPACK: case M_FLOAT_MULT: case M_DELTA_BITPACK: {
      uint32_t k = it.local >> 1, h = it.local & 1;
      uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
      uint32_t hb = h * kItemVals, hc = cnt > hb ? min((uint32_t)kItemVals, cnt - hb) : 0u;
      if (d.mode == M_FLOAT_MULT) {
        double scale = kFmScales[A.a];
        warp_unpack_half_fast(p, A.offs[0][k], h, cnt, [&](uint32_t i, uint64_t v) {
          stg[skew(i - hb)] = f64_bits(__ddiv_rn(__ll2double_rn((long long)v), scale));
        });
      } else if (d.mode == M_DELTA_BITPACK) {
        warp_unpack_half_fast(p, A.offs[0][k], h, cnt, [&](uint32_t i, uint64_t v) { stg[skew(i - hb)] = unzigzag64(v); });
      } else {
        warp_unpack_half_fast(p, A.offs[0][k], h, cnt, [&](uint32_t i, uint64_t v) { stg[skew(i - hb)] = v; });
      }
      __syncwarp();
      if (d.mode == M_DELTA_BITPACK) warp_prefix_skewed(stg, hc, pre[frame_pre[it.frame].x + it.local].a);
      warp_store_item(O, d.value_off + (uint64_t)k * kSub + hb, hc, [&](uint32_t q) { return stg[skew(q)]; });
      break;
    }
    case M_ALP: {
      uint32_t k = it.local >> 1, h = it.local & 1;
      uint32_t off = A.offs[0][k];
      int ee = p[off], ff = p[off + 1];
      uint32_t exc = ld_u16(p + off + 2);
      int64_t mn = (int64_t)ld_u64(p + off + 4);
      uint32_t w = p[off + 12];
      uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
      uint32_t hb = h * kItemVals, hc = cnt > hb ? min((uint32_t)kItemVals, cnt - hb) : 0u;
      const uint8_t* words = p + off + 13;
      if (w == 0) {
        uint64_t v = f64_bits(alp_decode_value(mn, ee, ff));
        for (uint32_t q = l; q < hc; q += 32) stg[skew(q)] = v;
      } else {
        uint32_t mask = w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u);
        for (uint32_t r = h * 16; r < h * 16 + 16; r++) {
          uint32_t idx = r * 32 + l;
          uint32_t bit = r * w, word = bit >> 5, sh = bit & 31;
          uint32_t v = ld_u32(words + 4u * (word * 32u + l)) >> sh;
          if (sh + w > 32) v |= ld_u32(words + 4u * ((word + 1) * 32u + l)) << (32 - sh);
          v &= mask;
          if (idx < cnt) stg[skew(idx - hb)] = f64_bits(alp_decode_value((int64_t)((uint64_t)mn + v), ee, ff));
        }
      }
      __syncwarp();
      if (exc && l == 0) {  // in order, so a repeated position keeps the last exception
        const uint8_t* xp = words + 128u * w;
        for (uint32_t x = 0; x < exc; x++) {
          uint32_t pos = ld_u16(xp + 10 * x);
          if (pos >= hb && pos < hb + kItemVals) stg[skew(pos - hb)] = ld_u64(xp + 10 * x + 2);
        }
      }
      __syncwarp();
      warp_store_item(O, d.value_off + (uint64_t)k * kSub + hb, hc, [&](uint32_t q) { return stg[skew(q)]; });
      break;
    }
    case M_ALP_RD: {  // frames without exceptions only
      uint32_t k = it.local >> 1, h = it.local & 1;
      uint32_t lbw = (uint32_t)A.a, dsz = (uint32_t)A.b, rbw = 64 - lbw;
      uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
      uint32_t hb = h * kItemVals, hc = cnt > hb ? min((uint32_t)kItemVals, cnt - hb) : 0u;
      uint32_t bad = 0;
      warp_unpack_half_fast(p, A.offs[0][k], h, cnt, [&](uint32_t i, uint64_t c) { stg[skew(i - hb)] = c; });
      __syncwarp();
      warp_unpack_half_fast(p, A.offs[1][k], h, cnt, [&](uint32_t i, uint64_t r) {
        uint64_t c = stg[skew(i - hb)];
        if (c >= dsz) bad = 1;
        else stg[skew(i - hb)] = (A.dict8[c] << rbw) | r;
      });
      __syncwarp();
      if (warp_or_u32(bad)) {
        e = E_CORRUPT;
        break;
      }
      warp_store_item(O, d.value_off + (uint64_t)k * kSub + hb, hc, [&](uint32_t q) { return stg[skew(q)]; });
      break;
    }
    case M_RLE: {
      uint64_t nr = A.a;
      const uint8_t* rv = p + A.b;
      uint32_t nrs = (uint32_t)((nr + kSub - 1) / kSub);
      const PreRec* R = pre + frame_pre[it.frame].x;  // .a = first value of each run chunk
      const uint32_t* ends = reinterpret_cast<const uint32_t*>(scratch + d.value_off);  // chunk-local run ends
      uint64_t lo = (uint64_t)it.local * kItemVals, hi = qmin(lo + kItemVals, n);
      uint32_t kc = 0;  // last chunk starting at or before lo
      for (uint32_t b = 0; b < nrs; b += 32) {
        bool ok = b + l < nrs && R[b + l].a <= lo;
        uint32_t m = __ballot_sync(0xffffffffu, ok);
        if (m) kc = b + 31 - __clz(m);
        if (m != 0xffffffffu) break;
      }
      uint64_t cs = R[kc].a;
      uint32_t ck = (uint32_t)qmin(kSub, nr - (uint64_t)kc * kSub);
      // first run of the chunk ending after lo: a ballot over every 32nd
      // run end, then over the 32 ends of that stretch (two dependent loads)
      const uint32_t* ce = ends + (uint64_t)kc * kSub;
      uint32_t a;
      {
        uint32_t q = 32u * (uint32_t)l + 31u;
        bool past = q < ck ? (cs + ce[q] > lo) : true;
        uint32_t m = __ballot_sync(0xffffffffu, past);
        uint32_t seg = __ffs(m) - 1;  // the stretch holding the answer (a lane past ck always votes)
        uint32_t q2 = 32u * seg + (uint32_t)l;
        bool past2 = q2 < ck ? (cs + ce[q2] > lo) : true;
        uint32_t m2 = __ballot_sync(0xffffffffu, past2);
        a = 32u * seg + (uint32_t)(__ffs(m2) - 1);
        if (a > ck) a = ck;
      }
      // expand the runs overlapping [lo, hi) into the staging buffer, one run
      // per lane at a time, then store
      uint64_t r = (uint64_t)kc * kSub + a;  // first run ending after lo
      for (;;) {
        uint64_t rr = r + (uint64_t)l;
        uint64_t st = hi, en = hi;
        if (rr < nr) {
          uint64_t kk = rr / kSub;
          uint64_t cbase = R[kk].a;
          en = cbase + ends[rr];
          st = (rr % kSub) ? cbase + ends[rr - 1] : cbase;
          if (st < lo) st = lo;
          if (en > hi) en = hi;
          uint64_t v = ld_u64(rv + 8ull * rr);
          for (uint64_t i = st; i < en; i++) stg[skew((uint32_t)(i - lo))] = v;
        }
        // stop once a lane's run reached hi (runs are in order)
        bool done = rr >= nr || en >= hi;
        if (__ballot_sync(0xffffffffu, done)) break;
        r += 32;
      }
      __syncwarp();
      warp_store_item(O, d.value_off + lo, (uint32_t)(hi - lo), [&](uint32_t q) { return stg[skew(q)]; });
      break;
    }
    case M_XORZ: {
      const PreRec& R = pre[frame_pre[it.frame].x + it.local];
      uint64_t vbase = R.b, carry = R.a;  // values before the item, the last one's value
      uint64_t* xb = xbuf_all[warp];
      uint64_t pnext = ~0ull;  // the next round's first position (the last round's end)
      for (int rd = 0; rd < kXorzRounds; rd++) {
        uint64_t s0 = (uint64_t)it.local * kXorzItemBytes + (uint64_t)rd * kItemBytes;
        if (s0 >= d.plen) break;
        XLane X = xorz_round(p, d.plen, s0, xb);
        uint32_t bad = 0;
        // the lane's values relative to its start, then the carry of the
        // values before: the item's, the earlier rounds' and lanes'
        uint64_t own = xorz_lane_values<true>(X, xb, s0, stg, vbase, n, d.plen, bad);
        uint64_t inc = own;
        for (int o = 1; o < 32; o <<= 1) {
          uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
          if (l >= o) inc ^= u;
        }
        uint64_t base = carry ^ inc ^ own;
        for (uint32_t q = 0; q < X.cnt; q++) stg[skew(X.before + q)] ^= base;
        carry ^= __shfl_sync(0xffffffffu, inc, 31);
        __syncwarp();
        if (warp_or_u32(bad)) {
          e = E_CORRUPT;
          break;
        }
        if (vbase < n) {
          uint32_t cnt = (uint32_t)qmin((uint64_t)X.total, n - vbase);
          warp_store_item(O, d.value_off + vbase, cnt, [&](uint32_t q) { return stg[skew(q)]; }, &pnext);
        }
        vbase += X.total;
        __syncwarp();  // the staging buffers are reused by the next round
      }
      break;
    }
    default:
      e = E_UNSUPPORTED;
      break;
  }
  if (e && l == 0) atomicMin(err, ((unsigned long long)it.frame << 8) | e);
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

// sel[m] = position of the (512*m)-th valid value: the owner of every 512th
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
    uint64_t m = (r + kSelStep - 1) / kSelStep * kSelStep;
    if (m < r + c && m < nvalid) {
      for (uint64_t k = m - r; k; k--) bits &= bits - 1u;  // drop the lower set bits
      sel[m / kSelStep] = w * 32 + (uint64_t)(__ffs(bits) - 1);
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
static void set_decode_frames_smem() {
  static std::atomic<unsigned long long> done{0};
  once_per_device(done, [] {
    cudaFuncSetAttribute(k_decode_frames, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(DecSmem));
  });
}

uint64_t decode_aux_bytes(int nf) { return (uint64_t)(nf > 0 ? nf : 1) * sizeof(FrameAux); }

void launch_decode_frames(const uint8_t* stream, const FrameDesc* frames, int nf, int dtype, const DecodeOut& out,
                          uint64_t* scratch, void* aux, unsigned long long* err, cudaStream_t st) {
  const BatchView bv{nullptr, nullptr};
  if (nf <= 0) return;
  FrameAux* A = reinterpret_cast<FrameAux*>(aux);
  k_walk_frames<<<(nf + 127) / 128, 128, 0, st>>>(stream, frames, nf, dtype, A, err, bv);
  set_decode_frames_smem();
  k_decode_frames<<<nf, kDecThreads, sizeof(DecSmem), st>>>(stream, frames, nf, dtype, A, out, scratch, err, nullptr,
                                                            nullptr, bv);
  count_launches(2);
}

void launch_decode_items(const uint8_t* stream, const FrameDesc* frames, int nf, int dtype, const DecodeOut& out,
                         const ItemPlan& plan, void* pre, uint64_t* scratch, void* aux, unsigned long long* err,
                         cudaStream_t st, const BatchView* batch) {
  const BatchView bv = batch ? *batch : BatchView{nullptr, nullptr};
  if (nf <= 0) return;
  FrameAux* A = reinterpret_cast<FrameAux*>(aux);
  PreRec* P = reinterpret_cast<PreRec*>(pre);
  k_walk_frames<<<(nf + 127) / 128, 128, 0, st>>>(stream, frames, nf, dtype, A, err, bv);
  int launches = 1;
  if (plan.npre) {
    k_prepass<<<(plan.npre + kItemWarps - 1) / kItemWarps, kItemWarps * 32, 0, st>>>(stream, frames, A,
                                                                                   plan.pre_items, plan.npre, P,
                                                                                   scratch, bv);
    launches++;
  }
  if (plan.need_scan) {
    k_prepass_scan<<<(nf + kItemWarps - 1) / kItemWarps, kItemWarps * 32, 0, st>>>(stream, frames, nf, A,
                                                                                 plan.frame_pre, P, err);
    launches++;
  }
  if (plan.nmain) {
    k_decode_items<<<(plan.nmain + kItemWarps - 1) / kItemWarps, kItemWarps * 32, 0, st>>>(
        stream, frames, dtype, A, plan.main_items, plan.nmain, plan.frame_pre, P, out, scratch, err, bv);
    launches++;
  }
  if (plan.nlist) {
    set_decode_frames_smem();
    k_decode_frames<<<plan.nlist, kDecThreads, sizeof(DecSmem), st>>>(stream, frames, (int)plan.nlist, dtype, A, out,
                                                                       scratch, err, plan.list, plan.ent, bv);
    launches++;
  }
  count_launches(launches);
}

uint64_t prepass_rec_bytes() { return sizeof(PreRec); }

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
