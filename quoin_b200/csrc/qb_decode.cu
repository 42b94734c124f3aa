// Block decoder (reference src/decoder.rs:145-190 and the per-codec decode
// functions).  One CTA per frame: thread 0 walks and validates the frame's
// sub-block chain (the sub-block sizes are data-dependent), then the whole CTA
// unpacks the FastLanes-transposed words with coalesced loads and stores.
// Every payload read is bounded by the frame's plen; malformed frames set an
// error word instead of faulting.
#include "qb_common.cuh"
#include "qb_layout.h"
#include "qb_kernels.h"

namespace qb {

constexpr int kDecThreads = 256;
constexpr int kMaxSubs = kMaxBlock / kSub;  // 128
constexpr int kDictSmem = 2048;

struct DecSmem {
  uint32_t offs[kMaxSubs + 1];
  uint32_t offs2[kMaxSubs + 1];
  uint64_t buf[kSub];
  uint64_t warp_tot[kDecThreads / 32 + 1];
  uint64_t dict8[8];
  uint64_t dict[kDictSmem];
  uint64_t sc[8];  // scalars broadcast from thread 0
  uint32_t err;
  uint32_t flag;
};

// ---------------------------------------------------------------------------
// FoR sub-block chain (reference codecs/for_bitpack.rs:108-157).  Thread 0
// only.  Sub-block k = [width u8][min u64][128*width bytes].
// ---------------------------------------------------------------------------
__device__ uint32_t for_walk(const uint8_t* p, uint64_t plen, uint64_t pos, uint64_t n_values, uint32_t* offs,
                             uint64_t* end) {
  uint64_t n64;
  uint32_t e = rd_varint(p, plen, &pos, &n64);
  if (e) return e;
  if (n64 != n_values) return E_CORRUPT;
  uint32_t nsub = (uint32_t)((n_values + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    if (pos >= plen) return E_TRUNCATED;
    uint32_t w = p[pos];
    if (w > 64) return E_CORRUPT;
    if (plen - pos - 1 < 8) return E_TRUNCATED;
    uint64_t need = 128ull * w;
    if (plen - pos - 9 < need) return E_TRUNCATED;
    offs[k] = (uint32_t)pos;
    pos += 9 + need;
  }
  offs[nsub] = (uint32_t)pos;
  if (end) *end = pos;
  return E_OK;
}

// Unpack one FoR sub-block whose header starts at p[off]; calls f(i, min + r)
// for i < count.  Thread t owns FastLanes lane (t % 32) [or t % 16 for the
// 64-bit kernel], so each warp load/store touches consecutive words.
template <class F>
__device__ inline void for_unpack(const uint8_t* p, uint32_t off, uint32_t count, F f) {
  uint32_t w = p[off];
  uint64_t mn = ld_u64(p + off + 1);
  const uint8_t* words = p + off + 9;
  int t = threadIdx.x;
  if (w == 0) {
    for (uint32_t i = t; i < count; i += kDecThreads) f(i, mn);
  } else if (w <= 32) {
    uint32_t mask = w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u);
    int l = t & 31;
#pragma unroll 4
    for (int r = t >> 5; r < 32; r += kDecThreads / 32) {
      uint32_t idx = (uint32_t)(r * 32 + l);
      uint32_t bit = (uint32_t)r * w, word = bit >> 5, sh = bit & 31;
      uint32_t v = ld_u32(words + 4u * (word * 32u + l)) >> sh;
      if (sh + w > 32) v |= ld_u32(words + 4u * ((word + 1) * 32u + l)) << (32 - sh);
      v &= mask;
      if (idx < count) f(idx, mn + (uint64_t)v);
    }
  } else {
    uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1ull);
    int l = t & 15;
#pragma unroll 4
    for (int r = t >> 4; r < 64; r += kDecThreads / 16) {
      uint32_t idx = (uint32_t)(r * 16 + l);
      uint32_t bit = (uint32_t)r * w, word = bit >> 6, sh = bit & 63;
      uint64_t v = ld_u64(words + 8u * (word * 16u + l)) >> sh;
      if (sh + w > 64) v |= ld_u64(words + 8u * ((word + 1) * 16u + l)) << (64 - sh);
      v &= mask;
      if (idx < count) f(idx, mn + v);
    }
  }
}

__device__ inline uint32_t bcast_err(DecSmem& S, uint32_t e) {
  if (threadIdx.x == 0) S.err = e;
  __syncthreads();
  uint32_t r = S.err;
  __syncthreads();
  return r;
}

// Block-wide inclusive prefix of S.buf[0..count) (u64, wrapping) plus carry;
// writes the running values with `write(i, value)`.  Returns the new carry.
template <class W>
__device__ inline uint64_t chunk_prefix(DecSmem& S, uint32_t count, uint64_t carry, W write) {
  int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  uint32_t i0 = (uint32_t)t * 4;
  uint64_t v[4], s = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    v[k] = (i0 + k < count) ? S.buf[i0 + k] : 0;
    s += v[k];
  }
  uint64_t inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += u;
  }
  if (lane == 31) S.warp_tot[wid] = inc;
  __syncthreads();
  uint64_t wo = 0;
  for (int w = 0; w < wid; w++) wo += S.warp_tot[w];
  uint64_t tot = 0;
  for (int w = 0; w < kDecThreads / 32; w++) tot += S.warp_tot[w];
  uint64_t run = carry + wo + inc - s;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    run += v[k];
    if (i0 + k < count) write(i0 + k, run);
  }
  __syncthreads();
  return carry + tot;
}

// FoR-decode n values at p[pos..plen) into dst (generic pointer).
__device__ uint32_t dec_for(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t pos, uint64_t n, uint64_t* dst) {
  uint32_t e = E_OK;
  if (threadIdx.x == 0) e = for_walk(p, plen, pos, n, S.offs, nullptr);
  e = bcast_err(S, e);
  if (e) return e;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    uint64_t* o = dst + (size_t)k * kSub;
    for_unpack(p, S.offs[k], cnt, [&](uint32_t i, uint64_t v) { o[i] = v; });
  }
  return E_OK;
}

// DeltaBitpack (reference codecs/delta_bitpack.rs:48-64).
__device__ uint32_t dec_delta(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst) {
  if (plen < 8) return E_TRUNCATED;
  uint64_t base = ld_u64(p);
  const uint8_t* q = p + 8;
  uint64_t qlen = plen - 8;
  uint32_t e = E_OK;
  if (threadIdx.x == 0) e = for_walk(q, qlen, 0, n, S.offs, nullptr);
  e = bcast_err(S, e);
  if (e) return e;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  uint64_t carry = base;
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    for_unpack(q, S.offs[k], cnt, [&](uint32_t i, uint64_t v) { S.buf[i] = unzigzag64(v); });
    __syncthreads();
    uint64_t* o = dst + (size_t)k * kSub;
    carry = chunk_prefix(S, cnt, carry, [&](uint32_t i, uint64_t v) { o[i] = v; });
  }
  return E_OK;
}

// ALP (reference codecs/alp.rs:168-248).
__device__ uint32_t dec_alp(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst) {
  uint32_t e = E_OK;
  if (threadIdx.x == 0) {
    uint64_t pos = 0, n64;
    e = rd_varint(p, plen, &pos, &n64);
    if (!e && n64 != n) e = E_CORRUPT;
    uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
    for (uint32_t k = 0; !e && k < nsub; k++) {
      uint64_t count = qmin(kSub, n - (uint64_t)k * kSub);
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t ee = p[pos];
      if (pos + 1 >= plen) { e = E_TRUNCATED; break; }
      uint32_t ff = p[pos + 1];
      if (ee > 18 || ff > ee) { e = E_CORRUPT; break; }
      if (plen < pos + 4) { e = E_TRUNCATED; break; }
      uint32_t exc = ld_u16(p + pos + 2);
      if (plen < pos + 12 || pos + 12 >= plen) { e = E_TRUNCATED; break; }
      uint32_t w = p[pos + 12];
      if (w > 32) { e = E_CORRUPT; break; }
      S.offs[k] = (uint32_t)pos;
      uint64_t q = pos + 13;
      if (plen - q < 128ull * w) { e = E_TRUNCATED; break; }
      q += 128ull * w;
      for (uint32_t x = 0; x < exc; x++) {
        if (plen < q + 2 || plen < q + 10) { e = E_TRUNCATED; break; }
        if (ld_u16(p + q) >= count) { e = E_CORRUPT; break; }
        q += 10;
      }
      pos = q;
    }
  }
  e = bcast_err(S, e);
  if (e) return e;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t off = S.offs[k];
    int ee = p[off], ff = p[off + 1];
    uint32_t exc = ld_u16(p + off + 2);
    int64_t mn = (int64_t)ld_u64(p + off + 4);
    uint32_t w = p[off + 12];
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    uint64_t* o = dst + (size_t)k * kSub;
    const uint8_t* words = p + off + 13;
    int t = threadIdx.x, l = t & 31;
    if (w == 0) {
      uint64_t v = f64_bits(alp_decode_value(mn, ee, ff));
      for (uint32_t i = t; i < cnt; i += kDecThreads) o[i] = v;
    } else {
      uint32_t mask = w == 32 ? 0xFFFFFFFFu : ((1u << w) - 1u);
      for (int r = t >> 5; r < 32; r += kDecThreads / 32) {
        uint32_t idx = (uint32_t)(r * 32 + l);
        uint32_t bit = (uint32_t)r * w, word = bit >> 5, sh = bit & 31;
        uint32_t v = ld_u32(words + 4u * (word * 32u + l)) >> sh;
        if (sh + w > 32) v |= ld_u32(words + 4u * ((word + 1) * 32u + l)) << (32 - sh);
        v &= mask;
        int64_t d = (int64_t)((uint64_t)mn + (uint64_t)v);
        if (idx < cnt) o[idx] = f64_bits(alp_decode_value(d, ee, ff));
      }
    }
    if (exc) {
      __syncthreads();
      if (threadIdx.x == 0) {  // sequential patch keeps "last exception wins"
        const uint8_t* xp = words + 128u * w;
        for (uint32_t x = 0; x < exc; x++) o[ld_u16(xp + 10 * x)] = ld_u64(xp + 10 * x + 2);
      }
      __syncthreads();
    }
  }
  return E_OK;
}

// ALP-RD with bit-packed code and right streams (reference codecs/alp_rd.rs:208-285).
__device__ uint32_t dec_alprd(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst) {
  uint32_t e = E_OK;
  if (threadIdx.x == 0) {
    uint64_t pos = 0;
    do {
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t lbw = p[pos++];
      if (lbw < 1 || lbw > 63) { e = E_CORRUPT; break; }
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t dsz = p[pos++];
      if (dsz > 8) { e = E_CORRUPT; break; }
      for (uint32_t j = 0; j < dsz; j++) {
        if (plen < pos + 8) { e = E_TRUNCATED; break; }
        S.dict8[j] = ld_u64(p + pos);
        pos += 8;
      }
      if (e) break;
      uint64_t nexc;
      e = rd_varint(p, plen, &pos, &nexc);
      if (e) break;
      if (nexc > n) { e = E_CORRUPT; break; }
      uint64_t exc_start = pos;
      for (uint64_t x = 0; x < nexc; x++) {
        uint64_t pp;
        e = rd_varint(p, plen, &pos, &pp);
        if (e) break;
        if (plen < pos + 8) { e = E_TRUNCATED; break; }
        pos += 8;
        if (pp >= n) { e = E_CORRUPT; break; }
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
      if (ctag == 1 || rtag == 1) { e = ctag > 1 ? E_CORRUPT : E_UNSUPPORTED; break; }
      if (ctag != 0) { e = E_CORRUPT; break; }
      e = for_walk(p + cpos, clen, 0, n, S.offs, nullptr);
      if (e) break;
      if (rtag != 0) { e = E_CORRUPT; break; }
      e = for_walk(p + rpos, plen - rpos, 0, n, S.offs2, nullptr);
      if (e) break;
      S.sc[0] = lbw;
      S.sc[1] = dsz;
      S.sc[2] = nexc;
      S.sc[3] = exc_start;
      S.sc[4] = cpos;
      S.sc[5] = rpos;
    } while (0);
    S.flag = 0;
  }
  e = bcast_err(S, e);
  if (e) return e;
  uint32_t lbw = (uint32_t)S.sc[0], dsz = (uint32_t)S.sc[1], rbw = 64 - lbw;
  const uint8_t* cp = p + S.sc[4];
  const uint8_t* rp = p + S.sc[5];
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    for_unpack(cp, S.offs[k], cnt, [&](uint32_t i, uint64_t v) { S.buf[i] = v; });
    __syncthreads();
    uint64_t* o = dst + (size_t)k * kSub;
    for_unpack(rp, S.offs2[k], cnt, [&](uint32_t i, uint64_t r) {
      uint64_t c = S.buf[i];
      if (c >= dsz) {
        S.flag = 1;
      } else {
        o[i] = (S.dict8[c] << rbw) | r;
      }
    });
    __syncthreads();
  }
  if (S.flag) return E_CORRUPT;
  if (threadIdx.x == 0 && S.sc[2]) {
    uint64_t pos = S.sc[3], rmask = (1ull << rbw) - 1ull;
    for (uint64_t x = 0; x < S.sc[2]; x++) {
      uint64_t pp;
      rd_varint(p, plen, &pos, &pp);
      uint64_t l = ld_u64(p + pos);
      pos += 8;
      dst[pp] = (l << rbw) | (dst[pp] & rmask);
    }
  }
  __syncthreads();
  return E_OK;
}

// FLOAT_MULT with a bit-packed k stream (reference codecs/float_mult.rs:100-133).
__device__ uint32_t dec_floatmult(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst) {
  if (plen < 1) return E_TRUNCATED;
  uint32_t tag = p[0];
  if (plen < 2) return E_TRUNCATED;
  uint32_t si = p[1];
  if (si >= 7) return E_CORRUPT;
  if (tag == 1) return E_UNSUPPORTED;
  if (tag != 0) return E_CORRUPT;
  double scale = kFmScales[si];
  uint32_t e = E_OK;
  const uint8_t* q = p + 2;
  if (threadIdx.x == 0) e = for_walk(q, plen - 2, 0, n, S.offs, nullptr);
  e = bcast_err(S, e);
  if (e) return e;
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    uint64_t* o = dst + (size_t)k * kSub;
    for_unpack(q, S.offs[k], cnt,
               [&](uint32_t i, uint64_t v) { o[i] = f64_bits(__ddiv_rn(__ll2double_rn((long long)v), scale)); });
  }
  return E_OK;
}

// DICT with raw / delta values and bit-packed codes (reference codecs/dict.rs:154-207).
__device__ uint32_t dec_dict(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst,
                             uint64_t* scratch) {
  uint32_t e = E_OK;
  if (threadIdx.x == 0) {
    uint64_t pos = 0;
    do {
      uint64_t card;
      e = rd_varint(p, plen, &pos, &card);
      if (e) break;
      if (card > n) { e = E_CORRUPT; break; }
      if (pos >= plen) { e = E_TRUNCATED; break; }
      uint32_t vtag = p[pos++];
      uint64_t vlen;
      e = rd_varint(p, plen, &pos, &vlen);
      if (e) break;
      if (vlen > plen - pos) { e = E_TRUNCATED; break; }
      uint64_t vpos = pos;
      if (vtag == 0) {
        if (vlen != card * 8) { e = E_CORRUPT; break; }
      } else if (vtag == 1) {
        if (vlen < 8) { e = E_TRUNCATED; break; }
        e = for_walk(p + vpos + 8, vlen - 8, 0, card, S.offs2, nullptr);
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
      e = for_walk(p, plen, pos, n, S.offs, nullptr);
      if (e) break;
      S.sc[0] = card;
      S.sc[1] = vtag;
      S.sc[2] = vpos;
    } while (0);
    S.flag = 0;
  }
  e = bcast_err(S, e);
  if (e) return e;
  uint64_t card = S.sc[0];
  uint32_t vtag = (uint32_t)S.sc[1];
  const uint8_t* vb = p + S.sc[2];
  const uint64_t* dict = nullptr;
  if (vtag == 1) {  // delta-decode the sorted dictionary into smem or scratch
    uint64_t* dd = card <= kDictSmem ? S.dict : scratch;
    uint64_t carry = ld_u64(vb);
    const uint8_t* q = vb + 8;
    uint32_t ns = (uint32_t)((card + kSub - 1) / kSub);
    for (uint32_t k = 0; k < ns; k++) {
      uint32_t cnt = (uint32_t)qmin(kSub, card - (uint64_t)k * kSub);
      for_unpack(q, S.offs2[k], cnt, [&](uint32_t i, uint64_t v) { S.buf[i] = unzigzag64(v); });
      __syncthreads();
      uint64_t* o = dd + (size_t)k * kSub;
      carry = chunk_prefix(S, cnt, carry, [&](uint32_t i, uint64_t v) { o[i] = v; });
    }
    __syncthreads();
    dict = dd;
  }
  uint32_t nsub = (uint32_t)((n + kSub - 1) / kSub);
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t cnt = (uint32_t)qmin(kSub, n - (uint64_t)k * kSub);
    uint64_t* o = dst + (size_t)k * kSub;
    for_unpack(p, S.offs[k], cnt, [&](uint32_t i, uint64_t c) {
      if (c >= card) {
        S.flag = 1;
      } else {
        o[i] = dict ? dict[c] : ld_u64(vb + 8 * c);
      }
    });
  }
  __syncthreads();
  return S.flag ? E_CORRUPT : E_OK;
}

// RLE (reference codecs/rle.rs:44-75).
__device__ uint32_t dec_rle(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst) {
  uint32_t e = E_OK;
  if (threadIdx.x == 0) {
    uint64_t pos = 0, nr;
    do {
      e = rd_varint(p, plen, &pos, &nr);
      if (e) break;
      if (nr > n) { e = E_CORRUPT; break; }
      if (plen - pos < nr * 8) { e = E_TRUNCATED; break; }
      uint64_t vpos = pos;
      pos += nr * 8;
      e = for_walk(p, plen, pos, nr, S.offs, nullptr);
      S.sc[0] = nr;
      S.sc[1] = vpos;
    } while (0);
    S.flag = 0;
  }
  e = bcast_err(S, e);
  if (e) return e;
  uint64_t nr = S.sc[0];
  const uint8_t* rv = p + S.sc[1];
  uint32_t nsub = (uint32_t)((nr + kSub - 1) / kSub);
  uint64_t carry = 0;
  uint64_t* ends = S.dict;  // 1024 inclusive run ends of the current chunk
  for (uint32_t k = 0; k < nsub; k++) {
    uint32_t cnt = (uint32_t)qmin(kSub, nr - (uint64_t)k * kSub);
    for_unpack(p, S.offs[k], cnt, [&](uint32_t i, uint64_t v) { S.buf[i] = v; });
    __syncthreads();
    uint64_t start = carry;
    carry = chunk_prefix(S, cnt, carry, [&](uint32_t i, uint64_t v) {
      ends[i] = v;
      if (v > n || v < start) S.flag = 1;  // overrun (v < start: the prefix wrapped)
    });
    __syncthreads();
    if (S.flag) return E_CORRUPT;
    uint64_t hi = carry;  // <= n
    for (uint64_t i = start + threadIdx.x; i < hi; i += kDecThreads) {
      uint32_t lo = 0, up = cnt;  // first run with end > i
      while (lo < up) {
        uint32_t mid = (lo + up) >> 1;
        if (ends[mid] > i) up = mid; else lo = mid + 1;
      }
      dst[i] = ld_u64(rv + 8ull * ((uint64_t)k * kSub + lo));
    }
    __syncthreads();
  }
  return carry != n ? E_LENGTH_MISMATCH : E_OK;
}

// XORZ (reference codecs/xorz.rs:18-32): LEB128 XOR chain, decoded by one thread.
__device__ uint32_t dec_xorz(DecSmem& S, const uint8_t* p, uint64_t plen, uint64_t n, uint64_t* dst) {
  uint32_t e = E_OK;
  if (threadIdx.x == 0) {
    uint64_t pos = 0, prev = 0;
    for (uint64_t i = 0; i < n; i++) {
      uint64_t x;
      e = rd_varint(p, plen, &pos, &x);
      if (e) break;
      prev ^= x;
      dst[i] = prev;
    }
    if (!e && pos != plen) e = E_CORRUPT;
  }
  return bcast_err(S, e);
}

__global__ void __launch_bounds__(kDecThreads) k_decode_frames(const uint8_t* __restrict__ stream,
                                                              const FrameDesc* __restrict__ frames, int nf,
                                                              int dtype, uint64_t* __restrict__ lane,
                                                              uint64_t* __restrict__ scratch,
                                                              unsigned long long* __restrict__ err) {
  __shared__ DecSmem S;
  int f = blockIdx.x;
  if (f >= nf) return;
  FrameDesc d = frames[f];
  const uint8_t* p = stream + d.payload_off;
  uint64_t plen = d.plen, n = d.n;
  uint64_t* out = lane + d.value_off;
  uint32_t e = E_OK;
  int t = threadIdx.x;
  switch (d.mode) {
    case M_RAW: {
      uint32_t lb = lane_bytes(dtype);
      if (plen != n * lb) { e = E_CORRUPT; break; }
      if (dtype == DT_F32) {
        for (uint64_t i = t; i < n; i += kDecThreads) out[i] = f32bits_to_f64bits(ld_u32(p + 4 * i));
      } else if (lb == 4) {
        for (uint64_t i = t; i < n; i += kDecThreads) out[i] = ld_u32(p + 4 * i);
      } else {
        for (uint64_t i = t; i < n; i += kDecThreads) out[i] = ld_u64(p + 8 * i);
      }
      break;
    }
    case M_CONST: {
      if (plen != 8) { e = E_CORRUPT; break; }
      uint64_t v = ld_u64(p);
      for (uint64_t i = t; i < n; i += kDecThreads) out[i] = v;
      break;
    }
    case M_STRIDE: {
      if (plen != 16) { e = E_CORRUPT; break; }
      uint64_t first = ld_u64(p), stride = ld_u64(p + 8);
      for (uint64_t i = t; i < n; i += kDecThreads) out[i] = first + i * stride;
      break;
    }
    case M_XORZ: e = dec_xorz(S, p, plen, n, out); break;
    case M_FOR_BITPACK: e = dec_for(S, p, plen, 0, n, out); break;
    case M_DELTA_BITPACK: e = dec_delta(S, p, plen, n, out); break;
    case M_ALP: e = dec_alp(S, p, plen, n, out); break;
    case M_ALP_RD: e = dec_alprd(S, p, plen, n, out); break;
    case M_FLOAT_MULT: e = dec_floatmult(S, p, plen, n, out); break;
    case M_DICT: e = dec_dict(S, p, plen, n, out, scratch ? scratch + d.value_off : nullptr); break;
    case M_RLE: e = dec_rle(S, p, plen, n, out); break;
    default: e = E_UNSUPPORTED; break;
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
void launch_decode_frames(const uint8_t* stream, const FrameDesc* frames, int nf, int dtype, uint64_t* lane,
                          uint64_t* scratch, unsigned long long* err, cudaStream_t st) {
  if (nf > 0) k_decode_frames<<<nf, kDecThreads, 0, st>>>(stream, frames, nf, dtype, lane, scratch, err);
  count_launches(nf > 0 ? 1 : 0);
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
