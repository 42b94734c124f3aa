// Column lowering and validity handling on the device: typed values -> u64
// lane with null compaction (reference lib.rs:389-403,446-454,
// validity.rs:122-127), the decimal limb split (decimal.rs:174-212,339-377)
// and the validity run-length blob (validity.rs:40-70).
#include "qb_common.cuh"
#include "qb_kernels.h"
#include "qb_scan.cuh"

namespace qb {

__device__ inline uint64_t lower_one(const uint8_t* base, uint64_t i, int dtype) {
  switch (dtype) {
    case DT_I32: return (uint64_t)(int64_t)reinterpret_cast<const int32_t*>(base)[i];
    case DT_U32: return (uint64_t)reinterpret_cast<const uint32_t*>(base)[i];
    case DT_F32: return f32bits_to_f64bits(reinterpret_cast<const uint32_t*>(base)[i]);
    default: return reinterpret_cast<const uint64_t*>(base)[i];
  }
}

__device__ inline uint32_t bm_word_at(const uint8_t* bm, uint64_t w, uint64_t n) {
  uint64_t nbytes = (n + 7) / 8;
  uint32_t bits = 0;
  for (int k = 0; k < 4; k++)
    if (w * 4 + k < nbytes) bits |= (uint32_t)bm[w * 4 + k] << (8 * k);
  uint64_t rem = n - w * 32;
  if (rem < 32) bits &= (1u << rem) - 1u;
  return bits;
}

// A warp lowers 8 bitmap words (256 positions) per step: lanes 0-7 fetch the
// words and their ranks, every lane loads its 8 values up front, then each
// valid value goes to lane[rank].
__global__ void k_lower(const uint8_t* __restrict__ values, int dtype, const uint8_t* __restrict__ bm,
                        const uint64_t* __restrict__ word_rank, uint64_t n, uint64_t* __restrict__ lane) {
  uint64_t nw = (n + 31) / 32;
  int l = threadIdx.x & 31;
  uint32_t below = (1u << l) - 1u;
  uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w0 = warp * 8; w0 < nw; w0 += nwarps * 8) {
    uint32_t mybits = 0;
    uint64_t myrank = 0;
    if (bm && l < 8 && w0 + l < nw) {
      mybits = bm_word_at(bm, w0 + l, n);
      myrank = word_rank[w0 + l];
    }
    uint64_t vals[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint64_t i = (w0 + q) * 32 + l;
      vals[q] = i < n ? lower_one(values, i, dtype) : 0ull;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint64_t i = (w0 + q) * 32 + l;
      uint32_t bits = __shfl_sync(0xffffffffu, mybits, q);
      uint64_t rank = __shfl_sync(0xffffffffu, myrank, q);
      if (i >= n) continue;
      if (!bm) lane[i] = vals[q];
      else if ((bits >> l) & 1u) lane[rank + __popc(bits & below)] = vals[q];
    }
  }
}

static unsigned grid_for_words(uint64_t n) {
  uint64_t nw = (n + 31) / 32;
  uint64_t g = (nw + 7) / 8;
  if (g > 148ull * 32) g = 148ull * 32;
  return g ? (unsigned)g : 1u;
}
static unsigned grid_for_lower(uint64_t n) {
  uint64_t nw = (n + 31) / 32;
  uint64_t g = (nw + 63) / 64;  // 8 warps x 8 words per block step
  if (g > 148ull * 32) g = 148ull * 32;
  return g ? (unsigned)g : 1u;
}

void launch_lower(const void* values, int dtype, const uint8_t* bm, const uint64_t* word_rank, uint64_t n,
                  uint64_t* lane, cudaStream_t st) {
  if (n) k_lower<<<grid_for_lower(n), 256, 0, st>>>((const uint8_t*)values, dtype, bm, word_rank, n, lane);
  count_launches(n ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Decimal: signed minimum over valid values, then limbs of (v - vmin).
// ---------------------------------------------------------------------------
struct L4 {
  uint64_t l[4];
};
__device__ inline L4 load_dec(const uint8_t* values, uint64_t i, int nl) {
  const uint64_t* p = reinterpret_cast<const uint64_t*>(values + i * 8ull * nl);
  L4 r;
  for (int k = 0; k < 4; k++) r.l[k] = k < nl ? p[k] : (uint64_t)((int64_t)p[nl - 1] >> 63);
  return r;
}
__device__ inline bool lt_signed4(const L4& a, const L4& b) {  // reference decimal.rs:254-269
  uint64_t sa = a.l[3] >> 63, sb = b.l[3] >> 63;
  if (sa != sb) return sa == 1;
  for (int i = 3; i >= 0; i--)
    if (a.l[i] != b.l[i]) return a.l[i] < b.l[i];
  return false;
}
__device__ inline bool is_valid_bit(const uint8_t* bm, uint64_t i) { return !bm || ((bm[i >> 3] >> (i & 7)) & 1); }

// Partial minima: tmp[b] = {valid flag, 4 limbs}.
__global__ void k_decimal_vmin_partial(const uint8_t* __restrict__ values, int nl, const uint8_t* __restrict__ bm,
                                       uint64_t n, uint64_t* __restrict__ tmp) {
  __shared__ L4 s_v[256];
  __shared__ int s_ok[256];
  L4 best;
  int ok = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    if (!is_valid_bit(bm, i)) continue;
    L4 x = load_dec(values, i, nl);
    if (!ok || lt_signed4(x, best)) best = x;
    ok = 1;
  }
  s_ok[threadIdx.x] = ok;
  if (ok) s_v[threadIdx.x] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    int any = 0;
    L4 m;
    for (int t = 0; t < (int)blockDim.x; t++)
      if (s_ok[t] && (!any || lt_signed4(s_v[t], m))) {
        m = s_v[t];
        any = 1;
      }
    tmp[blockIdx.x * 5] = any;
    for (int k = 0; k < 4; k++) tmp[blockIdx.x * 5 + 1 + k] = any ? m.l[k] : 0;
  }
}
__global__ void k_decimal_vmin_final(const uint64_t* __restrict__ tmp, int nparts, uint64_t* __restrict__ vmin) {
  if (threadIdx.x || blockIdx.x) return;
  int any = 0;
  L4 m;
  for (int k = 0; k < 4; k++) m.l[k] = 0;
  for (int b = 0; b < nparts; b++) {
    if (!tmp[b * 5]) continue;
    L4 x;
    for (int k = 0; k < 4; k++) x.l[k] = tmp[b * 5 + 1 + k];
    if (!any || lt_signed4(x, m)) m = x;
    any = 1;
  }
  for (int k = 0; k < 4; k++) vmin[k] = m.l[k];
}

void launch_decimal_vmin(const uint8_t* values, int nlimbs, const uint8_t* bm, uint64_t n, uint64_t* vmin_tmp,
                         uint64_t* vmin, cudaStream_t st) {
  int parts = 148 * 4;
  k_decimal_vmin_partial<<<parts, 256, 0, st>>>(values, nlimbs, bm, n, vmin_tmp);
  k_decimal_vmin_final<<<1, 32, 0, st>>>(vmin_tmp, parts, vmin);
  count_launches(2);
}

// limbs[k * stride + j] = limb k of (v_i - vmin) for the j-th valid value i.
__global__ void k_decimal_split(const uint8_t* __restrict__ values, int nl, const uint8_t* __restrict__ bm,
                                const uint64_t* __restrict__ word_rank, uint64_t n, const uint64_t* __restrict__ vmin,
                                uint64_t* __restrict__ limbs, uint64_t stride) {
  uint64_t nw = (n + 31) / 32, nbytes = (n + 7) / 8;
  int l = threadIdx.x & 31;
  uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint64_t vm[4];
  for (int k = 0; k < 4; k++) vm[k] = vmin[k];
  for (uint64_t w = warp; w < nw; w += nwarps) {
    uint64_t i = w * 32 + l;
    uint64_t j = i;
    bool valid = i < n;
    if (bm) {
      uint32_t byte = (w * 4 + (l >> 3) < nbytes) ? bm[w * 4 + (l >> 3)] : 0u;
      uint32_t bits = 0;
      for (int k = 0; k < 4; k++) bits |= __shfl_sync(0xffffffffu, byte, k * 8) << (8 * k);
      valid = valid && ((bits >> l) & 1u);
      j = word_rank[w] + __popc(bits & ((1u << l) - 1u));
    }
    if (!valid) continue;
    const uint64_t* p = reinterpret_cast<const uint64_t*>(values + i * 8ull * nl);
    uint64_t borrow = 0;
    for (int k = 0; k < nl; k++) {  // reference decimal.rs:281-293 (sub with borrow)
      uint64_t a = p[k], b = vm[k];
      uint64_t d1 = a - b;
      uint64_t b1 = a < b;
      uint64_t d2 = d1 - borrow;
      uint64_t b2 = d1 < borrow;
      limbs[k * stride + j] = d2;
      borrow = b1 | b2;
    }
  }
}

void launch_decimal_split(const uint8_t* values, int nlimbs, const uint8_t* bm, const uint64_t* word_rank,
                          uint64_t n, const uint64_t* vmin, uint64_t* limbs, uint64_t limb_stride, cudaStream_t st) {
  if (n) k_decimal_split<<<grid_for_words(n), 256, 0, st>>>(values, nlimbs, bm, word_rank, n, vmin, limbs, limb_stride);
  count_launches(n ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Validity blob: the smaller of [1] ++ LEB128 alternating run lengths
// (starting with a null run) or [0] ++ the raw bitmap bytes.
// ---------------------------------------------------------------------------
__device__ inline uint32_t bm_word(const uint8_t* bm, uint64_t w, uint64_t n) {
  uint64_t nbytes = (n + 7) / 8;
  uint32_t bits = 0;
  for (int k = 0; k < 4; k++)
    if (w * 4 + k < nbytes) bits |= (uint32_t)bm[w * 4 + k] << (8 * k);
  uint64_t rem = n - w * 32;
  if (rem < 32) bits &= (1u << rem) - 1u;
  return bits;
}
// Transition mask of word w: bit j set when bit (32w + j) differs from its
// predecessor (the bit before position 0 is taken as 0, i.e. a null).
__device__ inline uint32_t trans_mask(const uint8_t* bm, uint64_t w, uint64_t n) {
  uint32_t b = bm_word(bm, w, n);
  uint32_t prev = w ? (bm_word(bm, w - 1, n) >> 31) : 0u;
  uint32_t t = b ^ ((b << 1) | prev);
  uint64_t rem = n - w * 32;
  if (rem < 32) t &= (1u << rem) - 1u;
  return t;
}

__global__ void k_vb_last(const uint8_t* __restrict__ bm, uint64_t n, uint64_t* __restrict__ last) {
  uint64_t nw = (n + 31) / 32;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t t = trans_mask(bm, w, n);
    last[w] = t ? w * 32 + (31 - __clz(t)) : 0ull;
  }
}
__global__ void k_vb_sizes(const uint8_t* __restrict__ bm, uint64_t n, const uint64_t* __restrict__ prevpos,
                           uint64_t* __restrict__ sizes) {
  uint64_t nw = (n + 31) / 32;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t t = trans_mask(bm, w, n);
    uint64_t prev = prevpos[w], bytes = 0;
    while (t) {
      uint64_t p = w * 32 + (__ffs(t) - 1);
      t &= t - 1;
      bytes += varint_len(p - prev);
      prev = p;
    }
    sizes[w] = bytes;
  }
}
// state[0] = last transition (max-scan grand), state[1] = bytes of runs that
// end at a transition (sum-scan grand); writes the blob and its length.
__global__ void k_vb_write(const uint8_t* __restrict__ bm, uint64_t n, const uint64_t* __restrict__ prevpos,
                           const uint64_t* __restrict__ offs, const uint64_t* __restrict__ state,
                           uint8_t* __restrict__ out, uint64_t* __restrict__ blob_len) {
  uint64_t nw = (n + 31) / 32, raw_len = (n + 7) / 8;
  uint64_t t_last = state[0];
  uint64_t rle_len = state[1] + varint_len(n - t_last);
  bool rle = rle_len < raw_len;
  uint64_t gtid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, gsz = (uint64_t)gridDim.x * blockDim.x;
  if (gtid == 0) {
    out[0] = rle ? 1 : 0;
    *blob_len = 1 + (rle ? rle_len : raw_len);
  }
  if (rle) {
    for (uint64_t w = gtid; w < nw; w += gsz) {
      uint32_t t = trans_mask(bm, w, n);
      uint64_t prev = prevpos[w], pos = 1 + offs[w];
      while (t) {
        uint64_t p = w * 32 + (__ffs(t) - 1);
        t &= t - 1;
        uint64_t v = p - prev;
        do {
          uint8_t b = (uint8_t)(v & 0x7f);
          v >>= 7;
          out[pos++] = v ? (b | 0x80) : b;
        } while (v);
        prev = p;
      }
    }
    if (gtid == 0) {
      uint64_t v = n - t_last, pos = 1 + state[1];
      do {
        uint8_t b = (uint8_t)(v & 0x7f);
        v >>= 7;
        out[pos++] = v ? (b | 0x80) : b;
      } while (v);
    }
  } else {
    for (uint64_t i = gtid; i < raw_len; i += gsz) out[1 + i] = bm[i];
  }
}

// Number of bit transitions of the bitmap (added to *count).  The RLE blob
// holds one LEB128 run length per transition plus the final run, each at least
// a byte, so transitions + 1 >= ceil(n/8) proves the RAW blob is chosen.
__global__ void k_bitmap_transitions(const uint8_t* __restrict__ bm, uint64_t n, unsigned long long* count) {
  uint64_t nw = (n + 31) / 32;
  uint32_t c = 0;
  for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (uint64_t)gridDim.x * blockDim.x)
    c += __popc(trans_mask(bm, w, n));
  c = warp_sum(c);
  __shared__ uint32_t part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) t += part[k];
    if (t) atomicAdd(count, t);
  }
}
// A short column's bitmap (at most kSmallWords 32-bit words) in one CTA of
// 1,024 threads: every word's exclusive valid rank, the valid count and the
// 0/1 transition count -- k_word_popcount, the rank scan and
// k_bitmap_transitions in one launch, since short columns pay per launch.
__global__ void __launch_bounds__(1024) k_valid_small(const uint8_t* __restrict__ bm, uint64_t n,
                                                      uint64_t* __restrict__ rank, uint64_t* __restrict__ total,
                                                      unsigned long long* __restrict__ trans) {
  __shared__ uint64_t wsum[32];
  __shared__ uint32_t wtr[32];
  uint32_t nw = (uint32_t)((n + 31) / 32), t = threadIdx.x, l = t & 31, warp = t >> 5;
  uint32_t c[kSmallPer];
  uint32_t s = 0, tr = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t w = t * kSmallPer + k;
    c[k] = w < nw ? (uint32_t)__popc(bm_word_at(bm, w, n)) : 0u;
    s += c[k];
    if (w < nw) tr += __popc(trans_mask(bm, w, n));
  }
  uint64_t inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if ((int)l >= o) inc += u;
  }
  tr = warp_sum(tr);
  if (l == 31) wsum[warp] = inc;
  if (l == 0) wtr[warp] = tr;
  __syncthreads();
  if (warp == 0) {
    uint64_t x = wsum[l];
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, x, o);
      if ((int)l >= o) x += u;
    }
    wsum[l] = x;  // inclusive over warps
    uint32_t y = warp_sum(wtr[l]);
    if (l == 31) *total = x;
    if (l == 0) *trans = y;
  }
  __syncthreads();
  uint64_t run = (warp ? wsum[warp - 1] : 0ull) + inc - s;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t w = t * kSmallPer + k;
    if (w < nw) rank[w] = run;
    run += c[k];
  }
}

void launch_valid_small(const uint8_t* bm, uint64_t n, uint64_t* rank, uint64_t* total, unsigned long long* trans,
                        cudaStream_t st) {
  k_valid_small<<<1, 1024, 0, st>>>(bm, n, rank, total, trans);
  count_launches(1);
}

// Bits [bit_off, bit_off + n) of a validity bitmap (LSB first) re-packed from
// bit 0, trailing bits of the last byte cleared (the Arrow slice re-pack of
// arrow.rs:29-52, on the device).  The source holds ceil((bit_off + n) / 8)
// bytes; nothing past them is read.
__global__ void k_bitmap_repack(const uint8_t* __restrict__ src, uint64_t bit_off, uint64_t n,
                                uint8_t* __restrict__ dst) {
  uint64_t nb = (n + 7) / 8, src_bytes = (bit_off + n + 7) / 8;
  uint32_t sh = (uint32_t)(bit_off & 7);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nb; i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s0 = (bit_off >> 3) + i;
    uint32_t v = src[s0] >> sh;
    if (sh && s0 + 1 < src_bytes) v |= (uint32_t)src[s0 + 1] << (8 - sh);
    if (i == nb - 1 && (n & 7)) v &= (1u << (n & 7)) - 1u;
    dst[i] = (uint8_t)v;
  }
}

void launch_bitmap_repack(const uint8_t* src, uint64_t bit_off, uint64_t n, uint8_t* dst, cudaStream_t st) {
  uint64_t nb = (n + 7) / 8;
  if (!nb) return;
  unsigned g = (unsigned)((nb + 255) / 256 < 4096 ? (nb + 255) / 256 : 4096);
  k_bitmap_repack<<<g, 256, 0, st>>>(src, bit_off, n, dst);
  count_launches(1);
}

void launch_bitmap_transitions(const uint8_t* bm, uint64_t n, unsigned long long* count, cudaStream_t st) {
  uint64_t nw = (n + 31) / 32;
  unsigned g = (unsigned)qmin((nw + 255) / 256, 148ull * 8);
  if (g == 0) g = 1;
  k_bitmap_transitions<<<g, 256, 0, st>>>(bm, n, count);
  count_launches(1);
}

// The RAW validity blob straight into the stream: varint(1 + ceil(n/8)), tag
// 0, the bitmap bytes (validity.rs:40-70); *d_base = the stream offset after it.
__global__ void k_put_validity_raw(uint8_t* dst, uint64_t dst_off, const uint8_t* __restrict__ bm, uint64_t raw_len,
                                   uint64_t* d_base) {
  uint64_t len = 1 + raw_len;
  uint32_t vl = varint_len(len);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint64_t v = len;
    uint32_t k = 0;
    do {
      uint8_t b = (uint8_t)(v & 0x7f);
      v >>= 7;
      dst[k++] = v ? (b | 0x80) : b;
    } while (v);
    dst[vl] = 0;
    *d_base = dst_off + vl + len;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < raw_len; i += (uint64_t)gridDim.x * blockDim.x)
    dst[vl + 1 + i] = bm[i];
}
void launch_put_validity_raw(uint8_t* dst, uint64_t dst_off, const uint8_t* bm, uint64_t n, uint64_t* d_base,
                             cudaStream_t st) {
  k_put_validity_raw<<<148 * 4, 256, 0, st>>>(dst, dst_off, bm, (n + 7) / 8, d_base);
  count_launches(1);
}

uint64_t validity_tmp_words(uint64_t n) {
  uint64_t nw = (n + 31) / 32;
  return 3 * nw + scan_tiles(nw) + 8;
}

// The validity blob of a short column (at most kSmallWords words) in one CTA
// of 1,024 threads: the three passes above (last transitions + max scan, run
// bytes + sum scan, write) with block scans in place of the grid scans.
__global__ void __launch_bounds__(1024) k_vb_small(const uint8_t* __restrict__ bm, uint64_t n,
                                                   uint8_t* __restrict__ out, uint64_t* __restrict__ blob_len) {
  __shared__ uint64_t wa[32], wb[32];
  uint32_t nw = (uint32_t)((n + 31) / 32), t = threadIdx.x, l = t & 31, warp = t >> 5;
  uint32_t tm[kSmallPer];
  uint64_t mx = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t w = t * kSmallPer + k;
    tm[k] = w < nw ? trans_mask(bm, w, n) : 0u;
    if (tm[k]) mx = (uint64_t)w * 32 + (31 - __clz(tm[k]));  // words ascend: the thread's last transition
  }
  // exclusive max scan of the threads' last transitions (positions ascend, 0 = none yet)
  uint64_t inc = mx;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if ((int)l >= o) inc = u > inc ? u : inc;
  }
  uint64_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
  if (l == 0) ex = 0;
  if (l == 31) wa[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint64_t x = wa[l];
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, x, o);
      if ((int)l >= o) x = u > x ? u : x;
    }
    wa[l] = x;
  }
  __syncthreads();
  uint64_t before = warp ? wa[warp - 1] : 0ull;
  uint64_t prev0 = ex > before ? ex : before, t_last = wa[31];
  // bytes of the runs that end at this thread's transitions, then their offsets
  uint64_t prev = prev0, s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t tt = tm[k];
    uint32_t w = t * kSmallPer + k;
    while (tt) {
      uint64_t p = (uint64_t)w * 32 + (__ffs(tt) - 1);
      tt &= tt - 1;
      s += varint_len(p - prev);
      prev = p;
    }
  }
  uint64_t inc2 = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc2, o);
    if ((int)l >= o) inc2 += u;
  }
  if (l == 31) wb[warp] = inc2;
  __syncthreads();
  if (warp == 0) {
    uint64_t x = wb[l];
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, x, o);
      if ((int)l >= o) x += u;
    }
    wb[l] = x;
  }
  __syncthreads();
  uint64_t run_bytes = wb[31], raw_len = (n + 7) / 8;
  uint64_t rle_len = run_bytes + varint_len(n - t_last);
  bool rle = rle_len < raw_len;
  if (t == 0) {
    out[0] = rle ? 1 : 0;
    *blob_len = 1 + (rle ? rle_len : raw_len);
  }
  if (!rle) {
    for (uint64_t i = t; i < raw_len; i += blockDim.x) out[1 + i] = bm[i];
    return;
  }
  uint64_t pos = 1 + (warp ? wb[warp - 1] : 0ull) + inc2 - s;
  prev = prev0;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t tt = tm[k];
    uint32_t w = t * kSmallPer + k;
    while (tt) {
      uint64_t p = (uint64_t)w * 32 + (__ffs(tt) - 1);
      tt &= tt - 1;
      uint64_t v = p - prev;
      do {
        uint8_t b = (uint8_t)(v & 0x7f);
        v >>= 7;
        out[pos++] = v ? (b | 0x80) : b;
      } while (v);
      prev = p;
    }
  }
  if (t == 0) {
    uint64_t v = n - t_last, q = 1 + run_bytes;
    do {
      uint8_t b = (uint8_t)(v & 0x7f);
      v >>= 7;
      out[q++] = v ? (b | 0x80) : b;
    } while (v);
  }
}

void launch_validity_blob(const uint8_t* bm, uint64_t n, uint64_t* tmp, uint64_t* tile_tmp, uint8_t* out,
                          uint64_t* blob_len, cudaStream_t st) {
  uint64_t nw = (n + 31) / 32;
  if (nw <= kSmallWords) {
    k_vb_small<<<1, 1024, 0, st>>>(bm, n, out, blob_len);
    count_launches(1);
    return;
  }
  uint64_t* last = tmp;
  uint64_t* sizes = tmp + nw;
  uint64_t* state = tmp + 2 * nw;  // [0] t_last, [1] bytes
  unsigned g = (unsigned)qmin((nw + 255) / 256, 148ull * 16);
  if (g == 0) g = 1;
  k_vb_last<<<g, 256, 0, st>>>(bm, n, last);
  scan_exclusive<ScanMax>(last, last, nw, tile_tmp, state, st);
  k_vb_sizes<<<g, 256, 0, st>>>(bm, n, last, sizes);
  scan_exclusive<ScanSum>(sizes, sizes, nw, tile_tmp, state + 1, st);
  k_vb_write<<<g, 256, 0, st>>>(bm, n, last, sizes, state, out, blob_len);
  count_launches(9);
}

void launch_scan_sum(const uint64_t* in, uint64_t* out, uint64_t n, uint64_t* tile_tmp, uint64_t* grand,
                     cudaStream_t st) {
  scan_exclusive<ScanSum>(in, out, n ? n : 1, tile_tmp, grand, st);
  count_launches(3);
}

void launch_write_bytes(uint8_t* dst, const uint8_t* src_dev, uint64_t len, cudaStream_t st) {
  if (len) cudaMemcpyAsync(dst, src_dev, len, cudaMemcpyDeviceToDevice, st);
}

__global__ void k_put_header(uint8_t* dst, Bytes16 hdr, uint64_t* d_base) {
  if (threadIdx.x < 16) dst[threadIdx.x] = hdr.b[threadIdx.x];
  if (threadIdx.x == 0 && d_base) *d_base = 16;
}
void launch_put_header(uint8_t* dst, Bytes16 hdr, uint64_t* d_base, cudaStream_t st) {
  k_put_header<<<1, 32, 0, st>>>(dst, hdr, d_base);
  count_launches(1);
}

__global__ void k_put_validity(uint8_t* dst, uint64_t dst_off, const uint8_t* __restrict__ blob,
                               const uint64_t* __restrict__ blob_len, uint64_t* d_base) {
  uint64_t len = *blob_len;
  uint32_t vl = varint_len(len);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    uint64_t v = len;
    uint32_t k = 0;
    do {
      uint8_t b = (uint8_t)(v & 0x7f);
      v >>= 7;
      dst[k++] = v ? (b | 0x80) : b;
    } while (v);
    *d_base = dst_off + vl + len;
  }
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (uint64_t)gridDim.x * blockDim.x)
    dst[vl + i] = blob[i];
}
void launch_put_validity(uint8_t* dst, uint64_t dst_off, const uint8_t* blob, const uint64_t* blob_len,
                         uint64_t* d_base, cudaStream_t st) {
  k_put_validity<<<148 * 4, 256, 0, st>>>(dst, dst_off, blob, blob_len, d_base);
  count_launches(1);
}

}  // namespace qb
