// Block planner, per-block codec competition and winner emission
// (reference src/encoder.rs:154-469,644-759 and the encode functions of the
// in-path codecs).  One CTA per block.  The competition never materialises a
// candidate payload: every candidate's exact byte length is computed in closed
// form from warp-reduced statistics (sub-block widths, exception counts,
// distinct/run counts, ALP (e,f) search, ALP-RD cut search), the argmin of
// `len + penalty` is taken in the reference's candidate order with a strict
// `<`, and only the winner is written by k_emit.
#include "qb_common.cuh"
#include "qb_layout.h"
#include "qb_kernels.h"

namespace qb {

constexpr int kEncThreads = 512;
constexpr int kEncWarps = kEncThreads / 32;
constexpr int kSubsMax = kMaxBlock / kSub;  // 128
constexpr uint32_t kHashCap = 2048;         // smem hash slots (dict / ALP-RD left parts)
constexpr uint32_t kHashLimit = 1536;       // distinct keys before falling back to scratch
constexpr uint32_t kLbBits = 1u << 17;      // dict cardinality lower-bound bitset
constexpr uint32_t kRunsSmem = 4096;
constexpr uint32_t kNoLb = 0xFFFFFFFFu;

// 17-bit bucket of the dictionary cardinality lower-bound bitset.
__device__ __forceinline__ uint32_t dict_lb_bucket(uint64_t x) {
  return (uint32_t)((x * 0xD6E8FEB86659FD93ull) >> (64 - 17));
}
constexpr uint64_t kEmpty64 = ~0ull;
constexpr uint32_t kEmpty32 = 0xFFFFFFFFu;

__device__ unsigned long long g_wins[64];  // reference src/diag.rs:8-23

// Candidate decode weights (reference encoder.rs:79-89).
__host__ __device__ inline uint64_t decode_weight(int m) {
  switch (m) {
    case M_RAW: case M_CONST: case M_STRIDE: return 0;
    case M_XORZ: case M_FOR_BITPACK: case M_DELTA_BITPACK: case M_RLE: return 1;
    case M_ALP: case M_ALP_RD: case M_DICT: return 2;
    case M_PRED: return 3;
    case M_BYTE_TRANSPOSE: case M_FLOAT_MULT: return 6;
    case M_PRED_RC: case M_PRED2: return 10;
    default: return 7;
  }
}
__host__ __device__ inline uint64_t level_lambda(int level) {  // reference lib.rs:126-138
  return level == 0 ? 16 : level == 1 ? 4 : level == 2 ? 2 : 0;
}

// ---------------------------------------------------------------------------
// Small device utilities
// ---------------------------------------------------------------------------
__device__ inline void put_u8(uint8_t* d, uint32_t v) { *d = (uint8_t)v; }
__device__ inline void put_u16(uint8_t* d, uint32_t v) { d[0] = (uint8_t)v; d[1] = (uint8_t)(v >> 8); }
__device__ inline void put_u32(uint8_t* d, uint32_t v) {
#pragma unroll
  for (int i = 0; i < 4; i++) d[i] = (uint8_t)(v >> (8 * i));
}
__device__ inline void put_u64(uint8_t* d, uint64_t v) {
#pragma unroll
  for (int i = 0; i < 8; i++) d[i] = (uint8_t)(v >> (8 * i));
}
__device__ inline uint32_t put_varint(uint8_t* d, uint64_t v) {
  uint32_t n = 0;
  for (;;) {
    uint8_t b = (uint8_t)(v & 0x7f);
    v >>= 7;
    if (v) { d[n++] = b | 0x80; } else { d[n++] = b; return n; }
  }
}
__device__ inline uint64_t u64min(uint64_t a, uint64_t b) { return a < b ? a : b; }
__device__ inline uint64_t u64max(uint64_t a, uint64_t b) { return a > b ? a : b; }
__device__ inline uint32_t warp_or(uint32_t v) {
  for (int o = 16; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline uint64_t warp_or64(uint64_t v) {
  for (int o = 16; o; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline int64_t warp_min_i64(int64_t v) {
  for (int o = 16; o; o >>= 1) { int64_t u = __shfl_xor_sync(0xffffffffu, v, o); v = u < v ? u : v; }
  return v;
}
__device__ inline int64_t warp_max_i64(int64_t v) {
  for (int o = 16; o; o >>= 1) { int64_t u = __shfl_xor_sync(0xffffffffu, v, o); v = u > v ? u : v; }
  return v;
}
__device__ inline uint32_t pow2_at_least(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}
__device__ inline void atomic_min_u64(unsigned long long* a, uint64_t v) { atomicMin(a, (unsigned long long)v); }
__device__ inline void atomic_max_u64(unsigned long long* a, uint64_t v) { atomicMax(a, (unsigned long long)v); }

// In-place ascending bitonic sort of P (power of two) keys; all threads.
__device__ void block_bitonic_sort(uint64_t* a, uint32_t P) {
  for (uint32_t k = 2; k <= P; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        uint32_t ixj = i ^ j;
        if (ixj > i) {
          uint64_t x = a[i], y = a[ixj];
          bool up = (i & k) == 0;
          if ((x > y) == up) { a[i] = y; a[ixj] = x; }
        }
      }
      __syncthreads();
    }
  }
}

// (e, f) of the c-th pair in the reference's search order (alp.rs:61-62).
__device__ inline void alp_combo(uint32_t c, int* e, int* f) {
  int ee = 0;
  while ((uint32_t)((ee + 1) * (ee + 2) / 2) <= c) ee++;
  *e = ee;
  *f = (int)(c - (uint32_t)(ee * (ee + 1) / 2));
}

// FLOAT_MULT scale test (reference codecs/float_mult.rs:45-64): bit s set in
// the result when value x does NOT round-trip exactly through scale s.
__device__ inline uint32_t fm_fail_bits(uint64_t x, uint32_t alive) {
  uint32_t fail = 0;
  double xd = as_f64(x);
  while (alive) {
    int s = __ffs(alive) - 1;
    alive &= alive - 1;
    double sc = kFmScales[s];
    double k = round_half_away(__dmul_rn(xd, sc));
    bool ok = is_finite_f64(k) && fabs(k) < 9.0e18 && f64_bits(__ddiv_rn(k, sc)) == x;
    if (!ok) fail |= 1u << s;
  }
  return fail;
}
__device__ inline int64_t fm_k(uint64_t x, int s) {
  return __double2ll_rz(round_half_away(__dmul_rn(as_f64(x), kFmScales[s])));
}

// ---------------------------------------------------------------------------
// Shared memory of the competition and emission kernels
// ---------------------------------------------------------------------------
struct RdArea {
  uint64_t smp[4096];
  uint32_t hkey[kHashCap];
  uint32_t hcnt[kHashCap];
};
struct DictArea {
  uint64_t hkey[kHashCap];
  uint32_t hval[kHashCap];
  uint64_t sorted[kHashCap];
};
struct RleArea {
  uint32_t starts[kRunsSmem];
};
union BigArea {
  RdArea rd;
  DictArea dict;
  RleArea rle;
};
constexpr uint32_t kRansChunk = 4096;  // bytes staged per step of the serial rANS encoder
struct RansArea {
  uint32_t hist[256];
  uint2 fc[256];                    // (frequency, cumulative frequency) per symbol
  uint8_t buf[2][kRansChunk];       // double-buffered input bytes
  uint32_t hdr, emitted;
  uint32_t bound;  // a lower bound on the coded bytes (rans_plan)
};

struct EncSmem {
  uint8_t w_a[kSubsMax];   // FoR widths (also ALP widths in emit)
  uint8_t w_b[kSubsMax];   // delta / rights widths
  uint8_t w_c[kSubsMax];   // ALP / codes widths
  uint8_t w_d[kSubsMax];   // FLOAT_MULT widths
  uint8_t alp_ef[kSubsMax][2];
  uint16_t alp_exc[kSubsMax];
  uint32_t neq_k[kSubsMax];
  uint32_t subsz[kSubsMax + 1];
  uint64_t submin[kSubsMax];
  uint64_t item_min[kSubsMax], item_max[kSubsMax];
  unsigned long long xor_bytes, umin, umax, e_vmin, e_vmax, e_dmax, acc64;
  uint32_t neq, stride_bad, fm_mask, alp_fail, flag, ovf, card, has_max, max_rank, cnt32, dl;
  uint32_t distinct_bits[512];
  uint64_t alp_smp[kEncWarps][32];
  double rd_pv[24];
  uint64_t dict8[8];
  uint64_t red[kEncWarps];
  uint32_t red32[kEncWarps];
  uint64_t sc[8];
  uint32_t exp_lo, exp_hi;
  BigArea big;
  RansArea ra;
};

// ---------------------------------------------------------------------------
// Warp-level FoR statistics of one sub-block: width of (max - min).
// ---------------------------------------------------------------------------
template <class V>
__device__ inline void warp_minmax(uint32_t cnt, bool sgn, V val, uint64_t* mn_out, uint32_t* w_out) {
  int lane = threadIdx.x & 31;
  uint64_t umn = kEmpty64, umx = 0;
  int64_t smn = INT64_MAX, smx = INT64_MIN;
  for (uint32_t i0 = lane; i0 < cnt; i0 += 32 * 8) {
   uint64_t xs[8];
#pragma unroll
   for (int q = 0; q < 8; q++) {
     uint32_t iq = i0 + 32 * q;
     xs[q] = iq < cnt ? val(iq) : 0ull;
   }
#pragma unroll
   for (int q = 0; q < 8; q++) {
    if (i0 + 32 * q >= cnt) break;
    uint64_t x = xs[q];
    umn = u64min(umn, x);
    umx = u64max(umx, x);
    int64_t s = (int64_t)x;
    smn = s < smn ? s : smn;
    smx = s > smx ? s : smx;
   }
  }
  if (sgn) {
    smn = warp_min_i64(smn);
    smx = warp_max_i64(smx);
    *mn_out = (uint64_t)smn;
    *w_out = bit_width64((uint64_t)smx - (uint64_t)smn);
  } else {
    umn = warp_min(umn);
    umx = warp_max(umx);
    *mn_out = umn;
    *w_out = bit_width64(umx - umn);
  }
}

// Pack one FoR sub-block (header + FastLanes words) at dst; residual of
// index i = val(i) - mn for i < cnt, 0 for the padding (reference
// for_bitpack.rs:47-96, bitpack.rs:48-133).
template <class V>
__device__ inline void warp_for_pack(uint8_t* dst, uint32_t cnt, uint64_t mn, uint32_t w, V val) {
  int lane = threadIdx.x & 31;
  if (lane == 0) {
    put_u8(dst, w);
    put_u64(dst + 1, mn);
  }
  if (w == 0) return;
  uint8_t* words = dst + 9;
  if (w <= 32) {
    uint64_t acc = 0;
    uint32_t nb = 0, wd = 0;
    for (uint32_t r0 = 0; r0 < 32; r0 += 8) {
     uint32_t rs[8];
#pragma unroll
     for (int q = 0; q < 8; q++) {
       uint32_t iq = (r0 + q) * 32 + lane;
       rs[q] = iq < cnt ? (uint32_t)(val(iq) - mn) : 0u;
     }
#pragma unroll
     for (int q = 0; q < 8; q++) {
      uint32_t res = rs[q];
      if (w < 32) res &= (1u << w) - 1u;
      acc |= (uint64_t)res << nb;
      nb += w;
      if (nb >= 32) {
        put_u32(words + 4u * (wd * 32u + lane), (uint32_t)acc);
        wd++;
        acc >>= 32;
        nb -= 32;
      }
     }
    }
  } else if (lane < 16) {
    unsigned __int128 acc = 0;
    uint32_t nb = 0, wd = 0;
    for (uint32_t r0 = 0; r0 < 64; r0 += 8) {
     uint64_t rs[8];
#pragma unroll
     for (int q = 0; q < 8; q++) {
       uint32_t iq = (r0 + q) * 16 + lane;
       rs[q] = iq < cnt ? (val(iq) - mn) : 0ull;
     }
#pragma unroll
     for (int q = 0; q < 8; q++) {
      uint64_t res = rs[q];
      if (w < 64) res &= (1ull << w) - 1ull;
      acc |= (unsigned __int128)res << nb;
      nb += w;
      if (nb >= 64) {
        put_u64(words + 8u * (wd * 16u + lane), (uint64_t)acc);
        wd++;
        acc >>= 64;
        nb -= 64;
      }
     }
    }
  }
}

// Second half of the FoR stream writer: with S.w_a[k] / S.submin[k] set for
// every sub-block, lays out varint(M) + sub-blocks and (dst non-null) packs
// val(0..M).  Returns the byte length (all threads).
template <class V>
__device__ uint64_t block_for_write(EncSmem& S, uint8_t* dst, uint32_t M, V val) {
  int warp = threadIdx.x >> 5;
  uint32_t nsub = (M + kSub - 1) / kSub;
  if (threadIdx.x == 0) {
    uint32_t off = varint_len(M);
    for (uint32_t k = 0; k < nsub; k++) {
      S.subsz[k] = off;
      off += 9 + 128u * S.w_a[k];
    }
    S.subsz[nsub] = off;
    if (dst) put_varint(dst, M);
  }
  __syncthreads();
  uint64_t total = S.subsz[nsub];
  if (dst) {
    for (uint32_t k = warp; k < nsub; k += kEncWarps) {
      uint32_t cnt = min((uint32_t)kSub, M - k * kSub);
      warp_for_pack(dst + S.subsz[k], cnt, S.submin[k], S.w_a[k], [&](uint32_t i) { return val(k * kSub + i); });
    }
  }
  __syncthreads();
  return total;
}

// Whole-CTA FoR stream writer: varint(M) + sub-blocks of val(0..M).  When
// dst is null only the size is computed.  Returns the byte length (all threads).
template <class V>
__device__ uint64_t block_for(EncSmem& S, uint8_t* dst, uint32_t M, bool sgn, V val) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nsub = (M + kSub - 1) / kSub;
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t cnt = min((uint32_t)kSub, M - k * kSub);
    uint64_t mn;
    uint32_t w;
    warp_minmax(cnt, sgn, [&](uint32_t i) { return val(k * kSub + i); }, &mn, &w);
    if (lane == 0) {
      S.w_a[k] = (uint8_t)w;
      S.submin[k] = mn;
    }
  }
  __syncthreads();
  return block_for_write(S, dst, M, val);
}

// alp_roundtrips_r with the four powers of ten of its (e, f) given:
// pe = 10^e, pf = 10^-f (encode), qf = 10^f, qe = 10^-e (decode).
__device__ __forceinline__ bool alp_rt_pow(uint64_t bits, double pe, double pf, double qf, double qe, double* r) {
  double tmp = __dmul_rn(__dmul_rn(as_f64(bits), pe), pf);
  const double kUpper = 9.223372036854776e18, kMagic = 6755399441055744.0;
  if (!is_finite_f64(tmp) || tmp >= kUpper || tmp <= -kUpper) return false;
  double rr = __dadd_rn(__dadd_rn(tmp, kMagic), -kMagic);
  *r = rr;
  return f64_bits(__dmul_rn(__dmul_rn(rr, qf), qe)) == bits;
}

// ALP for one sub-block (reference alp.rs:49-166): find_ef on the 32-value
// sample, then the full encode statistics.  Warp-cooperative; returns false
// when the sub-block (hence the block) bails.
struct AlpSub {
  int e, f;
  uint32_t w, exc;
  int64_t mn, filler;
};
__device__ bool alp_subblock_ef(const uint64_t* sv, uint32_t cnt, int e, int f, const double* pexp,
                                const double* pfrac, AlpSub* out);
__device__ bool alp_subblock(const uint64_t* sv, uint32_t cnt, uint64_t* smp, const double* pexp, const double* pfrac,
                             AlpSub* out) {
  int lane = threadIdx.x & 31;
  uint32_t st = max(cnt / 32u, 1u);
  uint32_t sl = min(32u, (cnt + st - 1) / st);
  smp[lane] = (uint32_t)lane < sl ? sv[lane * st] : 0ull;
  __syncwarp();
  uint64_t best_cost = kEmpty64;
  uint32_t best_c = 0xFFFF, best_exc = 0;
  const double kInf = __longlong_as_double(0x7FF0000000000000ll);
  for (uint32_t c = lane; c < 190; c += 32) {
    int e, f;
    alp_combo(c, &e, &f);
    const double pe = pexp[e], pf = pfrac[f], qf = pexp[f], qe = pfrac[e];
    uint32_t ex = 0;
    double lo = kInf, hi = -kInf;  // digits as the integral doubles they are cast from
    for (uint32_t s = 0; s < sl; s++) {
      double r;
      if (alp_rt_pow(smp[s], pe, pf, qf, qe, &r)) {
        lo = r < lo ? r : lo;
        hi = r > hi ? r : hi;
      } else {
        ex++;
      }
    }
    int64_t lo_i = ex == sl ? 0 : f64_as_i64(lo), hi_i = ex == sl ? 0 : f64_as_i64(hi);
    uint32_t width = (ex == sl) ? 64u : (hi_i <= lo_i ? 0u : bit_width64((uint64_t)hi_i - (uint64_t)lo_i));
    uint64_t cost = (uint64_t)width * sl + (uint64_t)ex * 80;
    if (cost < best_cost) {
      best_cost = cost;
      best_c = c;
      best_exc = ex;
    }
  }
  for (int o = 16; o; o >>= 1) {
    uint64_t oc = __shfl_xor_sync(0xffffffffu, best_cost, o);
    uint32_t occ = __shfl_xor_sync(0xffffffffu, best_c, o);
    uint32_t oe = __shfl_xor_sync(0xffffffffu, best_exc, o);
    if (oc < best_cost || (oc == best_cost && occ < best_c)) {
      best_cost = oc;
      best_c = occ;
      best_exc = oe;
    }
  }
  __syncwarp();
  if (best_exc * 2 > sl) return false;
  int e, f;
  alp_combo(best_c, &e, &f);
  return alp_subblock_ef(sv, cnt, e, f, pexp, pfrac, out);
}

// The encode pass of one sub-block for a chosen (e, f) (alp.rs:109-166):
// exceptions, digit range, the filler digit.  Warp-cooperative; false when
// the digits need more than 32 bits.
__device__ bool alp_subblock_ef(const uint64_t* sv, uint32_t cnt, int e, int f, const double* pexp,
                                const double* pfrac, AlpSub* out) {
  int lane = threadIdx.x & 31;
  const double kInf = __longlong_as_double(0x7FF0000000000000ll);
  const double pe = pexp[e], pf = pfrac[f], qf = pexp[f], qe = pfrac[e];
  uint32_t exc = 0, first_li = 0xFFFFFFFFu;
  double rmn = kInf, rmx = -kInf, first_r = 0.0;
  for (uint32_t j = 0; j < 32; j++) {
    uint32_t li = j * 32 + lane;
    bool ok = li < cnt;
    double r = 0.0;
    bool rt = ok && alp_rt_pow(sv[li], pe, pf, qf, qe, &r);
    if (rt) {
      rmn = r < rmn ? r : rmn;
      rmx = r > rmx ? r : rmx;
      if (li < first_li) {
        first_li = li;
        first_r = r;
      }
    }
    exc += __popc(__ballot_sync(0xffffffffu, ok && !rt));
  }
  int64_t first_d = f64_as_i64(first_r);
  int64_t dmn = rmn == kInf ? INT64_MAX : f64_as_i64(rmn), dmx = rmx == -kInf ? INT64_MIN : f64_as_i64(rmx);
  dmn = warp_min_i64(dmn);
  dmx = warp_max_i64(dmx);
  for (int o = 16; o; o >>= 1) {
    uint32_t ol = __shfl_xor_sync(0xffffffffu, first_li, o);
    int64_t od = __shfl_xor_sync(0xffffffffu, first_d, o);
    if (ol < first_li) {
      first_li = ol;
      first_d = od;
    }
  }
  int64_t filler = first_li == 0xFFFFFFFFu ? 0 : first_d;
  if (first_li == 0xFFFFFFFFu) dmn = dmx = 0;
  uint32_t w = bit_width64((uint64_t)dmx - (uint64_t)dmn);
  if (w > 32) return false;
  out->e = e;
  out->f = f;
  out->w = w;
  out->exc = exc;
  out->mn = dmn;
  out->filler = filler;
  return true;
}

// ---------------------------------------------------------------------------
// ALP-RD: cut search on the sample (reference alp_rd.rs:80-107).  Uses the
// sorted sample: for a cut, the equal-left groups are runs of the sorted
// sample, and only the sum of the 8 largest group counts matters.
// ---------------------------------------------------------------------------
__device__ inline void top8_insert(uint32_t (&t)[8], uint32_t c) {
  if (c <= t[7]) return;
  t[7] = c;
#pragma unroll
  for (int i = 7; i > 0; i--) {
    if (t[i] > t[i - 1]) {
      uint32_t x = t[i];
      t[i] = t[i - 1];
      t[i - 1] = x;
    }
  }
}
__device__ inline uint32_t rd_code_bits(uint32_t dl) {
  if (dl <= 1) return 1;
  uint32_t b = bit_width64((uint64_t)(dl - 1));
  return b ? b : 1;
}

// Returns the chosen left bit width, or 0 when ALP-RD does not apply.  The
// sample is block[0], block[step], ... (step = max(n/2048, 1)); when `pre` is
// given it holds those values at pre[i * pre_stride].
__device__ uint32_t rd_choose_cut(EncSmem& S, const uint64_t* v, uint32_t n, const uint64_t* pre, uint32_t pre_stride) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t step = max(n / 2048u, 1u);
  uint32_t sn = (n + step - 1) / step;
  uint32_t P = pow2_at_least(sn);
  uint64_t* smp = S.big.rd.smp;
  for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)
    smp[i] = i < sn ? (pre ? pre[(uint64_t)i * pre_stride] : v[(uint64_t)i * step]) : kEmpty64;
  __syncthreads();
  block_bitonic_sort(smp, P);
  for (uint32_t lbw = warp + 1; lbw <= 24; lbw += blockDim.x / 32) {
    uint32_t rbw = 64 - lbw;
    uint32_t t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t last_start = 0, G = 0;
    for (uint32_t base = 0; base < sn; base += 32) {
      uint32_t i = base + lane;
      bool ok = i < sn;
      bool bnd = ok && (i == 0 || (smp[i] >> rbw) != (smp[i - 1] >> rbw));
      uint32_t m = __ballot_sync(0xffffffffu, bnd);
      G += __popc(m);
      if (bnd && i > 0) {
        uint32_t below = m & ((1u << lane) - 1u);
        uint32_t ps = below ? base + (31 - __clz(below)) : last_start;
        top8_insert(t, i - ps);
      }
      if (m) last_start = base + (31 - __clz(m));
    }
    if (lane == 0) top8_insert(t, sn - last_start);
    uint64_t cov = 0;
    for (int r = 0; r < 8; r++) {
      uint32_t mx = warp_max(t[0]);
      if (mx == 0) break;
      uint32_t who = __ballot_sync(0xffffffffu, t[0] == mx);
      if (lane == __ffs(who) - 1) {
#pragma unroll
        for (int i = 0; i < 7; i++) t[i] = t[i + 1];
        t[7] = 0;
      }
      cov += mx;
    }
    uint32_t dl = min(G, 8u);
    uint64_t num = (uint64_t)sn * (uint64_t)(rbw + rd_code_bits(dl)) + ((uint64_t)sn - cov) * 96ull;
    if (lane == 0) S.rd_pv[lbw - 1] = __ddiv_rn(__ull2double_rn(num), __ull2double_rn((uint64_t)sn));
  }
  __syncthreads();
  uint32_t best = 0;
  if (threadIdx.x == 0) {
    double bb = __longlong_as_double(0x7FF0000000000000ll);  // +inf
    for (uint32_t lbw = 1; lbw <= 24; lbw++) {
      if (S.rd_pv[lbw - 1] < bb) {
        bb = S.rd_pv[lbw - 1];
        best = lbw;
      }
    }
    if (best == 0 || bb >= 63.0) best = 0;
    S.sc[0] = best;
  }
  __syncthreads();
  best = (uint32_t)S.sc[0];
  __syncthreads();
  return best;
}

// Full-block top-8 left parts by (count desc, key asc) (reference
// alp_rd.rs:47-68).  Counts go to a smem hash; when the block has more
// distinct left parts than the smem table holds, a scratch table is used.
__device__ void rd_top8(EncSmem& S, const uint64_t* v, uint32_t n, uint32_t lbw, uint8_t* scratch) {
  uint32_t rbw = 64 - lbw;
  uint32_t* hk = S.big.rd.hkey;
  uint32_t* hc = S.big.rd.hcnt;
  for (uint32_t i = threadIdx.x; i < kHashCap; i += blockDim.x) {
    hk[i] = kEmpty32;
    hc[i] = 0;
  }
  if (threadIdx.x == 0) {
    S.ovf = 0;
    S.cnt32 = 0;
  }
  __syncthreads();
  // Counts are warp-aggregated: the lanes holding equal left parts (few
  // distinct ones is the common case) add once, by their lowest lane.
  int lane0 = threadIdx.x & 31;
  for (uint32_t base = threadIdx.x & ~31u; base < n; base += blockDim.x) {
    if (__any_sync(0xffffffffu, *(volatile uint32_t*)&S.ovf != 0)) break;
    uint32_t i = base + lane0;
    uint32_t key = i < n ? (uint32_t)(v[i] >> rbw) : kEmpty32;  // left parts are < 2^24
    uint32_t peers = __match_any_sync(0xffffffffu, key);
    if (key == kEmpty32 || lane0 != __ffs(peers) - 1) continue;
    uint32_t add = __popc(peers);
    uint32_t h = (uint32_t)(((uint64_t)key * 0x9E3779B97F4A7C15ull) >> 53);  // 11 bits
    for (uint32_t probe = 0; probe < kHashCap; probe++) {
      uint32_t cur = hk[h];
      if (cur == kEmpty32) {
        uint32_t old = atomicCAS(&hk[h], kEmpty32, key);
        if (old == kEmpty32) {
          if (atomicAdd(&S.cnt32, 1u) >= kHashLimit) S.ovf = 1;
          cur = key;
        } else {
          cur = old;
        }
      }
      if (cur == key) {
        atomicAdd(&hc[h], add);
        break;
      }
      h = (h + 1) & (kHashCap - 1);
    }
  }
  __syncthreads();
  uint32_t* tk = hk;
  uint32_t* tc = hc;
  uint32_t cap = kHashCap;
  if (S.ovf) {  // scratch table: capacity >= 2n, (key, count) pairs
    cap = pow2_at_least(2 * n);
    tk = reinterpret_cast<uint32_t*>(scratch);
    tc = tk + cap;
    uint32_t lg = 31 - __clz(cap);
    for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
      tk[i] = kEmpty32;
      tc[i] = 0;
    }
    __syncthreads();
    for (uint32_t base = threadIdx.x & ~31u; base < n; base += blockDim.x) {
      uint32_t i = base + lane0;
      uint32_t key = i < n ? (uint32_t)(v[i] >> rbw) : kEmpty32;
      uint32_t peers = __match_any_sync(0xffffffffu, key);
      if (key == kEmpty32 || lane0 != __ffs(peers) - 1) continue;
      uint32_t add = __popc(peers);
      uint32_t h = (uint32_t)(((uint64_t)key * 0x9E3779B97F4A7C15ull) >> (64 - lg));
      for (uint32_t probe = 0; probe < cap; probe++) {
        uint32_t cur = tk[h];
        if (cur == kEmpty32) {
          uint32_t old = atomicCAS(&tk[h], kEmpty32, key);
          cur = old == kEmpty32 ? key : old;
        }
        if (cur == key) {
          atomicAdd(&tc[h], add);
          break;
        }
        h = (h + 1) & (cap - 1);
      }
    }
    __syncthreads();
  }
  // 8 rounds of block argmax over (count desc, key asc).
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) S.dl = 0;
  for (int r = 0; r < 8; r++) {
    uint64_t best = 0;  // (count << 32) | (0xFFFFFFFF - key); 0 = none
    uint32_t bslot = 0;
    for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) {
      uint32_t c = tc[i];
      if (c) {
        uint64_t kk = ((uint64_t)c << 32) | (uint64_t)(0xFFFFFFFFu - tk[i]);
        if (kk > best) {
          best = kk;
          bslot = i;
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      uint64_t ob = __shfl_xor_sync(0xffffffffu, best, o);
      uint32_t os = __shfl_xor_sync(0xffffffffu, bslot, o);
      if (ob > best) {
        best = ob;
        bslot = os;
      }
    }
    if (lane == 0) {
      S.red[warp] = best;
      S.red32[warp] = bslot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint64_t b = 0;
      uint32_t s = 0;
      for (int w = 0; w < kEncWarps; w++)
        if (S.red[w] > b) {
          b = S.red[w];
          s = S.red32[w];
        }
      if (b) {
        S.dict8[S.dl++] = tk[s];
        tc[s] = 0;
      }
    }
    __syncthreads();
  }
}

// Code (0..dl-1) of a left part, or -1 for an exception.
__device__ inline int rd_code(const EncSmem& S, uint64_t left) {
  int c = -1;
  for (uint32_t j = 0; j < S.dl; j++)
    if (S.dict8[j] == left && c < 0) c = (int)j;
  return c;
}

// ---------------------------------------------------------------------------
// DICT preparation (reference dict.rs:87-123): distinct values, the sorted
// dictionary and a value -> rank lookup.  Fast path: smem hash.  Fallback:
// scratch hash + scratch bitonic sort + binary-search ranks.  Sets S.card and
// S.flag (1 = dictionary bails: cardinality > n/2+1).
// ---------------------------------------------------------------------------
// Stable LSD radix sort (8-bit digits) of m u64 keys in a, using b as the
// second buffer; digits on which every key agrees are skipped.  Returns the
// buffer that holds the sorted keys.  All threads of a kEncThreads CTA; the
// per-warp digit counters live in the dictionary smem area.
__device__ uint64_t* block_radix_sort(EncSmem& S, uint64_t* a, uint64_t* b, uint32_t m) {
  static_assert(kEncThreads >= 256 && kEncWarps * 256 * 4 <= sizeof(S.big.dict.sorted),
                "one thread per digit in the offset scan; per-warp digit counters fit the dictionary area");
  // per-warp digit counters [kEncWarps][256] over the sorted-keys array of
  // the dictionary area (not in use here)
  uint32_t* hist = reinterpret_cast<uint32_t*>(S.big.dict.sorted);
  int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint64_t k0 = m ? a[0] : 0ull, diff = 0;
  for (uint32_t i0 = t; i0 < m; i0 += blockDim.x * 8) {
    uint64_t ks[8];
#pragma unroll
    for (int q = 0; q < 8; q++) ks[q] = i0 + q * blockDim.x < m ? a[i0 + q * blockDim.x] : k0;
#pragma unroll
    for (int q = 0; q < 8; q++) diff |= ks[q] ^ k0;
  }
  diff = warp_or64(diff);
  if (lane == 0) S.red[warp] = diff;
  __syncthreads();
  diff = 0;
  for (int w = 0; w < kEncWarps; w++) diff |= S.red[w];
  __syncthreads();
  uint32_t seg = ((m + kEncWarps - 1) / kEncWarps + 31u) & ~31u;
  uint32_t s0 = min(warp * seg, m), s1 = min(s0 + seg, m);
  for (int shift = 0; shift < 64; shift += 8) {
    if (((diff >> shift) & 0xFFull) == 0) continue;
    for (int i = t; i < kEncWarps * 256; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (uint32_t i0 = s0 + lane; i0 < s1; i0 += 32 * 8) {
      uint64_t ks[8];
#pragma unroll
      for (int q = 0; q < 8; q++) ks[q] = i0 + 32 * q < s1 ? a[i0 + 32 * q] : 0ull;
#pragma unroll
      for (int q = 0; q < 8; q++)
        if (i0 + 32 * q < s1) atomicAdd(&hist[warp * 256 + (uint32_t)((ks[q] >> shift) & 0xFF)], 1u);
    }
    __syncthreads();
    {  // offsets: digit-major, then warp order (stability); thread t < 256 owns digit t
      uint32_t tot = 0, inc = 0;
      if (t < 256) {
        for (int w = 0; w < kEncWarps; w++) tot += hist[w * 256 + t];
        inc = tot;
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += u;
        }
        if (lane == 31) S.red32[warp] = inc;
      }
      __syncthreads();
      if (t < 256) {
        uint32_t run = inc - tot;
        for (int w = 0; w < warp; w++) run += S.red32[w];
        for (int w = 0; w < kEncWarps; w++) {
          uint32_t c = hist[w * 256 + t];
          hist[w * 256 + t] = run;
          run += c;
        }
      }
    }
    __syncthreads();
    for (uint32_t base = s0; base < s1; base += 32 * 8) {
      uint64_t ks[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        uint32_t i = base + q * 32 + lane;
        ks[q] = i < s1 ? a[i] : 0ull;
      }
#pragma unroll
      for (int q = 0; q < 8; q++) {
        uint32_t i = base + q * 32 + lane;
        uint32_t act = __ballot_sync(0xffffffffu, i < s1);
        if (i < s1) {
          uint32_t dg = (uint32_t)((ks[q] >> shift) & 0xFF);
          uint32_t peers = __match_any_sync(act, dg);
          uint32_t r = __popc(peers & ((1u << lane) - 1u));
          b[hist[warp * 256 + dg] + r] = ks[q];
          __syncwarp(act);
          if (r == 0) hist[warp * 256 + dg] += __popc(peers);
        }
        __syncwarp();
      }
    }
    __syncthreads();
    uint64_t* tmp = a;
    a = b;
    b = tmp;
  }
  return a;
}

struct DictView {
  bool smem;
  const uint64_t* sorted;  // card values ascending
  uint32_t card;
  const uint64_t* tkey = nullptr;  // scratch hash table (keys) and ranks, 2^lg slots
  const uint32_t* trank = nullptr;
  uint32_t lg = 0;
};

__device__ inline uint32_t dict_hash_slot(const uint64_t* hk, uint64_t x) {
  uint32_t h = (uint32_t)((x * 0x9E3779B97F4A7C15ull) >> 53);
  for (uint32_t probe = 0; probe < kHashCap; probe++) {
    uint64_t cur = hk[h];
    if (cur == x || cur == kEmpty64) return h;
    h = (h + 1) & (kHashCap - 1);
  }
  return 0;
}

__device__ inline uint32_t dict_rank(const EncSmem& S, const DictView& dv, uint64_t x) {
  if (dv.smem) {
    if (x == kEmpty64) return S.max_rank;
    return S.big.dict.hval[dict_hash_slot(S.big.dict.hkey, x)];
  }
  if (x == kEmpty64) return S.max_rank;
  uint32_t cap = 1u << dv.lg;
  uint32_t h = (uint32_t)((x * 0x9E3779B97F4A7C15ull) >> (64 - dv.lg));
  for (uint32_t probe = 0; probe < cap && dv.tkey[h] != x; probe++) h = (h + 1) & (cap - 1);
  return dv.trank[h];
}

// Insert x into the smem hash (no-op once the table has overflowed).
__device__ __forceinline__ void dict_insert(DictArea& D, EncSmem& S, uint64_t x) {
  if (*(volatile uint32_t*)&S.ovf) return;
  if (x == kEmpty64) {
    if (atomicExch(&S.has_max, 1u) == 0) atomicAdd(&S.card, 1u);
    return;
  }
  uint32_t h = (uint32_t)((x * 0x9E3779B97F4A7C15ull) >> 53);
  for (uint32_t probe = 0; probe < kHashCap; probe++) {
    uint64_t cur = D.hkey[h];
    if (cur == kEmpty64) {
      unsigned long long old = atomicCAS((unsigned long long*)&D.hkey[h], kEmpty64, x);
      if (old == kEmpty64) {
        if (atomicAdd(&S.card, 1u) >= kHashLimit) S.ovf = 1;
        return;
      }
      cur = old;
    }
    if (cur == x) return;
    h = (h + 1) & (kHashCap - 1);
  }
  S.ovf = 1;
}

// lb_pre: the block's 17-bit bucket count when the statistics pass computed it
// (block == one adaptive window), else kNoLb.
__device__ DictView dict_prepare(EncSmem& S, const uint64_t* v, uint32_t n, uint8_t* scratch, uint32_t lb_pre) {
  DictArea& D = S.big.dict;
  uint32_t max_card = n / 2 + 1;
  bool have_lb = lb_pre != kNoLb;
  if (have_lb && lb_pre > max_card) {  // the lower bound alone proves the bail
    if (threadIdx.x == 0) S.flag = 1;
    __syncthreads();
    DictView dv;
    dv.smem = false;
    dv.sorted = nullptr;
    dv.card = lb_pre;
    return dv;
  }
  for (uint32_t i = threadIdx.x; i < kHashCap; i += blockDim.x) {
    D.hkey[i] = kEmpty64;
    D.hval[i] = 0;
  }
  if (threadIdx.x == 0) {
    S.ovf = 0;
    S.card = 0;
    S.has_max = 0;
    S.flag = 0;
  }
  __syncthreads();
  // the shared-memory hash until it holds kHashLimit keys; the lower-bound
  // bitset is only built (below) for a block that overflows it
  for (uint32_t base = 0; base < n; base += blockDim.x * 8) {
    if (*(volatile uint32_t*)&S.ovf) break;
    uint64_t xs[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint32_t iq = base + q * blockDim.x + threadIdx.x;
      xs[q] = iq < n ? v[iq] : 0ull;
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
      if (base + q * blockDim.x + threadIdx.x < n) dict_insert(D, S, xs[q]);
  }
  __syncthreads();
  DictView dv;
  if (!S.ovf) {
    uint32_t card = S.card;
    if (card > max_card) {
      if (threadIdx.x == 0) S.flag = 1;
      __syncthreads();
      dv.smem = true;
      dv.sorted = nullptr;
      dv.card = card;
      return dv;
    }
    if (threadIdx.x == 0) S.cnt32 = 0;
    __syncthreads();
    uint32_t P = pow2_at_least(max(card, 1u));
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) D.sorted[i] = kEmpty64;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kHashCap; i += blockDim.x)
      if (D.hkey[i] != kEmpty64) D.sorted[atomicAdd(&S.cnt32, 1u)] = D.hkey[i];
    __syncthreads();
    block_bitonic_sort(D.sorted, P);
    for (uint32_t r = threadIdx.x; r < card; r += blockDim.x) {
      uint64_t x = D.sorted[r];
      if (x == kEmpty64) S.max_rank = r;
      else D.hval[dict_hash_slot(D.hkey, x)] = r;
    }
    __syncthreads();
    dv.smem = true;
    dv.sorted = D.sorted;
    dv.card = card;
    return dv;
  }
  // Overflow: a lower bound on the cardinality may prove the bail outright:
  // the window's 17-bit bucket count when the statistics pass computed it,
  // and, when that does not prove it, the distinct buckets of a 2^20-bit set
  // (fewer for a short block) built in the block's scratch range with
  // fire-and-forget atomics, whose collisions stay few at any cardinality
  // near the bail threshold.
  {
    uint32_t lb = have_lb ? lb_pre : 0u;
    if (lb <= max_card) {
      uint32_t lgb = 20;
      while (lgb > 10 && (1ull << (lgb - 3)) > (uint64_t)n * kEncScratchPerValue) lgb--;
      const uint32_t words = (1u << lgb) / 32;
      uint32_t* bits = reinterpret_cast<uint32_t*>(scratch);
      for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) bits[i] = 0;
      __syncthreads();
      for (uint32_t base = 0; base < n; base += blockDim.x * 8) {
        uint64_t xs[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
          uint32_t iq = base + q * blockDim.x + threadIdx.x;
          xs[q] = iq < n ? v[iq] : 0ull;
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          if (base + q * blockDim.x + threadIdx.x < n) {
            uint32_t h = (uint32_t)((xs[q] * 0xD6E8FEB86659FD93ull) >> (64 - lgb));
            atomicOr(&bits[h >> 5], 1u << (h & 31));
          }
        }
      }
      __syncthreads();
      uint32_t c = 0;
      for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) c += __popc(bits[i]);
      c = warp_sum(c);
      if ((threadIdx.x & 31) == 0) S.red32[threadIdx.x >> 5] = c;
      __syncthreads();
      uint32_t t = 0;
      for (int w = 0; w < kEncWarps; w++) t += S.red32[w];
      lb = t > lb ? t : lb;
    }
    __syncthreads();
    if (threadIdx.x == 0) S.cnt32 = lb;
    __syncthreads();
  }
  if (S.cnt32 > max_card) {
    if (threadIdx.x == 0) S.flag = 1;
    __syncthreads();
    dv.smem = false;
    dv.sorted = nullptr;
    dv.card = S.cnt32;
    return dv;
  }
  // Scratch path (more than kHashLimit distinct values): a u64 key hash table
  // T[cap] in scratch (cap = pow2 >= n, so the table stays at most about half
  // full for a dictionary that does not bail), the distinct keys compacted and
  // radix-sorted, and a rank table R[cap] beside T for the code lookups.
  // Scratch use: 12*cap + 16*max_card bytes <= 32*n.
  uint32_t cap = pow2_at_least(n), lg = 31 - __clz(cap);
  uint64_t* T = reinterpret_cast<uint64_t*>(scratch);
  uint32_t* R = reinterpret_cast<uint32_t*>(scratch + 8ull * cap);
  uint64_t* A = reinterpret_cast<uint64_t*>(scratch + 12ull * cap);
  uint64_t* B = A + max_card;
  for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x) T[i] = kEmpty64;
  if (threadIdx.x == 0) {
    S.card = 0;
    S.cnt32 = 0;
    S.has_max = 0;
    S.flag = 0;
  }
  __syncthreads();
  for (uint32_t base = 0; base < n; base += blockDim.x * 8) {
    if (__any_sync(0xffffffffu, *(volatile uint32_t*)&S.flag)) break;  // warp-uniform exit
    uint64_t xs[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint32_t iq = base + q * blockDim.x + threadIdx.x;
      xs[q] = iq < n ? v[iq] : 0ull;
    }
    // first probes of the eight values in flight together, then the CASes
    uint32_t hs[8];
    uint64_t cur0[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      hs[q] = (uint32_t)((xs[q] * 0x9E3779B97F4A7C15ull) >> (64 - lg));
      cur0[q] = base + q * blockDim.x + threadIdx.x < n ? T[hs[q]] : 0ull;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      if (base + q * blockDim.x + threadIdx.x < n && xs[q] != kEmpty64 && cur0[q] == kEmpty64)
        cur0[q] = atomicCAS((unsigned long long*)&T[hs[q]], kEmpty64, xs[q]);
      else
        cur0[q] = cur0[q] == kEmpty64 ? 1ull : cur0[q];  // (not used: 1 never equals kEmpty64)
    }
    uint32_t mine = 0;  // distinct keys this lane added (counted once per warp below)
#pragma unroll
    for (int q = 0; q < 8; q++) {
      if (base + q * blockDim.x + threadIdx.x >= n) continue;
      uint64_t x = xs[q];
      if (x == kEmpty64) {
        if (atomicExch(&S.has_max, 1u) == 0) mine++;
        continue;
      }
      if (cur0[q] == kEmpty64) {  // the first-probe CAS inserted x
        mine++;
        continue;
      }
      if (cur0[q] == x) continue;
      uint32_t h = (hs[q] + 1) & (cap - 1);
      for (uint32_t probe = 1; probe < cap; probe++) {
        uint64_t cur = T[h];
        if (cur == kEmpty64) {
          cur = atomicCAS((unsigned long long*)&T[h], kEmpty64, x);
          if (cur == kEmpty64) {
            mine++;
            break;
          }
        }
        if (cur == x) break;
        h = (h + 1) & (cap - 1);
      }
    }
    mine = warp_sum(mine);
    if ((threadIdx.x & 31) == 0 && mine && atomicAdd(&S.card, mine) + mine > max_card) S.flag = 1;
  }
  __syncthreads();
  dv.smem = false;
  dv.tkey = T;
  dv.trank = R;
  dv.lg = lg;
  if (S.flag) {  // cardinality > n/2 + 1
    dv.card = S.card;
    dv.sorted = nullptr;
    return dv;
  }
  uint32_t card = S.card, has_max = S.has_max;
  for (uint32_t i0 = threadIdx.x; i0 < cap; i0 += blockDim.x * 8) {
    uint64_t ks[8];
#pragma unroll
    for (int q = 0; q < 8; q++) ks[q] = i0 + q * blockDim.x < cap ? T[i0 + q * blockDim.x] : kEmpty64;
#pragma unroll
    for (int q = 0; q < 8; q++) {  // one counter update per warp and step
      bool ok = ks[q] != kEmpty64;
      uint32_t m = __ballot_sync(0xffffffffu, ok);
      uint32_t base_i = 0;
      if ((threadIdx.x & 31) == 0 && m) base_i = atomicAdd(&S.cnt32, (uint32_t)__popc(m));
      base_i = __shfl_sync(0xffffffffu, base_i, 0);
      if (ok) A[base_i + __popc(m & ((1u << (threadIdx.x & 31)) - 1u))] = ks[q];
    }
  }
  __syncthreads();
  uint64_t* srt = block_radix_sort(S, A, B, card - has_max);
  if (has_max && threadIdx.x == 0) srt[card - 1] = kEmpty64;
  if (threadIdx.x == 0) S.max_rank = card - 1;
  __syncthreads();
  for (uint32_t r0 = threadIdx.x; r0 + has_max < card; r0 += blockDim.x * 8) {
    uint64_t xs[8];
    uint32_t hs[8];
    uint64_t cur[8];
#pragma unroll
    for (int q = 0; q < 8; q++) xs[q] = r0 + q * blockDim.x + has_max < card ? srt[r0 + q * blockDim.x] : 0ull;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      hs[q] = (uint32_t)((xs[q] * 0x9E3779B97F4A7C15ull) >> (64 - lg));
      cur[q] = r0 + q * blockDim.x + has_max < card ? T[hs[q]] : 0ull;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint32_t r = r0 + q * blockDim.x;
      if (r + has_max >= card) break;
      uint32_t h = hs[q];
      if (cur[q] != xs[q]) {
        h = (h + 1) & (cap - 1);
        for (uint32_t probe = 1; probe < cap && T[h] != xs[q]; probe++) h = (h + 1) & (cap - 1);
      }
      R[h] = r;
    }
  }
  __syncthreads();
  dv.card = card;
  dv.sorted = srt;
  return dv;
}

// Byte length of the dictionary value blob and its tag (reference dict.rs:40-61).
__device__ uint64_t dict_values_len(EncSmem& S, const DictView& dv, uint32_t* tag) {
  const uint64_t* s = dv.sorted;
  uint64_t raw = 8ull * dv.card;
  uint64_t delta = 8 + block_for(S, nullptr, dv.card, false, [&](uint32_t i) {
                     return zigzag64(s[i] - (i ? s[i - 1] : s[0]));
                   });
  if (delta < raw) {
    *tag = 1;
    return delta;
  }
  *tag = 0;
  return raw;
}

// ---------------------------------------------------------------------------
// RLE run starts (reference rle.rs:10-42).  Requires S.neq_k (transitions per
// sub-block).  Returns the starts array (smem or scratch).
// ---------------------------------------------------------------------------
__device__ uint32_t* rle_starts(EncSmem& S, const uint64_t* v, uint32_t n, uint32_t runs, uint8_t* scratch) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* st = runs <= kRunsSmem ? S.big.rle.starts : reinterpret_cast<uint32_t*>(scratch);
  uint32_t nsub = (n + kSub - 1) / kSub;
  if (threadIdx.x == 0) {  // exclusive prefix of transitions per sub-block
    uint32_t acc = 0;
    for (uint32_t k = 0; k < nsub; k++) {
      uint32_t c = S.neq_k[k];
      S.subsz[k] = acc;
      acc += c;
    }
    st[0] = 0;
  }
  __syncthreads();
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
    uint64_t carry = base ? v[base - 1] : v[0];
    uint32_t before = S.subsz[k];
    for (uint32_t j0 = 0; j0 < 32; j0 += 8) {
     uint64_t xs[8];
#pragma unroll
     for (int q = 0; q < 8; q++) {
       uint32_t lq = (j0 + q) * 32 + lane;
       xs[q] = lq < cnt ? v[base + lq] : 0ull;
     }
#pragma unroll
     for (int q = 0; q < 8; q++) {
      uint32_t j = j0 + q;
      uint32_t li = j * 32 + lane;
      bool ok = li < cnt;
      uint32_t idx = base + li;
      uint64_t x = xs[q];
      uint64_t up = __shfl_up_sync(0xffffffffu, x, 1);
      uint64_t pv = lane ? up : carry;
      carry = __shfl_sync(0xffffffffu, x, 31);
      bool tr = ok && idx && x != pv;
      uint32_t m = __ballot_sync(0xffffffffu, tr);
      if (tr) st[1 + before + __popc(m & ((1u << lane) - 1u))] = idx;
      before += __popc(m);
     }
    }
  }
  __syncthreads();
  return st;
}

// ---------------------------------------------------------------------------
// Entropy stage of the Balanced candidate pool (reference entropy/rans.rs:25-108
// behind the rANS tag of entropy/mod.rs:49-60): static 12-bit frequencies,
// four interleaved states sharing one byte stream, L = 2^23.  A coded part is
// [2][varint(m)][varint(symbols)][(symbol, varint(freq))...][4 x u32 states]
// [bytes].  The encoder runs backward over the input and its state chains
// are sequential, so thread 0 runs them while the other warps stage the next
// 4096 input bytes in shared memory.
// ---------------------------------------------------------------------------
constexpr uint32_t kRansM = 4096, kRansL = 1u << 23;

// Histogram of byte_at(0 .. m) and the normalised frequencies (rans.rs:25-48:
// f = max(1, c * 4096 / m); while the sum exceeds 4096 the largest f > 1 loses
// one, ties to the highest symbol; a short sum goes to the largest f, ties to
// the highest symbol).  Returns the header length after the tag byte.
template <class B>
__device__ uint32_t rans_plan(RansArea& R, uint32_t m, B byte_at) {
  int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int i = t; i < 256; i += blockDim.x) R.hist[i] = 0;
  __syncthreads();
  for (uint32_t base = (uint32_t)warp * 32; base < m; base += blockDim.x) {
    uint32_t i = base + lane;
    uint32_t sym = i < m ? (uint32_t)byte_at(i) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, sym);
    if (sym < 256 && lane == __ffs(peers) - 1) atomicAdd(&R.hist[sym], (uint32_t)__popc(peers));
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t f[8], sum = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      uint32_t c = R.hist[lane + 32 * j];
      uint32_t q = (uint32_t)(((uint64_t)c * kRansM) / m);
      f[j] = c ? (q ? q : 1u) : 0u;
      sum += f[j];
    }
    sum = warp_sum(sum);
    while (sum > kRansM) {
      uint32_t key = 0;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if (f[j] > 1) key = max(key, (f[j] << 8) | (uint32_t)(lane + 32 * j));
      key = warp_max(key);
      uint32_t sym = key & 255u;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if ((uint32_t)(lane + 32 * j) == sym) f[j]--;
      sum--;
    }
    if (sum < kRansM) {
      uint32_t key = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) key = max(key, (f[j] << 8) | (uint32_t)(lane + 32 * j));
      key = warp_max(key);
      uint32_t sym = key & 255u;
#pragma unroll
      for (int j = 0; j < 8; j++)
        if ((uint32_t)(lane + 32 * j) == sym) f[j] += kRansM - sum;
    }
#pragma unroll
    for (int j = 0; j < 8; j++) R.fc[lane + 32 * j].x = f[j];
    // A lower bound on the coded bytes: any static model codes the sequence
    // in at least its empirical entropy (Gibbs), and a byte-renormalising
    // four-state coder emits at most 32 bits less (the states' growth from
    // 2^23 to below 2^31) and loses under 2^-11 bits a symbol to the state
    // rounding; a margin of 64 bits covers the floating-point sum.
    double e = 0.0;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      uint32_t c = R.hist[lane + 32 * j];
      if (c) e += (double)c * log2((double)m / (double)c);
    }
    for (int o = 16; o; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    double bits = e * (1.0 - 1e-9) - 0.001 * (double)m - 96.0;
    __syncwarp();
    if (lane == 0) {
      R.bound = bits > 0.0 ? (uint32_t)(bits / 8.0) : 0u;
      uint32_t c = 0, present = 0, h = 0;
      for (int sym = 0; sym < 256; sym++) {
        uint32_t fs = R.fc[sym].x;
        R.fc[sym].y = c;
        c += fs;
        if (fs) {
          present++;
          h += 1 + varint_len(fs);
        }
      }
      R.hdr = varint_len(m) + varint_len(present) + h;
    }
  }
  __syncthreads();
  uint32_t hdr = R.hdr;
  __syncthreads();
  return hdr;
}

// Header of a coded part (after its tag byte), from the planned frequencies.
__device__ void rans_put_header(const RansArea& R, uint32_t m, uint8_t* out) {
  uint32_t present = 0;
  for (int sym = 0; sym < 256; sym++) present += R.fc[sym].x ? 1u : 0u;
  uint32_t pos = put_varint(out, m);
  pos += put_varint(out + pos, present);
  for (int sym = 0; sym < 256; sym++)
    if (R.fc[sym].x) {
      out[pos++] = (uint8_t)sym;
      pos += put_varint(out + pos, R.fc[sym].x);
    }
}

// Renormalisation of one state before coding a symbol of frequency f: bytes
// leave from the low end while x >= f * 2^19 ((L >> 12) << 8 = 2^19).
// (f >= 1 for every symbol the histogram saw; the max keeps the loop finite
// whatever the input.)
template <bool WRITE>
__device__ __forceinline__ void rans_renorm(uint32_t& x, uint32_t f, uint32_t& e, uint8_t*& p) {
  uint32_t xm = max(f, 1u) << 19;
  while (x >= xm) {
    if (WRITE) *--p = (uint8_t)x;
    x >>= 8;
    e++;
  }
}
__device__ __forceinline__ uint32_t rans_code(uint32_t x, uint2 fc) {
  uint32_t f = max(fc.x, 1u);
  return ((x / f) << 12) + (x % f) + fc.y;
}

// Destination of a bit-packed stream of `len` bytes that a block stages for
// rANS: its scratch range (32 B per value) when it fits, else the shared
// big area, free once the ALP-RD dictionary is in S.dict8 (a sub-block pads
// to 1024 values, so a block of fewer than 257 values can exceed its range;
// such a stream is at most varint(n) + 9 + 128 * 64 bytes).
__device__ __forceinline__ uint8_t* stage_dst(EncSmem& S, uint8_t* scr, uint32_t n, uint64_t len) {
  return len <= 32ull * n ? scr : reinterpret_cast<uint8_t*>(&S.big);
}
static_assert(sizeof(BigArea) >= 3 + 9 + 128 * 64, "staged bit-packed stream of a short block");

// The encoder pass over byte_at(m - 1 .. 0) with the planned frequencies.
// Returns the number of stream bytes; WRITE stores them ending at `wend` and
// the four final states in the 16 bytes before the first of them.
template <bool WRITE, class B>
__device__ uint32_t rans_run(RansArea& R, uint32_t m, B byte_at, uint8_t* wend) {
  int t = threadIdx.x, warp = t >> 5;
  uint32_t nch = (m + kRansChunk - 1) / kRansChunk;
  auto fill = [&](uint32_t c, int slot) {  // warps 1.. stage chunk c
    uint32_t lo = c * kRansChunk, hi = min(lo + kRansChunk, m);
    for (uint32_t i = lo + (uint32_t)(t - 32); i < hi; i += blockDim.x - 32) R.buf[slot][i - lo] = (uint8_t)byte_at(i);
  };
  if (warp && nch) fill(nch - 1, 0);
  __syncthreads();
  uint32_t x0 = kRansL, x1 = kRansL, x2 = kRansL, x3 = kRansL, e = 0;
  uint8_t* p = wend;
  for (uint32_t k = 0; k < nch; k++) {
    uint32_t c = nch - 1 - k;
    if (warp && c > 0) fill(c - 1, (int)((k + 1) & 1));
    if (t == 0) {
      const uint8_t* bb = R.buf[k & 1];
      uint32_t lo = c * kRansChunk, i = min(lo + kRansChunk, m);
      while (i > lo && (i & 3)) {  // the top of the input, one step at a time
        i--;
        uint2 fc = R.fc[bb[i - lo]];
        uint32_t& x = (i & 3) == 3 ? x3 : (i & 3) == 2 ? x2 : (i & 3) == 1 ? x1 : x0;
        rans_renorm<WRITE>(x, fc.x, e, p);
        x = rans_code(x, fc);
      }
      while (i > lo) {  // steps i-1 .. i-4 code with states 3, 2, 1, 0
        i -= 4;
        uint2 f3 = R.fc[bb[i + 3 - lo]], f2 = R.fc[bb[i + 2 - lo]], f1 = R.fc[bb[i + 1 - lo]],
              f0 = R.fc[bb[i - lo]];
        rans_renorm<WRITE>(x3, f3.x, e, p);
        rans_renorm<WRITE>(x2, f2.x, e, p);
        rans_renorm<WRITE>(x1, f1.x, e, p);
        rans_renorm<WRITE>(x0, f0.x, e, p);
        x3 = rans_code(x3, f3);
        x2 = rans_code(x2, f2);
        x1 = rans_code(x1, f1);
        x0 = rans_code(x0, f0);
      }
    }
    __syncthreads();
  }
  if (t == 0) {
    if (WRITE) {
      put_u32(p - 16, x0);
      put_u32(p - 12, x1);
      put_u32(p - 8, x2);
      put_u32(p - 4, x3);
    }
    R.emitted = e;
  }
  __syncthreads();
  uint32_t r = R.emitted;
  __syncthreads();
  return r;
}

// Length of code_residuals(byte_at(0 .. m)) with the rANS tag: the coded part
// entropy_pick keeps at lambda >= 2 (m > 0).
template <class B>
// Callers only ask whether the length is below `limit`: when the entropy
// bound already reaches it, the serial sizing pass is skipped and a length at
// or above the limit (the bound) comes back.
__device__ uint32_t coded_len(RansArea& R, uint32_t m, B byte_at, uint64_t limit = ~0ull) {
  uint32_t h = rans_plan(R, m, byte_at);
  uint32_t lo = 1 + h + 16 + R.bound;  // uniform: R is read after rans_plan's barrier
  if ((uint64_t)lo >= limit) return lo;
  return 1 + h + 16 + rans_run<false>(R, m, byte_at, nullptr);
}

// Writes the coded part of byte_at(0 .. m) whose length (tag included) is len.
template <class B>
__device__ void coded_write(RansArea& R, uint32_t m, B byte_at, uint8_t* out, uint32_t len) {
  rans_plan(R, m, byte_at);
  if (threadIdx.x == 0) {
    out[0] = 2;
    rans_put_header(R, m, out + 1);
  }
  rans_run<true>(R, m, byte_at, out + len);
}

// FLOAT_MULT's entropy form (float_mult.rs:66-98): LEB128(zigzag(k_i - k_{i-1}))
// with k_{-1} = 0, written to dst; returns the byte count.  Thread t writes a
// contiguous run of values at offsets from a block scan of their lengths.
__device__ uint32_t fm_delta_bytes(EncSmem& S, const uint64_t* v, uint32_t n, int sc, uint8_t* dst) {
  int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint32_t seg = (n + blockDim.x - 1) / blockDim.x;
  uint32_t i0 = min((uint32_t)t * seg, n), i1 = min(i0 + seg, n);
  uint32_t len = 0;
  int64_t prev = i0 ? fm_k(v[i0 - 1], sc) : 0;
  for (uint32_t i = i0; i < i1; i++) {
    int64_t k = fm_k(v[i], sc);
    len += varint_len(zigzag64((uint64_t)k - (uint64_t)prev));
    prev = k;
  }
  uint32_t inc = warp_incl_scan(len);
  if (lane == 31) S.red32[warp] = inc;
  __syncthreads();
  uint32_t off = inc - len, tot = 0;
  for (int w = 0; w < kEncWarps; w++) {
    if (w < warp) off += S.red32[w];
    tot += S.red32[w];
  }
  prev = i0 ? fm_k(v[i0 - 1], sc) : 0;
  for (uint32_t i = i0; i < i1; i++) {
    int64_t k = fm_k(v[i], sc);
    off += put_varint(dst + off, zigzag64((uint64_t)k - (uint64_t)prev));
    prev = k;
  }
  __syncthreads();
  return tot;
}

// The entropy parts chosen for a block (Balanced in-pool), read by k_emit.
// Lengths include the rANS tag byte.
constexpr uint32_t kEntFm = 1, kEntRdCodes = 2, kEntRdRights = 4, kEntDictVals = 8, kEntDictCodes = 16;
struct EntRec {
  uint32_t flags;
  uint32_t fm;      // FLOAT_MULT coded deltas
  uint32_t rdc;     // ALP-RD coded codes
  uint32_t rdr;     // ALP-RD coded rights (the bit-packed rights bytes)
  uint32_t bt;      // BYTE_TRANSPOSE payload
  uint32_t dv;      // DICT coded transposed values
  uint32_t dc[2];   // DICT coded code planes
};
static_assert(sizeof(EntRec) == 32, "EntRec layout");

struct Cand {
  uint64_t len;
  bool ok;
};

// ---------------------------------------------------------------------------
// Competition, part 1: per-sub-block statistics.  One warp per 1024-value
// sub-block, one pass over the lane.  Quantities that depend on whether the
// sub-block opens a block (its first value's delta / XOR / equality with the
// previous value) are kept out of the internal sums and folded in by k_decide,
// so the statistics are computed before the block plan exists.
// ---------------------------------------------------------------------------
struct SubStats {
  uint64_t umin, umax, first, last, d;  // d = v[1] - v[0] of the sub-block
  int64_t smin, smax;
  uint64_t dzmin, dzmax;                // zigzag deltas of internal pairs (j >= 1)
  uint64_t e16min, e16max, e16dz;       // early-out samples j % 16 == 0
  uint64_t e64min, e64max, e64dz;       // early-out samples j % 64 == 0
  uint32_t xb, neq, cnt;                // internal XORZ bytes, internal transitions, values
  uint8_t stride_ok, alp_ok, alp_w, fm_pass;
  uint16_t alp_exc, pad16;
  uint32_t pad32;
};
static_assert(sizeof(SubStats) == 144, "SubStats layout");
struct FmStat {  // signed min / max of k = round(x * scale) per FLOAT_MULT scale
  int64_t kmin[7], kmax[7];
};

constexpr int kStatsWarps = 32;  // one CTA per 32768-value window in adaptive mode

// Start and length of statistics item `item` (one 1024-value sub-block): with
// a fixed block size the sub-blocks restart at every block boundary.
__device__ inline uint32_t sub_range(uint64_t item, uint64_t n, uint64_t fixed_bs, uint64_t* s) {
  if (fixed_bs) {
    uint64_t spb = (fixed_bs + kSub - 1) / kSub;
    uint64_t b = item / spb, k = item % spb;
    uint64_t bstart = b * fixed_bs, bend = qmin(bstart + fixed_bs, n);
    *s = bstart + k * kSub;
    return (bstart < n && *s < bend) ? (uint32_t)qmin(kSub, bend - *s) : 0u;
  }
  *s = item * kSub;
  return *s < n ? (uint32_t)qmin(kSub, n - *s) : 0u;
}

// ALP statistics of every sub-block (alp.rs:49-166), for float lanes at Fast
// and above: one warp per sub-block, after k_sub_stats (whose records it
// completes).  The power-of-ten tables are copied to shared memory, since the
// (e, f) search reads them at a different index in every lane.
constexpr int kAlpWarps = 8;
constexpr uint16_t kAlpEfKnown = 0x8000;  // SubStats::pad16 holds e | f << 8 of a sub-block that passed
__global__ void __launch_bounds__(kAlpWarps * 32) k_alp_stats(const uint64_t* __restrict__ v, uint64_t n,
                                                              uint64_t fixed_bs, uint64_t items,
                                                              SubStats* __restrict__ ss) {
  __shared__ uint64_t smp[kAlpWarps][32];
  __shared__ double pexp[19], pfrac[19];
  if (threadIdx.x < 19) {
    pexp[threadIdx.x] = kExp10[threadIdx.x];
    pfrac[threadIdx.x] = kFrac10[threadIdx.x];
  }
  __syncthreads();
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t item = (uint64_t)blockIdx.x * kAlpWarps + warp;
  if (item >= items) return;
  uint64_t s;
  uint32_t cnt = sub_range(item, n, fixed_bs, &s);
  if (!cnt) return;
  AlpSub a;
  bool ok = alp_subblock(v + s, cnt, smp[warp], pexp, pfrac, &a);
  if (lane == 0) {
    ss[item].alp_ok = ok ? 1 : 0;
    ss[item].alp_w = ok ? (uint8_t)a.w : 0;
    ss[item].alp_exc = ok ? (uint16_t)a.exc : 0;
    ss[item].pad16 = ok ? (uint16_t)(kAlpEfKnown | a.e | (a.f << 8)) : 0;  // the emitter reuses (e, f)
  }
}

template <bool FLOATS>
__global__ void __launch_bounds__(kStatsWarps * 32) k_sub_stats(
    const uint64_t* __restrict__ v, uint64_t n, uint64_t fixed_bs, int dtype, int level,
    SubStats* __restrict__ ss, FmStat* __restrict__ fms, uint64_t* __restrict__ smp16, uint8_t* __restrict__ grow,
    uint32_t* __restrict__ winbits) {
  __shared__ uint32_t bitsA[512], bitsB[512];
  __shared__ uint32_t lbits[kLbBits / 32];  // dictionary cardinality lower bound (window)
  __shared__ uint32_t s_lbc;
  __shared__ uint64_t s_first[kStatsWarps], s_last[kStatsWarps];
  __shared__ uint32_t s_neq[kStatsWarps], s_cnt[kStatsWarps];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool do_float = FLOATS && level >= 1;
  uint64_t item = (uint64_t)blockIdx.x * kStatsWarps + warp;
  uint64_t s;
  uint32_t cnt = sub_range(item, n, fixed_bs, &s);
  // window probe sampling (adaptive): window-relative stride max(len/4096, 1)
  uint64_t wstart = (uint64_t)blockIdx.x * kBaseQuantum;
  uint32_t wlen = fixed_bs ? 0u : (uint32_t)(wstart < n ? qmin(kBaseQuantum, n - wstart) : 0);
  uint32_t wstride = max(wlen / 4096u, 1u);
  const bool sgn = dtype_signed(dtype);
  if (!fixed_bs) {
    for (int i = threadIdx.x; i < 512; i += blockDim.x) {
      bitsA[i] = 0;
      bitsB[i] = 0;
    }
    for (int i = threadIdx.x; i < (int)(kLbBits / 32); i += blockDim.x) lbits[i] = 0;
    if (threadIdx.x == 0) s_lbc = 0;
    __syncthreads();
  }
  SubStats R;
  uint64_t umn = kEmpty64, umx = 0, dzmn = kEmpty64, dzmx = 0;
  int64_t smn = INT64_MAX, smx = INT64_MIN;
  uint64_t a16mn = kEmpty64, a16mx = 0, a16dz = 0, a64mn = kEmpty64, a64mx = 0, a64dz = 0;
  uint32_t nq = 0, xb = 0, fmfail = 0;
  int64_t kmn[7], kmx[7];
#pragma unroll
  for (int q = 0; q < 7; q++) {
    kmn[q] = INT64_MAX;
    kmx[q] = INT64_MIN;
  }
  const uint64_t* sv = v + s;
  uint64_t d = cnt >= 2 ? sv[1] - sv[0] : 0;
  uint32_t alive = do_float ? 0x7Fu : 0u;
  uint64_t carry = 0;
  for (uint32_t r0 = 0; r0 < 32; r0 += 8) {
    uint64_t xs[8];  // eight independent loads in flight per lane
#pragma unroll
    for (int q = 0; q < 8; q++) {
      uint32_t jq = (r0 + q) * 32 + lane;
      xs[q] = jq < cnt ? sv[jq] : 0ull;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
    uint32_t r = r0 + q;
    uint32_t j = r * 32 + lane;
    bool ok = j < cnt;
    uint64_t x = xs[q];
    // one rotation gives every lane its predecessor; lane 0's is the previous
    // row's last value, which the rotation hands it for the next row
    uint64_t rot = __shfl_sync(0xffffffffu, x, (lane + 31) & 31);
    uint64_t pv = lane ? rot : carry;
    carry = rot;
    if (ok) {
      umn = u64min(umn, x);
      umx = u64max(umx, x);
      if (sgn) {
        int64_t sx = (int64_t)x;
        smn = sx < smn ? sx : smn;
        smx = sx > smx ? sx : smx;
      }
      if (j > 0) {
        uint64_t dz = zigzag64(x - pv);
        dzmn = u64min(dzmn, dz);
        dzmx = u64max(dzmx, dz);
        xb += varint_len(x ^ pv);
        nq += x != pv ? 1u : 0u;
      }
      if (!fixed_bs) {
        if (j == 0 || x != pv) {  // a repeat's bucket is already set
          uint32_t lb17 = dict_lb_bucket(x);
          atomicOr(&lbits[lb17 >> 5], 1u << (lb17 & 31));
        }
      }
      if (FLOATS && alive) {
        double xd = as_f64(x);
        uint32_t a2 = alive;
        while (a2) {
          int q = __ffs(a2) - 1;
          a2 &= a2 - 1;
          double sc = kFmScales[q];
          double k = round_half_away(__dmul_rn(xd, sc));
          bool good = is_finite_f64(k) && fabs(k) < 9.0e18 && f64_bits(__ddiv_rn(k, sc)) == x;
          if (!good) {
            fmfail |= 1u << q;
          } else {
            int64_t ki = __double2ll_rz(k);
            kmn[q] = ki < kmn[q] ? ki : kmn[q];
            kmx[q] = ki > kmx[q] ? ki : kmx[q];
          }
        }
      }
    }
    // a scale that failed anywhere in the sub-block is out: stop trying it
    if (FLOATS && alive) alive &= ~warp_or(fmfail);
    }
  }
  // Sampled statistics, kept out of the per-value loop (only a few lanes of a
  // row would take them): early-out samples at j % 16 / j % 64 == 0 and the
  // window probe samples (stride wstride, and stride 32).
  for (uint32_t j = 16u * lane; j < cnt; j += 512) {
    uint64_t x = sv[j], pv = j ? sv[j - 1] : 0ull;
    a16mn = u64min(a16mn, x);
    a16mx = u64max(a16mx, x);
    if (j > 0) a16dz = u64max(a16dz, zigzag64(x - pv));
    if (smp16 && !fixed_bs) smp16[(s + j) >> 4] = x;
    if ((j & 63) == 0) {
      a64mn = u64min(a64mn, x);
      a64mx = u64max(a64mx, x);
      if (j > 0) a64dz = u64max(a64dz, zigzag64(x - pv));
    }
  }
  if (!fixed_bs && cnt) {
    uint32_t off = (uint32_t)(s - wstart) % wstride;
    for (uint32_t j = (off ? wstride - off : 0u) + wstride * lane; j < cnt; j += wstride * 32) {
      uint32_t bk = (uint32_t)(((sv[j] * 0x9E3779B97F4A7C15ull) >> 50) & 0x3FFF);
      atomicOr(&bitsA[bk >> 5], 1u << (bk & 31));
    }
    uint32_t jb = 32u * lane;  // window offset of the sub-block is a multiple of 1024
    if (jb < cnt) {
      uint32_t bk = (uint32_t)(((sv[jb] * 0x9E3779B97F4A7C15ull) >> 50) & 0x3FFF);
      atomicOr(&bitsB[bk >> 5], 1u << (bk & 31));
    }
  }
  R.umin = warp_min(umn);
  R.umax = warp_max(umx);
  R.smin = warp_min_i64(smn);
  R.smax = warp_max_i64(smx);
  R.dzmin = warp_min(dzmn);
  R.dzmax = warp_max(dzmx);
  R.e16min = warp_min(a16mn);
  R.e16max = warp_max(a16mx);
  R.e16dz = warp_max(a16dz);
  R.e64min = warp_min(a64mn);
  R.e64max = warp_max(a64mx);
  R.e64dz = warp_max(a64dz);
  R.xb = warp_sum(xb);
  R.neq = warp_sum(nq);
  // every internal delta equals d exactly when the zigzag deltas are all zigzag(d)
  R.stride_ok = (cnt < 2 || (R.dzmin == R.dzmax && R.dzmax == zigzag64(d))) ? 1 : 0;
  R.cnt = cnt;
  R.first = cnt ? sv[0] : 0;
  R.last = cnt ? sv[cnt - 1] : 0;
  R.d = d;
  R.fm_pass = do_float ? (uint8_t)(0x7Fu & ~warp_or(fmfail)) : 0;
  R.alp_ok = 0;
  R.alp_w = 0;
  R.alp_exc = 0;
  R.pad16 = 0;
  R.pad32 = 0;
  if (FLOATS && do_float) {
#pragma unroll
    for (int q = 0; q < 7; q++) {
      int64_t a = warp_min_i64(kmn[q]), b = warp_max_i64(kmx[q]);
      if (lane == 0) {
        fms[item].kmin[q] = a;
        fms[item].kmax[q] = b;
      }
    }
  }
  if (lane == 0) {
    ss[item] = R;
    s_first[warp] = R.first;
    s_last[warp] = R.last;
    s_neq[warp] = R.neq;
    s_cnt[warp] = cnt;
  }
  if (fixed_bs) return;
  // Window probe (reference encoder.rs:166-176, 705-750): grow the block at
  // this window when the sampled distinct count is low or most consecutive
  // values repeat.  consec_eq = len - transitions (the first element counts
  // against itself).
  __syncthreads();
  {
    uint32_t c = 0;
    for (int i = threadIdx.x; i < (int)(kLbBits / 32); i += blockDim.x) c += __popc(lbits[i]);
    c = warp_sum(c);
    if (lane == 0 && c) atomicAdd(&s_lbc, c);
  }
  __syncthreads();
  if (threadIdx.x == 0) winbits[(uint64_t)blockIdx.x * kWinWords + 1024] = s_lbc;
  if (warp == 0 && wlen) {
    uint32_t dc = 0;
    for (int i = lane; i < 512; i += 32) dc += __popc(bitsA[i]);
    dc = warp_sum(dc);
    uint32_t tr = 0;
    if (lane < kStatsWarps && s_cnt[lane]) {
      tr = s_neq[lane];
      if (lane > 0 && s_first[lane] != s_last[lane - 1]) tr++;
    }
    tr = warp_sum(tr);
    if (lane == 0) {
      uint32_t consec = wlen - tr;
      grow[blockIdx.x] = (dc < 2048 || (uint64_t)consec * 2 > wlen) ? 1 : 0;
    }
    for (int i = lane; i < 512; i += 32) {
      winbits[(uint64_t)blockIdx.x * kWinWords + i] = bitsA[i];
      winbits[(uint64_t)blockIdx.x * kWinWords + 512 + i] = bitsB[i];
    }
  }
}

// ---------------------------------------------------------------------------
// Competition, part 2: one CTA per block.  Candidate sizes in closed form
// from the sub-block statistics, the integer early-out, the ALP-RD cut search,
// and the DICT / RLE passes for compressible blocks (encoder.rs:275-469).
// ---------------------------------------------------------------------------
__device__ uint32_t popc_bits_block(EncSmem& S, const uint32_t* bits) {
  uint32_t c = 0;
  for (int i = threadIdx.x; i < 512; i += blockDim.x) c += __popc(bits[i]);
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0) S.red32[threadIdx.x >> 5] = c;
  __syncthreads();
  uint32_t t = 0;
  for (int w = 0; w < kEncWarps; w++) t += S.red32[w];
  __syncthreads();
  return t;
}

// ---------------------------------------------------------------------------
// Selection::Sample (reference encoder.rs:470-620) at Fastest and Fast: the
// candidate modes are sized on a stratified sample of the block (8 runs of 64
// values spread over it, or the whole block up to 512 values) and the
// smallest estimate, first in SAMPLE_MODES order on ties, is the one encoded
// in full.  The in-pool members at these levels: Xorz, ForBitpack,
// DeltaBitpack, Alp and AlpRd (float columns), Dict, Rle; FloatMult and
// ByteTranspose are entropy modes (Balanced and above).
// ---------------------------------------------------------------------------
__device__ __noinline__ int sample_winner(EncSmem& S, const uint64_t* v, uint32_t n, int dtype, uint8_t* scr) {
  int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint64_t* smp = reinterpret_cast<uint64_t*>(&S.ra.buf[0][0]);  // 512 values (the rANS staging is idle)
  uint32_t m = n <= 512u ? n : 512u;
  for (uint32_t i = t; i < m; i += blockDim.x) {
    uint32_t src = i;
    if (n > 512u) {  // build_sample: run r starts at r * (n - 64) / 7
      uint32_t r = i >> 6;
      src = (uint32_t)((uint64_t)r * (n - 64u) / 7u) + (i & 63u);
    }
    smp[i] = v[src];
  }
  if (t == 0) {
    S.sc[0] = 0;            // XORZ bytes
    S.sc[1] = kEmpty64;     // unsigned min
    S.sc[2] = 0;            // unsigned max
    S.sc[3] = kEmpty64;     // signed min, as x ^ 2^63 (signed order in unsigned compares)
    S.sc[4] = 0;            // signed max, likewise
    S.sc[5] = kEmpty64;     // zigzag delta min
    S.sc[6] = 0;            // zigzag delta max
    S.cnt32 = 0;            // transitions
  }
  __syncthreads();
  const bool fl = dtype_float(dtype), sgn = dtype_signed(dtype);
  const uint64_t kBias = 0x8000000000000000ull;  // signed order as unsigned order
  {
    uint64_t xb = 0, umn = kEmpty64, umx = 0, bmn = kEmpty64, bmx = 0, dmn = kEmpty64, dmx = 0;
    uint32_t tr = 0;
    for (uint32_t i = t; i < m; i += blockDim.x) {
      uint64_t x = smp[i], pv = i ? smp[i - 1] : 0ull;
      xb += varint_len(x ^ pv);
      umn = u64min(umn, x);
      umx = u64max(umx, x);
      bmn = u64min(bmn, x ^ kBias);
      bmx = u64max(bmx, x ^ kBias);
      uint64_t dz = i ? zigzag64(x - pv) : 0ull;  // delta_bitpack: d_0 = 0
      dmn = u64min(dmn, dz);
      dmx = u64max(dmx, dz);
      tr += (i && x != pv) ? 1u : 0u;
    }
    xb = warp_sum(xb);
    umn = warp_min(umn);
    umx = warp_max(umx);
    bmn = warp_min(bmn);
    bmx = warp_max(bmx);
    dmn = warp_min(dmn);
    dmx = warp_max(dmx);
    tr = warp_sum(tr);
    if (lane == 0) {
      atomicAdd((unsigned long long*)&S.sc[0], (unsigned long long)xb);
      atomic_min_u64((unsigned long long*)&S.sc[1], umn);
      atomic_max_u64((unsigned long long*)&S.sc[2], umx);
      atomic_min_u64((unsigned long long*)&S.sc[3], bmn);
      atomic_max_u64((unsigned long long*)&S.sc[4], bmx);
      atomic_min_u64((unsigned long long*)&S.sc[5], dmn);
      atomic_max_u64((unsigned long long*)&S.sc[6], dmx);
      atomicAdd(&S.cnt32, tr);
    }
  }
  __syncthreads();
  uint64_t vl = varint_len(m);
  uint64_t est_xorz = S.sc[0];
  uint64_t est_for = vl + 9 + 128ull * bit_width64(sgn ? S.sc[4] - S.sc[3] : S.sc[2] - S.sc[1]);
  uint64_t est_delta = 8 + vl + 9 + 128ull * bit_width64(S.sc[6] - S.sc[5]);
  uint32_t transitions = S.cnt32;
  __syncthreads();
  int win = M_XORZ;
  uint64_t win_est = est_xorz;
  auto take = [&](int mode, uint64_t est) {
    if (est < win_est) {
      win_est = est;
      win = mode;
    }
  };
  take(M_FOR_BITPACK, est_for);
  take(M_DELTA_BITPACK, est_delta);
  if (fl) {
    // ALP (alp.rs:93-166): one sub-block
    if (warp == 0) {
      AlpSub a;
      bool ok = alp_subblock(smp, m, S.alp_smp[0], kExp10, kFrac10, &a);
      if (lane == 0) S.sc[7] = ok ? vl + 13 + 128ull * a.w + 10ull * a.exc : kEmpty64;
    }
    __syncthreads();
    uint64_t est_alp = S.sc[7];
    __syncthreads();
    if (est_alp != kEmpty64) take(M_ALP, est_alp);
    // ALP-RD (alp_rd.rs:132-206), bit-packed streams
    uint32_t lbw = rd_choose_cut(S, smp, m, nullptr, 0);
    if (lbw) {
      rd_top8(S, smp, m, lbw, scr);
      uint32_t rbw = 64 - lbw;
      uint64_t rmask = (1ull << rbw) - 1ull;
      if (t == 0) {
        S.sc[0] = 0;         // exception bytes
        S.sc[1] = kEmpty64;  // code min
        S.sc[2] = 0;         // code max
        S.sc[3] = kEmpty64;  // right min
        S.sc[4] = 0;         // right max
        S.cnt32 = 0;         // exceptions
      }
      __syncthreads();
      uint64_t eb = 0, cmn = kEmpty64, cmx = 0, rmn = kEmpty64, rmx = 0;
      uint32_t ne = 0;
      for (uint32_t i = t; i < m; i += blockDim.x) {
        uint64_t x = smp[i];
        int c = rd_code(S, x >> rbw);
        uint64_t code = c < 0 ? 0ull : (uint64_t)c;
        if (c < 0) {
          ne++;
          eb += varint_len(i) + 8;
        }
        cmn = u64min(cmn, code);
        cmx = u64max(cmx, code);
        rmn = u64min(rmn, x & rmask);
        rmx = u64max(rmx, x & rmask);
      }
      eb = warp_sum(eb);
      ne = warp_sum(ne);
      cmn = warp_min(cmn);
      cmx = warp_max(cmx);
      rmn = warp_min(rmn);
      rmx = warp_max(rmx);
      if (lane == 0) {
        atomicAdd((unsigned long long*)&S.sc[0], (unsigned long long)eb);
        atomic_min_u64((unsigned long long*)&S.sc[1], cmn);
        atomic_max_u64((unsigned long long*)&S.sc[2], cmx);
        atomic_min_u64((unsigned long long*)&S.sc[3], rmn);
        atomic_max_u64((unsigned long long*)&S.sc[4], rmx);
        atomicAdd(&S.cnt32, ne);
      }
      __syncthreads();
      uint64_t nexc = S.cnt32;
      uint64_t clen = vl + 9 + 128ull * bit_width64(S.sc[2] - S.sc[1]);
      uint64_t rlen = vl + 9 + 128ull * bit_width64(S.sc[4] - S.sc[3]);
      if (nexc * 4 <= m)
        take(M_ALP_RD, 2 + 8ull * S.dl + varint_len(nexc) + S.sc[0] + 1 + varint_len(clen) + clen + 1 + rlen);
      __syncthreads();
    }
  }
  // DICT (dict.rs:87-152), bit-packed codes
  DictView dv = dict_prepare(S, smp, m, scr, kNoLb);
  if (!S.flag) {
    uint32_t vtag;
    uint64_t vlen = dict_values_len(S, dv, &vtag);
    if (t == 0) {
      S.sc[1] = kEmpty64;
      S.sc[2] = 0;
    }
    __syncthreads();
    uint64_t rmn = kEmpty64, rmx = 0;
    for (uint32_t i = t; i < m; i += blockDim.x) {
      uint64_t r = dict_rank(S, dv, smp[i]);
      rmn = u64min(rmn, r);
      rmx = u64max(rmx, r);
    }
    rmn = warp_min(rmn);
    rmx = warp_max(rmx);
    if (lane == 0) {
      atomic_min_u64((unsigned long long*)&S.sc[1], rmn);
      atomic_max_u64((unsigned long long*)&S.sc[2], rmx);
    }
    __syncthreads();
    uint64_t clen = vl + 9 + 128ull * bit_width64(S.sc[2] - S.sc[1]);
    take(M_DICT, varint_len(dv.card) + 1 + varint_len(vlen) + vlen + 1 + clen);
  }
  __syncthreads();
  // RLE (rle.rs:10-42): completed runs beyond m/2 + 1 bail
  if (transitions <= m / 2 + 1) {
    if (t == 0) {
      uint32_t runs = transitions + 1, start = 0, lmn = 0xFFFFFFFFu, lmx = 0;
      for (uint32_t i = 1; i <= m; i++)
        if (i == m || smp[i] != smp[i - 1]) {
          uint32_t len = i - start;
          lmn = min(lmn, len);
          lmx = max(lmx, len);
          start = i;
        }
      S.sc[0] = varint_len(runs) + 8ull * runs + varint_len(runs) + 9 + 128ull * bit_width64((uint64_t)(lmx - lmn));
    }
    __syncthreads();
    take(M_RLE, S.sc[0]);
  }
  __syncthreads();
  return win;
}

// ENT: the Balanced in-pool competition, with the rANS-coded forms of
// FLOAT_MULT, ALP-RD and DICT and the BYTE_TRANSPOSE candidate; the chosen
// coded parts go to ent[b] for the emission.
template <bool ENT, bool SAMPLE>
__global__ void __launch_bounds__(kEncThreads) k_decide(const uint64_t* __restrict__ lane, FrameDesc* frames,
                                                        const uint32_t* __restrict__ nbp, uint64_t fixed_bs,
                                                        int dtype, int level, const SubStats* __restrict__ ss,
                                                        const FmStat* __restrict__ fms,
                                                        const uint64_t* __restrict__ smp16,
                                                        const uint32_t* __restrict__ winbits,
                                                        uint8_t* __restrict__ scratch, EntRec* __restrict__ ent) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  EncSmem& S = *reinterpret_cast<EncSmem*>(smem_raw);
  uint32_t b = blockIdx.x;
  if (b >= *nbp) return;
  FrameDesc fd = frames[b];
  const uint64_t* v = lane + fd.value_off;
  uint32_t n = fd.n;
  uint8_t* scr = scratch + fd.value_off * kEncScratchPerValue;
  bool fam_float = dtype_float(dtype);
  bool reduced = level == 0;
  bool sgn = dtype_signed(dtype);
  uint64_t lambda = level_lambda(level);
  uint64_t lb = lane_bytes(dtype);
  uint64_t decoded_bytes = (uint64_t)n * lb, raw_bytes = (uint64_t)n * 8;
  uint32_t nsub = (n + kSub - 1) / kSub;
  uint64_t g0 = fixed_bs ? (uint64_t)b * ((fixed_bs + kSub - 1) / kSub) : fd.value_off / kSub;
  int t = threadIdx.x, lane_id = t & 31, warp = t >> 5;
  uint32_t step = max(n / 2048u, 1u);
  EntRec er = {0, 0, 0, 0, 0, 0, {0, 0}};
  // Early-out samples from the statistics when the block is a full adaptive block.
  bool pre_e = !fixed_bs && (step == 16 || step == 64) && (fd.value_off % kBaseQuantum) == 0;
  if (t == 0) {
    S.xor_bytes = 0;
    S.umin = kEmpty64;
    S.umax = 0;
    S.e_vmin = kEmpty64;
    S.e_vmax = 0;
    S.e_dmax = 0;
    S.neq = 0;
    S.stride_bad = 0;
    S.fm_mask = 0x7F;
    S.alp_fail = 0;
    S.acc64 = 0;
    S.sc[1] = 0;
    S.sc[2] = 0;
    S.sc[4] = 0;
  }
  __syncthreads();
  uint64_t D = n >= 2 ? v[1] - v[0] : 0;
  uint64_t my_for = 0, my_delta = 0, my_alp = 0;
  for (uint32_t k = t; k < nsub; k += blockDim.x) {
    SubStats R = ss[g0 + k];
    uint64_t pl = k ? ss[g0 + k - 1].last : 0;
    uint32_t wf = sgn ? bit_width64((uint64_t)R.smax - (uint64_t)R.smin) : bit_width64(R.umax - R.umin);
    uint64_t dzf = k ? zigzag64(R.first - pl) : 0;
    uint64_t dmn = R.cnt > 1 ? u64min(R.dzmin, dzf) : dzf, dmx = R.cnt > 1 ? u64max(R.dzmax, dzf) : dzf;
    my_for += 9 + 128ull * wf;
    my_delta += 9 + 128ull * bit_width64(dmx - dmn);
    uint32_t nq = R.neq + ((k && R.first != pl) ? 1u : 0u);
    S.neq_k[k] = nq;
    S.item_min[k] = R.umin;
    S.item_max[k] = R.umax;
    atomicAdd(&S.neq, nq);
    atomicAdd(&S.xor_bytes, (unsigned long long)(R.xb + varint_len(R.first ^ pl)));
    atomic_min_u64(&S.umin, R.umin);
    atomic_max_u64(&S.umax, R.umax);
    bool sok = R.stride_ok && (R.cnt < 2 || R.d == D) && (k == 0 || R.first - pl == D);
    if (!sok) atomicOr(&S.stride_bad, 1u);
    if (pre_e) {
      uint64_t emn = step == 16 ? R.e16min : R.e64min, emx = step == 16 ? R.e16max : R.e64max;
      uint64_t edz = step == 16 ? R.e16dz : R.e64dz;
      if (k) edz = u64max(edz, dzf);
      atomic_min_u64(&S.e_vmin, emn);
      atomic_max_u64(&S.e_vmax, emx);
      atomic_max_u64(&S.e_dmax, edz);
    }
    if (fam_float && !reduced) {
      atomicAnd(&S.fm_mask, (uint32_t)R.fm_pass);
      if (!R.alp_ok) atomicOr(&S.alp_fail, 1u);
      my_alp += 13 + 128ull * R.alp_w + 10ull * R.alp_exc;
    }
  }
  my_for = warp_sum(my_for);
  my_delta = warp_sum(my_delta);
  my_alp = warp_sum(my_alp);
  if (lane_id == 0) {
    atomicAdd((unsigned long long*)&S.sc[1], (unsigned long long)my_for);
    atomicAdd((unsigned long long*)&S.sc[2], (unsigned long long)my_delta);
    atomicAdd((unsigned long long*)&S.sc[4], (unsigned long long)my_alp);
  }
  __syncthreads();
  uint64_t vl = varint_len(n);
  uint64_t sz_for = vl + S.sc[1], sz_delta = 8 + vl + S.sc[2], sz_alp = vl + S.sc[4];
  // Selection::Sample: the mode whose estimate on the block's sample is the
  // smallest; it alone is sized in full below (encoder.rs:574-620).
  int win = -1;
  if (SAMPLE) win = sample_winner(S, v, n, dtype, scr);

  // Integer early-out (encoder.rs:295-298, 655-683) with the block's features
  // (the sampled selection has none).
  bool eo = false;
  if (!SAMPLE && !fam_float) {
    uint32_t consec_eq = n - S.neq;
    bool repeats = (uint64_t)consec_eq * 2 > (uint64_t)n;
    uint32_t dstride = max(n / 4096u, 1u);
    uint32_t distinct;
    uint64_t wi = fd.value_off / kBaseQuantum;
    if (!fixed_bs && dstride == 8 && n == (uint32_t)kBaseQuantum) {
      distinct = popc_bits_block(S, winbits + wi * kWinWords);
    } else if (!fixed_bs && dstride == 32 && n == (uint32_t)kMaxBlock) {
      for (int i = t; i < 512; i += blockDim.x)
        S.distinct_bits[i] = winbits[wi * kWinWords + 512 + i] | winbits[(wi + 1) * kWinWords + 512 + i] |
                             winbits[(wi + 2) * kWinWords + 512 + i] | winbits[(wi + 3) * kWinWords + 512 + i];
      __syncthreads();
      distinct = popc_bits_block(S, S.distinct_bits);
    } else {
      for (int i = t; i < 512; i += blockDim.x) S.distinct_bits[i] = 0;
      __syncthreads();
      for (uint32_t i = t; (uint64_t)i * dstride < n; i += blockDim.x) {
        uint64_t h = v[(uint64_t)i * dstride] * 0x9E3779B97F4A7C15ull;
        uint32_t bk = (uint32_t)((h >> 50) & 0x3FFF);
        atomicOr(&S.distinct_bits[bk >> 5], 1u << (bk & 31));
      }
      __syncthreads();
      distinct = popc_bits_block(S, S.distinct_bits);
    }
    bool distinct_low = distinct < 2048;
    if (!(distinct_low || repeats || n < 256)) {
      if (!pre_e) {
        if (t == 0) {
          S.e_vmin = v[0];
          S.e_vmax = v[0];
          S.e_dmax = 0;
        }
        __syncthreads();
        for (uint32_t i = t; (uint64_t)i * step < n; i += blockDim.x) {
          uint32_t idx = i * step;
          uint64_t x = v[idx];
          atomic_min_u64(&S.e_vmin, x);
          atomic_max_u64(&S.e_vmax, x);
          if (idx >= step) atomic_max_u64(&S.e_dmax, zigzag64(x - v[idx - 1]));
        }
        __syncthreads();
      }
      uint32_t thr = (uint32_t)(lb * 8) - 4;
      uint32_t vw = bit_width64(S.e_vmax - S.e_vmin), dw = bit_width64(S.e_dmax);
      eo = vw >= thr && dw >= thr;
    }
  }
  if (eo) {
    if (t == 0) {
      frames[b].mode = M_RAW;
      frames[b].plen = (uint32_t)decoded_bytes;
      frames[b].aux = 0;
      atomicAdd(&g_wins[M_RAW], 1ull);
    }
    return;
  }

  Cand c_fm = {0, false}, c_alp = {0, false}, c_rd = {0, false};
  uint32_t fm_scale = 0, rd_lbw = 0;
  if (fam_float && (SAMPLE ? (win == M_ALP || win == M_ALP_RD) : !reduced)) {
    uint32_t mask = SAMPLE ? 0u : S.fm_mask;  // FLOAT_MULT is an entropy mode for the sampled pool
    if (mask) {  // FLOAT_MULT (float_mult.rs:66-98, bit-packed k)
      fm_scale = __ffs(mask) - 1;
      uint64_t my = 0;
      for (uint32_t k = t; k < nsub; k += blockDim.x) {
        const FmStat& F = fms[g0 + k];
        my += 9 + 128ull * bit_width64((uint64_t)F.kmax[fm_scale] - (uint64_t)F.kmin[fm_scale]);
      }
      my = warp_sum(my);
      if (lane_id == 0) S.red[warp] = my;
      __syncthreads();
      uint64_t tot = 0;
      for (int w = 0; w < kEncWarps; w++) tot += S.red[w];
      __syncthreads();
      c_fm.ok = true;
      c_fm.len = 2 + vl + tot;
      if (ENT) {  // FM_ENTROPY, kept when strictly smaller (float_mult.rs:80-92)
        uint32_t m = fm_delta_bytes(S, v, n, (int)fm_scale, scr);
        uint32_t el = coded_len(S.ra, m, [&](uint32_t i) { return (uint32_t)scr[i]; }, c_fm.len - 2);
        if (el < c_fm.len - 2) {
          c_fm.len = 2 + el;
          er.flags |= kEntFm;
          er.fm = el;
        }
      }
    }
    c_alp.ok = !S.alp_fail;  // ALP (alp.rs:93-166)
    c_alp.len = sz_alp;
    if (SAMPLE && win == M_ALP && reduced) {  // Fastest gathered no ALP statistics: size it here
      if (t == 0) {
        S.acc64 = 0;
        S.alp_fail = 0;
      }
      __syncthreads();
      for (uint32_t k = warp; k < nsub; k += kEncWarps) {
        uint32_t cnt = min((uint32_t)kSub, n - k * kSub);
        AlpSub a;
        bool ok = alp_subblock(v + (uint64_t)k * kSub, cnt, S.alp_smp[warp], kExp10, kFrac10, &a);
        if (lane_id == 0) {
          if (ok) atomicAdd(&S.acc64, (unsigned long long)(13 + 128ull * a.w + 10ull * a.exc));
          else atomicOr(&S.alp_fail, 1u);
        }
      }
      __syncthreads();
      c_alp.ok = !S.alp_fail;
      c_alp.len = vl + S.acc64;
    }
    // ALP-RD (alp_rd.rs:132-206, bit-packed streams)
    bool pre_s = smp16 && !fixed_bs && (step == 16 || step == 64) && (fd.value_off % kBaseQuantum) == 0;
    rd_lbw = (SAMPLE && win != M_ALP_RD) ? 0u
                                         : rd_choose_cut(S, v, n, pre_s ? smp16 + fd.value_off / 16 : nullptr,
                                                         step / 16);
    if (rd_lbw && !SAMPLE && !ENT) {
      // The rights' FoR size is exact from one cheap pass (each sub-block's
      // range of x & rmask); with the smallest possible rest of the payload
      // (a 2-byte header, varint(nexc), the tags and lengths, one 9-byte
      // header per code sub-block) and ALP-RD's decode penalty, it may
      // already reach the best score of the candidates sized so far, and
      // ALP-RD cannot win (strict <): its dictionary and exception passes are
      // skipped.
      uint32_t rbw = 64 - rd_lbw;
      uint64_t rmask = (1ull << rbw) - 1ull;
      if (t == 0) S.acc64 = 0;
      __syncthreads();
      for (uint32_t k = warp; k < nsub; k += kEncWarps) {
        uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
        uint64_t rmn = kEmpty64, rmx = 0;
        for (uint32_t i = lane_id; i < cnt; i += 32) {
          uint64_t r = v[base + i] & rmask;
          rmn = u64min(rmn, r);
          rmx = u64max(rmx, r);
        }
        rmn = warp_min(rmn);
        rmx = warp_max(rmx);
        if (lane_id == 0) atomicAdd(&S.acc64, (unsigned long long)(9 + 128ull * bit_width64(rmx - rmn)));
      }
      __syncthreads();
      uint64_t floor_len = 6 + 2 * vl + 9ull * nsub + S.acc64;
      uint64_t best = decoded_bytes + ((lambda * decode_weight(M_RAW) * decoded_bytes) >> 8);
      auto sc_of = [&](int m, uint64_t len) { return len + ((lambda * decode_weight(m) * decoded_bytes) >> 8); };
      if (S.umin == S.umax) best = u64min(best, sc_of(M_CONST, 8));
      if (n >= 2 && !S.stride_bad) best = u64min(best, sc_of(M_STRIDE, 16));
      if (!reduced) best = u64min(best, sc_of(M_XORZ, S.xor_bytes));
      best = u64min(best, sc_of(M_FOR_BITPACK, sz_for));
      best = u64min(best, sc_of(M_DELTA_BITPACK, sz_delta));
      if (c_fm.ok) best = u64min(best, sc_of(M_FLOAT_MULT, c_fm.len));
      if (c_alp.ok) best = u64min(best, sc_of(M_ALP, c_alp.len));
      if (sc_of(M_ALP_RD, floor_len) >= best) rd_lbw = 0;
      __syncthreads();
    }
    if (rd_lbw) {
      rd_top8(S, v, n, rd_lbw, scr);
      uint32_t rbw = 64 - rd_lbw;
      uint64_t rmask = (1ull << rbw) - 1ull;
      if (t == 0) {
        S.acc64 = 0;
        S.cnt32 = 0;
      }
      __syncthreads();
      for (uint32_t k = warp; k < nsub; k += kEncWarps) {
        uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
        uint64_t cmx = 0, rmn = kEmpty64, rmx = 0, cmn = kEmpty64, eb = 0;
        uint32_t ne = 0;
        for (uint32_t i = lane_id; i < cnt; i += 32) {
          uint64_t x = v[base + i];
          int c = rd_code(S, x >> rbw);
          uint64_t code = c < 0 ? 0 : (uint64_t)c;
          if (c < 0) {
            ne++;
            eb += varint_len(base + i) + 8;
          }
          cmn = u64min(cmn, code);
          cmx = u64max(cmx, code);
          rmn = u64min(rmn, x & rmask);
          rmx = u64max(rmx, x & rmask);
        }
        cmn = warp_min(cmn);
        cmx = warp_max(cmx);
        rmn = warp_min(rmn);
        rmx = warp_max(rmx);
        ne = warp_sum(ne);
        eb = warp_sum(eb);
        if (lane_id == 0) {
          S.w_a[k] = (uint8_t)bit_width64(cmx - cmn);
          S.w_b[k] = (uint8_t)bit_width64(rmx - rmn);
          atomicAdd(&S.cnt32, ne);
          atomicAdd(&S.acc64, (unsigned long long)eb);
        }
      }
      __syncthreads();
      uint64_t nexc = S.cnt32, excb = S.acc64, clen = vl, rlen = vl;
      for (uint32_t k = 0; k < nsub; k++) {
        clen += 9 + 128ull * S.w_a[k];
        rlen += 9 + 128ull * S.w_b[k];
      }
      c_rd.ok = nexc * 4 <= n;
      if (ENT && c_rd.ok) {  // T_ENT codes / rights, kept when strictly smaller (alp_rd.rs:176-200)
        uint32_t cl = coded_len(S.ra, n, [&](uint32_t i) {
          int c = rd_code(S, v[i] >> rbw);
          return (uint32_t)(c < 0 ? 0 : c);
        }, clen);
        if (cl < clen) {
          clen = cl;
          er.flags |= kEntRdCodes;
          er.rdc = cl;
        }
        uint8_t* rdst = stage_dst(S, scr, n, rlen);
        uint32_t rb = (uint32_t)block_for(S, rdst, n, false, [&](uint32_t i) { return v[i] & rmask; });
        uint32_t rl = coded_len(S.ra, rb, [&](uint32_t i) { return (uint32_t)rdst[i]; }, rlen);
        if (rl < rlen) {
          rlen = rl;
          er.flags |= kEntRdRights;
          er.rdr = rl;
        }
      }
      c_rd.len = 2 + 8ull * S.dl + varint_len(nexc) + excb + 1 + varint_len(clen) + clen + 1 + rlen;
      __syncthreads();
    }
  }

  // Selection up to ALP-RD (encoder.rs:301-344), then the compressibility gate.
  int best_mode = M_RAW;
  uint64_t best_len = decoded_bytes;
  uint64_t best_score = best_len + ((lambda * decode_weight(M_RAW) * decoded_bytes) >> 8);
  auto consider = [&](int m, uint64_t len) {
    uint64_t sc = len + ((lambda * decode_weight(m) * decoded_bytes) >> 8);
    if (sc < best_score) {
      best_score = sc;
      best_mode = m;
      best_len = len;
    }
  };
  if (S.umin == S.umax) consider(M_CONST, 8);
  if (n >= 2 && !S.stride_bad) consider(M_STRIDE, 16);
  if (SAMPLE) {  // the sample's winner, sized in full (DICT / RLE below)
    if (win == M_XORZ) consider(M_XORZ, S.xor_bytes);
    if (win == M_FOR_BITPACK) consider(M_FOR_BITPACK, sz_for);
    if (win == M_DELTA_BITPACK) consider(M_DELTA_BITPACK, sz_delta);
    if (win == M_ALP && c_alp.ok) consider(M_ALP, c_alp.len);
    if (win == M_ALP_RD && c_rd.ok) consider(M_ALP_RD, c_rd.len);
  } else {
    if (!reduced) consider(M_XORZ, S.xor_bytes);
    consider(M_FOR_BITPACK, sz_for);
    consider(M_DELTA_BITPACK, sz_delta);
    if (c_fm.ok) consider(M_FLOAT_MULT, c_fm.len);
    if (c_alp.ok) consider(M_ALP, c_alp.len);
    if (c_rd.ok) consider(M_ALP_RD, c_rd.len);
  }
  bool block_compressible = best_len * 20 < raw_bytes * 19;  // encoder.rs:394,644-646

  if (ENT && block_compressible) {
    // BYTE_TRANSPOSE (encoder.rs:414-420) when the exponent-field range is at
    // most 64 or most consecutive values repeat (encoder.rs:705-750)
    if (t == 0) {
      S.exp_lo = 0x7FF;
      S.exp_hi = 0;
    }
    __syncthreads();
    uint32_t elo = 0x7FF, ehi = 0;
    for (uint32_t i = t; i < n; i += blockDim.x) {
      uint32_t ex = (uint32_t)(v[i] >> 52) & 0x7FFu;
      elo = min(elo, ex);
      ehi = max(ehi, ex);
    }
    elo = warp_min(elo);
    ehi = warp_max(ehi);
    if (lane_id == 0) {
      atomicMin(&S.exp_lo, elo);
      atomicMax(&S.exp_hi, ehi);
    }
    __syncthreads();
    bool repeats = (uint64_t)(n - S.neq) * 2 > (uint64_t)n;
    if (S.exp_hi - S.exp_lo <= 64 || repeats) {
      // BYTE_TRANSPOSE wins only below best_score less its decode penalty
      uint64_t pen = (lambda * decode_weight(M_BYTE_TRANSPOSE) * decoded_bytes) >> 8;
      uint32_t bl = coded_len(S.ra, 8 * n, [&](uint32_t i) {
        uint32_t pl = i / n;
        return (uint32_t)(v[i - pl * n] >> (8 * pl)) & 255u;
      }, best_score > pen ? best_score - pen : 0ull);
      er.bt = bl;
      consider(M_BYTE_TRANSPOSE, bl);
    }
  }

  if (SAMPLE ? (win == M_DICT || win == M_RLE) : (block_compressible && !reduced)) {
    // DICT (dict.rs:87-152, bit-packed codes).  The dictionary is sorted, so
    // a sub-block's code range is [rank(min), rank(max)].
    bool one_win = !fixed_bs && (fd.value_off % kBaseQuantum) == 0 && n <= (uint32_t)kBaseQuantum;
    uint32_t lb_pre = one_win ? winbits[(fd.value_off / kBaseQuantum) * kWinWords + 1024] : kNoLb;
    bool want_dict = !SAMPLE || win == M_DICT;
    // A DICT payload holds at least 22 bytes (card, value tag and length, 8
    // value bytes, code tag, varint(n) and one 9-byte sub-block header): when
    // that and DICT's decode penalty already reach the best score, it cannot
    // win (strict <) and its passes are skipped.
    if (!SAMPLE && best_score <= 22 + ((lambda * decode_weight(M_DICT) * decoded_bytes) >> 8)) want_dict = false;
    DictView dv;
    if (want_dict) dv = dict_prepare(S, v, n, scr, lb_pre);
    if (want_dict && !S.flag) {
      uint32_t vtag;
      uint64_t vlen = dict_values_len(S, dv, &vtag);
      if (ENT) {  // TRANSPOSE values, kept when strictly smaller (dict.rs:52-59)
        const uint64_t* sv = dv.sorted;
        uint32_t card = dv.card;
        uint32_t tl = coded_len(S.ra, 8 * card, [&](uint32_t i) {
          uint32_t pl = i / card;
          return (uint32_t)(sv[i - pl * card] >> (8 * pl)) & 255u;
        }, vlen);
        if (tl < vlen) {
          vlen = tl;
          vtag = 2;
          er.flags |= kEntDictVals;
          er.dv = tl;
        }
      }
      uint64_t my = 0;
      for (uint32_t k = t; k < nsub; k += blockDim.x) {
        uint32_t r0 = dict_rank(S, dv, S.item_min[k]), r1 = dict_rank(S, dv, S.item_max[k]);
        my += 9 + 128ull * bit_width64((uint64_t)(r1 - r0));
      }
      my = warp_sum(my);
      if (lane_id == 0) S.red[warp] = my;
      __syncthreads();
      uint64_t clen = vl;
      for (int w = 0; w < kEncWarps; w++) clen += S.red[w];
      __syncthreads();
      if (ENT && dv.card <= 65536u) {  // CODES_ENTROPY byte planes, kept when strictly smaller (dict.rs:128-145)
        uint32_t nb = dv.card <= 256u ? 1u : 2u;
        uint64_t el = 1;
        uint32_t pls[2] = {0, 0};
        for (uint32_t pl = 0; pl < nb; pl++) {
          pls[pl] = coded_len(S.ra, n, [&](uint32_t i) { return (dict_rank(S, dv, v[i]) >> (8 * pl)) & 255u; },
                              clen);
          el += varint_len(pls[pl]) + pls[pl];
        }
        if (el < clen) {
          clen = el;
          er.flags |= kEntDictCodes;
          er.dc[0] = pls[0];
          er.dc[1] = pls[1];
        }
      }
      consider(M_DICT, varint_len(dv.card) + 1 + varint_len(vlen) + vlen + 1 + clen);
    }
    __syncthreads();
    // RLE (rle.rs:10-42)
    uint32_t neq = S.neq;
    // likewise RLE's floor: the run values and two varint(runs) plus a 9-byte
    // header per 1,024 run lengths
    const uint64_t rle_floor = 2 * varint_len(neq + 1) + 8ull * (neq + 1) + 9ull * ((neq + 1 + kSub - 1) / kSub) +
                               ((lambda * decode_weight(M_RLE) * decoded_bytes) >> 8);
    if ((!SAMPLE || win == M_RLE) && neq <= n / 2 + 1 && (SAMPLE || best_score > rle_floor)) {
      uint32_t runs = neq + 1;
      uint32_t* st = rle_starts(S, v, n, runs, scr);
      uint64_t lens = block_for(S, nullptr, runs, false, [&](uint32_t r) {
        return (uint64_t)((r + 1 < runs ? st[r + 1] : n) - st[r]);
      });
      consider(M_RLE, varint_len(runs) + 8ull * runs + lens);
    }
  }
  if (t == 0) {
    frames[b].mode = (uint32_t)best_mode;
    frames[b].plen = (uint32_t)best_len;
    frames[b].aux = best_mode == M_FLOAT_MULT ? fm_scale : best_mode == M_ALP_RD ? rd_lbw : 0;
    atomicAdd(&g_wins[best_mode], 1ull);
    if (ENT) ent[b] = er;
  }
}

// ---------------------------------------------------------------------------
// Emission kernel: writes the frame header and the winner's payload.
// ---------------------------------------------------------------------------
__device__ void emit_raw(const uint64_t* v, uint32_t n, int dtype, uint8_t* out) {
  uint32_t lb = lane_bytes(dtype);
#pragma unroll 8
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    uint64_t x = v[i];
    if (dtype == DT_F32) put_u32(out + 4ull * i, f64bits_to_f32bits(x));
    else if (lb == 4) put_u32(out + 4ull * i, (uint32_t)x);
    else put_u64(out + 8ull * i, x);
  }
}

// S.subsz[k] holds each sub-block's LEB128 byte count on entry.
__device__ void emit_xorz(EncSmem& S, const uint64_t* v, uint32_t n, uint8_t* out) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nsub = (n + kSub - 1) / kSub;
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t k = 0; k < nsub; k++) {
      uint32_t c = S.subsz[k];
      S.subsz[k] = acc;
      acc += c;
    }
  }
  __syncthreads();
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
    uint32_t off = S.subsz[k];
    uint64_t carry = base ? v[base - 1] : 0ull;
    for (uint32_t j0 = 0; j0 < 32; j0 += 8) {
      uint64_t xs[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        uint32_t li = (j0 + q) * 32 + lane;
        xs[q] = li < cnt ? v[base + li] : 0ull;
      }
#pragma unroll
      for (int q = 0; q < 8; q++) {
        uint32_t li = (j0 + q) * 32 + lane;
        bool ok = li < cnt;
        uint64_t up = __shfl_up_sync(0xffffffffu, xs[q], 1);
        uint64_t x = ok ? xs[q] ^ (lane ? up : carry) : 0ull;
        carry = __shfl_sync(0xffffffffu, xs[q], 31);
        uint32_t sz = ok ? varint_len(x) : 0u;
        uint32_t inc = warp_incl_scan(sz);
        if (ok) put_varint(out + off + inc - sz, x);
        off += __shfl_sync(0xffffffffu, inc, 31);
      }
    }
  }
}

__device__ void emit_alp(EncSmem& S, const uint64_t* v, uint32_t n, const SubStats* ss, uint8_t* out) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nsub = (n + kSub - 1) / kSub;
  __shared__ int64_t s_fill[kSubsMax];
  __shared__ double s_pexp[19], s_pfrac[19];  // the (e, f) search reads them at per-lane indices
  if (threadIdx.x < 19) {
    s_pexp[threadIdx.x] = kExp10[threadIdx.x];
    s_pfrac[threadIdx.x] = kFrac10[threadIdx.x];
  }
  __syncthreads();
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t cnt = min((uint32_t)kSub, n - k * kSub);
    AlpSub a;
    uint16_t ef = ss ? ss[k].pad16 : 0;  // the statistics' (e, f), or search again (Sample at Fastest)
    if (ef & kAlpEfKnown) {
      a.e = ef & 0xFF;
      a.f = (ef >> 8) & 0x7F;
      alp_subblock_ef(v + (uint64_t)k * kSub, cnt, a.e, a.f, s_pexp, s_pfrac, &a);
    } else {
      alp_subblock(v + (uint64_t)k * kSub, cnt, S.alp_smp[warp], s_pexp, s_pfrac, &a);  // succeeded in the competition
    }
    if (lane == 0) {
      S.alp_ef[k][0] = (uint8_t)a.e;
      S.alp_ef[k][1] = (uint8_t)a.f;
      S.w_c[k] = (uint8_t)a.w;
      S.alp_exc[k] = (uint16_t)a.exc;
      S.submin[k] = (uint64_t)a.mn;
      s_fill[k] = a.filler;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t off = put_varint(out, n);
    for (uint32_t k = 0; k < nsub; k++) {
      S.subsz[k] = off;
      off += 13 + 128u * S.w_c[k] + 10u * S.alp_exc[k];
    }
  }
  __syncthreads();
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
    uint8_t* d = out + S.subsz[k];
    int e = S.alp_ef[k][0], f = S.alp_ef[k][1];
    uint32_t w = S.w_c[k];
    int64_t mn = (int64_t)S.submin[k], fill = s_fill[k];
    if (lane == 0) {
      put_u8(d, e);
      put_u8(d + 1, f);
      put_u16(d + 2, S.alp_exc[k]);
      put_u64(d + 4, (uint64_t)mn);
      put_u8(d + 12, w);
    }
    const uint64_t* sv = v + base;
    // Digits (exceptions and padding take the filler digit), FastLanes packed.
    if (w > 0) {
      uint64_t acc = 0;
      uint32_t nb = 0, wd = 0;
      for (uint32_t r = 0; r < 32; r++) {
        uint32_t i = r * 32 + lane;
        int64_t dg = fill;
        if (i < cnt) {
          int64_t dd;
          if (alp_roundtrips(sv[i], e, f, &dd)) dg = dd;
        }
        uint32_t res = (uint32_t)((uint64_t)dg - (uint64_t)mn);
        if (w < 32) res &= (1u << w) - 1u;
        acc |= (uint64_t)res << nb;
        nb += w;
        if (nb >= 32) {
          put_u32(d + 13 + 4u * (wd * 32u + lane), (uint32_t)acc);
          wd++;
          acc >>= 32;
          nb -= 32;
        }
      }
    }
    // Exceptions in position order.
    uint8_t* xp = d + 13 + 128u * w;
    uint32_t before = 0;
    for (uint32_t j = 0; j < 32; j++) {
      uint32_t li = j * 32 + lane;
      bool ok = li < cnt;
      int64_t dd;
      bool ex = ok && !alp_roundtrips(sv[li], e, f, &dd);
      uint32_t m = __ballot_sync(0xffffffffu, ex);
      if (ex) {
        uint8_t* q = xp + 10u * (before + __popc(m & ((1u << lane) - 1u)));
        put_u16(q, li);
        put_u64(q + 2, sv[li]);
      }
      before += __popc(m);
    }
  }
}

__device__ void emit_alprd(EncSmem& S, const uint64_t* v, uint32_t n, uint32_t lbw, uint8_t* scr, uint8_t* out,
                           const EntRec* er) {
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t nsub = (n + kSub - 1) / kSub;
  rd_top8(S, v, n, lbw, scr);
  uint32_t rbw = 64 - lbw;
  uint64_t rmask = (1ull << rbw) - 1ull;
  // exception bytes per sub-block
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
    uint32_t eb = 0, ne = 0;
    for (uint32_t i = lane; i < cnt; i += 32) {
      if (rd_code(S, v[base + i] >> rbw) < 0) {
        eb += varint_len(base + i) + 8;
        ne++;
      }
    }
    eb = warp_sum(eb);
    ne = warp_sum(ne);
    if (lane == 0) {
      S.subsz[k] = eb;
      S.neq_k[k] = ne;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t pos = 0;
    put_u8(out + pos++, lbw);
    put_u8(out + pos++, S.dl);
    for (uint32_t j = 0; j < S.dl; j++, pos += 8) put_u64(out + pos, S.dict8[j]);
    uint64_t nexc = 0;
    for (uint32_t k = 0; k < nsub; k++) nexc += S.neq_k[k];
    pos += put_varint(out + pos, nexc);
    for (uint32_t k = 0; k < nsub; k++) {
      uint32_t c = S.subsz[k];
      S.subsz[k] = pos;
      pos += c;
    }
    S.sc[6] = pos;  // codes tag position
  }
  __syncthreads();
  for (uint32_t k = warp; k < nsub; k += kEncWarps) {
    uint32_t base = k * kSub, cnt = min((uint32_t)kSub, n - base);
    uint32_t off = S.subsz[k];
    for (uint32_t j = 0; j < 32; j++) {
      uint32_t li = j * 32 + lane;
      bool ok = li < cnt;
      uint64_t x = ok ? v[base + li] : 0;
      bool ex = ok && rd_code(S, x >> rbw) < 0;
      uint32_t sz = ex ? varint_len(base + li) + 8 : 0u;
      uint32_t inc = warp_incl_scan(sz);
      if (ex) {
        uint8_t* q = out + off + inc - sz;
        uint32_t vlb = put_varint(q, base + li);
        put_u64(q + vlb, x >> rbw);
      }
      off += __shfl_sync(0xffffffffu, inc, 31);
    }
  }
  __syncthreads();
  uint64_t pos = S.sc[6];
  auto code_of = [&](uint32_t i) -> uint64_t {
    int c = rd_code(S, v[i] >> rbw);
    return c < 0 ? 0ull : (uint64_t)c;
  };
  uint64_t rpos;
  if (er && (er->flags & kEntRdCodes)) {
    uint32_t clen = er->rdc, cvl = varint_len(clen);
    if (threadIdx.x == 0) {
      put_u8(out + pos, 1);
      put_varint(out + pos + 1, clen);
    }
    coded_write(S.ra, n, [&](uint32_t i) { return (uint32_t)code_of(i); }, out + pos + 1 + cvl, clen);
    rpos = pos + 1 + cvl + clen;
  } else {
    uint64_t clen = block_for(S, nullptr, n, false, code_of);
    uint32_t cvl = varint_len(clen);
    if (threadIdx.x == 0) {
      put_u8(out + pos, 0);
      put_varint(out + pos + 1, clen);
    }
    block_for(S, out + pos + 1 + cvl, n, false, code_of);
    rpos = pos + 1 + cvl + clen;
  }
  auto right_of = [&](uint32_t i) { return v[i] & rmask; };
  if (er && (er->flags & kEntRdRights)) {  // the bit-packed rights, coded
    uint8_t* rdst = stage_dst(S, scr, n, block_for(S, nullptr, n, false, right_of));
    uint32_t rb = (uint32_t)block_for(S, rdst, n, false, right_of);
    if (threadIdx.x == 0) put_u8(out + rpos, 1);
    coded_write(S.ra, rb, [&](uint32_t i) { return (uint32_t)rdst[i]; }, out + rpos + 1, er->rdr);
  } else {
    if (threadIdx.x == 0) put_u8(out + rpos, 0);
    block_for(S, out + rpos + 1, n, false, right_of);
  }
}

__device__ void emit_dict(EncSmem& S, const uint64_t* v, uint32_t n, const SubStats* ss, uint8_t* scr, uint8_t* out,
                          const EntRec* er) {
  DictView dv = dict_prepare(S, v, n, scr, kNoLb);
  uint32_t vtag;
  uint64_t vlen = dict_values_len(S, dv, &vtag);
  if (er && (er->flags & kEntDictVals)) {
    vtag = 2;
    vlen = er->dv;
  }
  uint64_t pos = 0;
  if (threadIdx.x == 0) {
    pos = put_varint(out, dv.card);
    put_u8(out + pos++, vtag);
    pos += put_varint(out + pos, vlen);
    S.sc[6] = pos;
  }
  __syncthreads();
  pos = S.sc[6];
  const uint64_t* s = dv.sorted;
  uint32_t card = dv.card;
  if (vtag == 0) {
    for (uint32_t i = threadIdx.x; i < card; i += blockDim.x) put_u64(out + pos + 8ull * i, s[i]);
  } else if (vtag == 1) {
    if (threadIdx.x == 0) put_u64(out + pos, s[0]);
    block_for(S, out + pos + 8, card, false, [&](uint32_t i) { return zigzag64(s[i] - (i ? s[i - 1] : s[0])); });
  } else {
    coded_write(S.ra, 8 * card, [&](uint32_t i) {
      uint32_t pl = i / card;
      return (uint32_t)(s[i - pl * card] >> (8 * pl)) & 255u;
    }, out + pos, (uint32_t)vlen);
  }
  __syncthreads();
  pos += vlen;
  if (er && (er->flags & kEntDictCodes)) {  // nplanes, then varint(len) + coded plane each
    uint32_t nb = card <= 256u ? 1u : 2u;
    if (threadIdx.x == 0) {
      put_u8(out + pos, 1);
      put_u8(out + pos + 1, nb);
    }
    pos += 2;
    for (uint32_t pl = 0; pl < nb; pl++) {
      uint32_t len = er->dc[pl];
      if (threadIdx.x == 0) put_varint(out + pos, len);
      pos += varint_len(len);
      coded_write(S.ra, n, [&](uint32_t i) { return (dict_rank(S, dv, v[i]) >> (8 * pl)) & 255u; }, out + pos, len);
      pos += len;
    }
    return;
  }
  if (threadIdx.x == 0) put_u8(out + pos, 0);
  // The dictionary is sorted, so a sub-block's codes run from the rank of its
  // smallest value to the rank of its largest (the statistics' unsigned
  // min / max): the FoR widths and bases without a pass over the codes.
  uint32_t nsub = (n + kSub - 1) / kSub;
  for (uint32_t k = threadIdx.x; k < nsub; k += blockDim.x) {
    uint32_t r0 = dict_rank(S, dv, ss[k].umin), r1 = dict_rank(S, dv, ss[k].umax);
    S.w_a[k] = (uint8_t)bit_width64((uint64_t)(r1 - r0));
    S.submin[k] = r0;
  }
  __syncthreads();
  block_for_write(S, out + pos + 1, n, [&](uint32_t i) { return (uint64_t)dict_rank(S, dv, v[i]); });
}

// The block's run starts from its transitions per sub-block, which the
// statistics pass counted: the sub-block's own plus its first value against
// the previous sub-block's last (as the competition counts them).
__device__ void emit_rle(EncSmem& S, const uint64_t* v, uint32_t n, const SubStats* ss, uint8_t* scr,
                         uint8_t* out) {
  uint32_t nsub = (n + kSub - 1) / kSub;
  for (uint32_t k = threadIdx.x; k < nsub; k += blockDim.x) {
    const SubStats& R = ss[k];
    S.neq_k[k] = R.neq + ((k && R.first != ss[k - 1].last) ? 1u : 0u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (uint32_t k = 0; k < nsub; k++) t += S.neq_k[k];
    S.cnt32 = t + 1;
  }
  __syncthreads();
  uint32_t runs = S.cnt32;
  uint32_t* st = rle_starts(S, v, n, runs, scr);
  uint32_t vl = varint_len(runs);
  if (threadIdx.x == 0) put_varint(out, runs);
  for (uint32_t r = threadIdx.x; r < runs; r += blockDim.x) put_u64(out + vl + 8ull * r, v[st[r]]);
  block_for(S, out + vl + 8ull * runs, runs, false,
            [&](uint32_t r) { return (uint64_t)((r + 1 < runs ? st[r + 1] : n) - st[r]); });
}

template <bool ENT>
__global__ void __launch_bounds__(kEncThreads) k_emit(const uint64_t* __restrict__ lane,
                                                      const FrameDesc* __restrict__ frames,
                                                      const uint32_t* __restrict__ nbp, uint64_t fixed_bs, int dtype,
                                                      const SubStats* __restrict__ ss,
                                                      const FmStat* __restrict__ fms,
                                                      uint8_t* __restrict__ scratch, uint8_t* __restrict__ outbuf,
                                                      uint64_t out_cap, const EntRec* __restrict__ ent) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  EncSmem& S = *reinterpret_cast<EncSmem*>(smem_raw);
  uint32_t b = blockIdx.x;
  if (b >= *nbp) return;
  FrameDesc fd = frames[b];
  if (fd.payload_off + fd.plen > out_cap) return;  // the caller sees the total and reports the shortfall
  const uint64_t* v = lane + fd.value_off;
  uint32_t n = fd.n;
  uint8_t* scr = scratch + fd.value_off * kEncScratchPerValue;
  uint8_t* hdr = outbuf + fd.payload_off - 9;
  uint8_t* out = outbuf + fd.payload_off;
  if (threadIdx.x == 0) {
    put_u8(hdr, fd.mode);
    put_u32(hdr + 1, n);
    put_u32(hdr + 5, fd.plen);
  }
  bool sgn = dtype_signed(dtype);
  // FoR / DELTA / FLOAT_MULT / XORZ sub-block layouts come from the statistics
  // pass (the same numbers the competition sized the frame with).
  uint32_t nsub = (n + kSub - 1) / kSub;
  uint64_t g0 = fixed_bs ? (uint64_t)b * ((fixed_bs + kSub - 1) / kSub) : fd.value_off / kSub;
  int m = (int)fd.mode;
  EntRec er = {0, 0, 0, 0, 0, 0, {0, 0}};
  if (ENT) er = ent[b];
  const EntRec* erp = ENT ? &er : nullptr;
  if (m == M_FOR_BITPACK || m == M_DELTA_BITPACK || m == M_FLOAT_MULT || m == M_XORZ) {
    for (uint32_t k = threadIdx.x; k < nsub; k += blockDim.x) {
      const SubStats& R = ss[g0 + k];
      uint64_t pl = k ? ss[g0 + k - 1].last : 0;
      uint32_t w = 0;
      uint64_t mn = 0;
      if (m == M_FOR_BITPACK) {
        w = sgn ? bit_width64((uint64_t)R.smax - (uint64_t)R.smin) : bit_width64(R.umax - R.umin);
        mn = sgn ? (uint64_t)R.smin : R.umin;
      } else if (m == M_DELTA_BITPACK) {
        uint64_t dzf = k ? zigzag64(R.first - pl) : 0;
        uint64_t dmn = R.cnt > 1 ? u64min(R.dzmin, dzf) : dzf, dmx = R.cnt > 1 ? u64max(R.dzmax, dzf) : dzf;
        w = bit_width64(dmx - dmn);
        mn = dmn;
      } else if (m == M_FLOAT_MULT) {
        const FmStat& F = fms[g0 + k];
        w = bit_width64((uint64_t)F.kmax[fd.aux] - (uint64_t)F.kmin[fd.aux]);
        mn = (uint64_t)F.kmin[fd.aux];
      } else {
        S.subsz[k] = R.xb + varint_len(R.first ^ pl);
      }
      S.w_a[k] = (uint8_t)w;
      S.submin[k] = mn;
    }
    __syncthreads();
  }
  switch (fd.mode) {
    case M_RAW: emit_raw(v, n, dtype, out); break;
    case M_CONST:
      if (threadIdx.x == 0) put_u64(out, v[0]);
      break;
    case M_STRIDE:
      if (threadIdx.x == 0) {
        put_u64(out, v[0]);
        put_u64(out + 8, v[1] - v[0]);
      }
      break;
    case M_XORZ: emit_xorz(S, v, n, out); break;
    case M_FOR_BITPACK: block_for_write(S, out, n, [&](uint32_t i) { return v[i]; }); break;
    case M_DELTA_BITPACK:
      if (threadIdx.x == 0) put_u64(out, v[0]);
      block_for_write(S, out + 8, n, [&](uint32_t i) { return zigzag64(v[i] - (i ? v[i - 1] : v[0])); });
      break;
    case M_FLOAT_MULT: {
      int s = (int)fd.aux;
      bool coded = ENT && (er.flags & kEntFm);
      if (threadIdx.x == 0) {
        put_u8(out, coded ? 1 : 0);
        put_u8(out + 1, s);
      }
      if (coded) {
        uint32_t mb = fm_delta_bytes(S, v, n, s, scr);
        coded_write(S.ra, mb, [&](uint32_t i) { return (uint32_t)scr[i]; }, out + 2, er.fm);
      } else {
        block_for_write(S, out + 2, n, [&](uint32_t i) { return (uint64_t)fm_k(v[i], s); });
      }
      break;
    }
    case M_BYTE_TRANSPOSE:  // transpose.rs:10-32 (Balanced in-pool only)
      if (ENT)
        coded_write(S.ra, 8 * n, [&](uint32_t i) {
          uint32_t pl = i / n;
          return (uint32_t)(v[i - pl * n] >> (8 * pl)) & 255u;
        }, out, fd.plen);
      break;
    case M_ALP: emit_alp(S, v, n, ss ? ss + g0 : nullptr, out); break;
    case M_ALP_RD: emit_alprd(S, v, n, fd.aux, scr, out, erp); break;
    case M_DICT: emit_dict(S, v, n, ss + g0, scr, out, erp); break;
    case M_RLE: emit_rle(S, v, n, ss + g0, scr, out); break;
    default: break;
  }
}

// ---------------------------------------------------------------------------
// Window probe, block planning and frame offsets.
// ---------------------------------------------------------------------------

// Block plan (reference encoder.rs:154-178): fills frames[].value_off / .n.
constexpr int kPlanThreads = 1024;
__global__ void __launch_bounds__(kPlanThreads)
    k_plan(const uint8_t* __restrict__ grow, uint64_t n, uint64_t fixed_bs, FrameDesc* frames, uint32_t* nb) {
  if (fixed_bs) {
    uint64_t nblk = (n + fixed_bs - 1) / fixed_bs;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nblk; i += (uint64_t)gridDim.x * blockDim.x) {
      FrameDesc f;
      f.value_off = i * fixed_bs;
      f.n = (uint32_t)qmin(fixed_bs, n - f.value_off);
      f.payload_off = 0;
      f.plen = 0;
      f.mode = 0;
      f.aux = 0;
      frames[i] = f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *nb = (uint32_t)nblk;
    return;
  }
  // Adaptive: the block starts form a chain over the 32768-value windows
  // (grow -> +4 windows, else +1).  As a scan: the state before window w is
  // the number of windows still covered by the current block (0 = w starts a
  // block), and window w maps it by f_w(s) = s ? s - 1 : (grow[w] ? 3 : 0).
  // The maps compose (4 entries of 2 bits), so one CTA scans them in chunks
  // of 4096 windows, then compacts the starts into the frame table.
  if (blockIdx.x) return;
  constexpr int kPer = 4, kWarps = kPlanThreads / 32;
  __shared__ uint32_t s_wmap[kWarps], s_wcnt[kWarps];
  __shared__ uint32_t s_state, s_count;
  int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  uint64_t nwin = (n + kBaseQuantum - 1) / kBaseQuantum;
  if (t == 0) {
    s_state = 0;
    s_count = 0;
  }
  __syncthreads();
  auto apply = [](uint32_t m, uint32_t st) { return (m >> (2 * st)) & 3u; };
  auto compose = [&](uint32_t g, uint32_t f) {  // g after f
    uint32_t r = 0;
#pragma unroll
    for (uint32_t st = 0; st < 4; st++) r |= apply(g, apply(f, st)) << (2 * st);
    return r;
  };
  const uint32_t kId = 0u | (1u << 2) | (2u << 4) | (3u << 6);
  for (uint64_t w0 = 0; w0 < nwin; w0 += (uint64_t)kPlanThreads * kPer) {
    uint64_t wb = w0 + (uint64_t)t * kPer;
    uint8_t g[kPer];
    uint32_t m = kId;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      g[q] = wb + q < nwin ? grow[wb + q] : 0;
      uint32_t f = wb + q < nwin ? ((g[q] ? 3u : 0u) | (0u << 2) | (1u << 4) | (2u << 6)) : kId;
      m = compose(f, m);
    }
    // inclusive scan of the maps in window order
    uint32_t inc = m;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc = compose(inc, u);
    }
    if (lane == 31) s_wmap[warp] = inc;
    __syncthreads();
    uint32_t pre = kId;  // maps of the warps before this one
    for (int k = 0; k < warp; k++) pre = compose(s_wmap[k], pre);
    uint32_t ex = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) ex = kId;
    uint32_t st = apply(compose(ex, pre), s_state);  // state before window wb
    uint32_t starts = 0;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      if (wb + q < nwin && st == 0) starts |= 1u << q;
      if (wb + q < nwin) st = st ? st - 1 : (g[q] ? 3u : 0u);
    }
    uint32_t c = __popc(starts), ci = c;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(0xffffffffu, ci, o);
      if (lane >= o) ci += u;
    }
    if (lane == 31) s_wcnt[warp] = ci;
    __syncthreads();
    uint32_t base = s_count;
    for (int k = 0; k < warp; k++) base += s_wcnt[k];
    base += ci - c;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
      if (!(starts >> q & 1u)) continue;
      uint64_t s0 = (wb + q) * (uint64_t)kBaseQuantum;
      uint64_t end = g[q] ? qmin(s0 + kMaxBlock, n) : qmin(s0 + kBaseQuantum, n);
      FrameDesc f;
      f.value_off = s0;
      f.n = (uint32_t)(end - s0);
      f.payload_off = 0;
      f.plen = 0;
      f.mode = 0;
      f.aux = 0;
      frames[base++] = f;
    }
    __syncthreads();
    if (t == kPlanThreads - 1) {  // the last thread holds the chunk's final state
      s_state = st;
      uint32_t tot = 0;
      for (int k = 0; k < kWarps; k++) tot += s_wcnt[k];
      s_count += tot;
    }
    __syncthreads();
  }
  if (t == 0) *nb = s_count;
}

__global__ void k_frame_sizes(const FrameDesc* __restrict__ frames, const uint32_t* __restrict__ nbp, uint32_t maxb,
                              uint64_t* __restrict__ sizes) {
  uint32_t nb = *nbp;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < maxb; i += gridDim.x * blockDim.x)
    sizes[i] = i < nb ? 9ull + frames[i].plen : 0ull;
}
__global__ void k_frame_apply(FrameDesc* frames, const uint32_t* __restrict__ nbp, const uint64_t* __restrict__ offs,
                              const uint64_t* __restrict__ base_p) {
  uint32_t nb = *nbp;
  uint64_t base = *base_p;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x)
    frames[i].payload_off = base + offs[i] + 9;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static size_t enc_smem_bytes() { return sizeof(EncSmem); }

void launch_plan(const uint8_t* grow, uint64_t n, uint64_t fixed_bs, FrameDesc* frames, uint32_t* nb,
                 cudaStream_t st) {
  unsigned g = 1;
  if (fixed_bs) g = (unsigned)qmin(((n + fixed_bs - 1) / fixed_bs + kPlanThreads - 1) / kPlanThreads, 4096);
  if (g == 0) g = 1;
  k_plan<<<g, kPlanThreads, 0, st>>>(grow, n, fixed_bs, frames, nb);
  count_launches(1);
}

uint64_t sub_stats_items(uint64_t n, uint64_t fixed_bs) {
  if (fixed_bs) return ((n + fixed_bs - 1) / fixed_bs) * ((fixed_bs + kSub - 1) / kSub);
  return ((n + kBaseQuantum - 1) / kBaseQuantum) * (uint64_t)kStatsWarps;
}
uint64_t sub_stats_bytes() { return sizeof(SubStats); }
uint64_t fm_stats_bytes() { return sizeof(FmStat); }

void launch_sub_stats(const uint64_t* lane, uint64_t n, uint64_t fixed_bs, int dtype, int level, void* ss, void* fms,
                      uint64_t* smp16, uint8_t* grow, uint32_t* winbits, cudaStream_t st) {
  uint64_t items = sub_stats_items(n, fixed_bs);
  unsigned g = (unsigned)((items + kStatsWarps - 1) / kStatsWarps);
  if (!g) return;
  if (dtype_float(dtype)) {
    k_sub_stats<true><<<g, kStatsWarps * 32, 0, st>>>(lane, n, fixed_bs, dtype, level, (SubStats*)ss, (FmStat*)fms,
                                                       smp16, grow, winbits);
    if (level >= 1) {
      k_alp_stats<<<(unsigned)((items + kAlpWarps - 1) / kAlpWarps), kAlpWarps * 32, 0, st>>>(lane, n, fixed_bs, items,
                                                                                            (SubStats*)ss);
      count_launches(1);
    }
  } else
    k_sub_stats<false><<<g, kStatsWarps * 32, 0, st>>>(lane, n, fixed_bs, dtype, level, (SubStats*)ss,
                                                        (FmStat*)fms, nullptr, grow, winbits);
  count_launches(1);
}

void launch_decide(const uint64_t* lane, FrameDesc* frames, const uint32_t* nb, uint32_t max_blocks, uint64_t fixed_bs,
                   int dtype, int level, const void* ss, const void* fms, const uint64_t* smp16,
                   const uint32_t* winbits, uint8_t* scratch, void* ent, bool sample, cudaStream_t st) {
  int sm = (int)enc_smem_bytes();
  static std::atomic<unsigned long long> smem_set{0};
  once_per_device(smem_set, [sm] {
    cudaFuncSetAttribute(k_decide<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_decide<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_decide<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_emit<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    cudaFuncSetAttribute(k_emit<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
  });
  if (max_blocks) {
    if (ent)
      k_decide<true, false><<<max_blocks, kEncThreads, sm, st>>>(lane, frames, nb, fixed_bs, dtype, level,
                                                          (const SubStats*)ss, (const FmStat*)fms, smp16, winbits,
                                                          scratch, (EntRec*)ent);
    else if (sample)
      k_decide<false, true><<<max_blocks, kEncThreads, sm, st>>>(lane, frames, nb, fixed_bs, dtype, level,
                                                                 (const SubStats*)ss, (const FmStat*)fms, smp16,
                                                                 winbits, scratch, nullptr);
    else
      k_decide<false, false><<<max_blocks, kEncThreads, sm, st>>>(lane, frames, nb, fixed_bs, dtype, level,
                                                                  (const SubStats*)ss, (const FmStat*)fms, smp16,
                                                                  winbits, scratch, nullptr);
  }
  count_launches(max_blocks ? 1 : 0);
}

void launch_emit(const uint64_t* lane, const FrameDesc* frames, const uint32_t* nb, uint32_t max_blocks,
                 uint64_t fixed_bs, int dtype, const void* ss, const void* fms, uint8_t* scratch, uint8_t* out,
                 uint64_t out_cap, const void* ent, cudaStream_t st) {
  if (max_blocks) {
    if (ent)
      k_emit<true><<<max_blocks, kEncThreads, enc_smem_bytes(), st>>>(lane, frames, nb, fixed_bs, dtype,
                                                                      (const SubStats*)ss, (const FmStat*)fms,
                                                                      scratch, out, out_cap, (const EntRec*)ent);
    else
      k_emit<false><<<max_blocks, kEncThreads, enc_smem_bytes(), st>>>(lane, frames, nb, fixed_bs, dtype,
                                                                       (const SubStats*)ss, (const FmStat*)fms,
                                                                       scratch, out, out_cap, nullptr);
  }
  count_launches(max_blocks ? 1 : 0);
}

uint64_t ent_rec_bytes() { return sizeof(EntRec); }

unsigned long long* device_win_counters() {
  void* p = nullptr;
  cudaGetSymbolAddress(&p, g_wins);
  return reinterpret_cast<unsigned long long*>(p);
}

}  // namespace qb

#include "qb_scan.cuh"

namespace qb {
// At most kSmallWords frames in one CTA of 1,024 threads: k_frame_sizes, the
// exclusive scan and k_frame_apply in one launch.
__global__ void __launch_bounds__(1024) k_frame_offsets_small(FrameDesc* frames, const uint32_t* __restrict__ nbp,
                                                              const uint64_t* __restrict__ base_p,
                                                              uint64_t* __restrict__ total) {
  __shared__ uint64_t wsum[32];
  uint32_t nb = *nbp, t = threadIdx.x, l = t & 31, warp = t >> 5;
  uint64_t base = *base_p;
  uint64_t v[kSmallPer], s = 0;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t i = t * kSmallPer + k;
    v[k] = i < nb ? 9ull + frames[i].plen : 0ull;
    s += v[k];
  }
  uint64_t inc = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if ((int)l >= o) inc += u;
  }
  if (l == 31) wsum[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint64_t x = wsum[l];
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, x, o);
      if ((int)l >= o) x += u;
    }
    wsum[l] = x;
    if (l == 31) *total = x;
  }
  __syncthreads();
  uint64_t run = (warp ? wsum[warp - 1] : 0ull) + inc - s;
#pragma unroll
  for (uint32_t k = 0; k < kSmallPer; k++) {
    uint32_t i = t * kSmallPer + k;
    if (i < nb) frames[i].payload_off = base + run + 9;
    run += v[k];
  }
}

void launch_frame_offsets(FrameDesc* frames, const uint32_t* nb, uint32_t max_blocks, const uint64_t* base,
                          uint64_t* sizes_tmp, uint64_t* tile_tmp, uint64_t* total, cudaStream_t st) {
  if (max_blocks <= kSmallWords) {
    k_frame_offsets_small<<<1, 1024, 0, st>>>(frames, nb, base, total);
    count_launches(1);
    return;
  }
  unsigned g = (unsigned)qmin((max_blocks + 255) / 256, 1024);
  if (g == 0) g = 1;
  k_frame_sizes<<<g, 256, 0, st>>>(frames, nb, max_blocks, sizes_tmp);
  scan_exclusive_u64(sizes_tmp, sizes_tmp, max_blocks ? max_blocks : 1, tile_tmp, total, st);
  k_frame_apply<<<g, 256, 0, st>>>(frames, nb, sizes_tmp, base);
  count_launches(5);
}
}  // namespace qb
