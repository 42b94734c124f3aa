// Shared device helpers for the quoin B200 kernels: stream constants, bounded
// unaligned byte-stream loads, integer helpers and the exact FP64 operations the
// float codecs need (no contraction; every product/sum is an explicit
// round-to-nearest intrinsic so results equal the reference's IEEE doubles).
#pragma once
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace qb {

// Mode wire ids (reference src/mode.rs:23-67).
enum Mode : int {
  M_PRED = 0, M_CONST = 1, M_STRIDE = 2, M_XORZ = 3, M_LZ = 4, M_RAW = 5,
  M_ORDERED_DELTA = 7, M_ALP = 9, M_BYTE_TRANSPOSE = 11, M_FLOAT_MULT = 17,
  M_DICT = 19, M_DELTA2 = 20, M_PRED2 = 25, M_PRED_RC = 29, M_DELTA_DP = 45,
  M_FOR_BITPACK = 50, M_DELTA_BITPACK = 51, M_ALP_RD = 52, M_RLE = 53, M_PCO = 54
};

// Stream dtype wire ids (reference src/dtype.rs:68-78).
enum DType : int { DT_F64 = 0, DT_I64 = 1, DT_U64 = 2, DT_I32 = 3, DT_U32 = 4,
                   DT_F32 = 5, DT_DEC128 = 6, DT_DEC256 = 7 };

// Decode error kinds (reference src/error.rs:5-25); 0 = ok.
enum Err : uint32_t { E_OK = 0, E_BAD_MAGIC = 1, E_UNSUPPORTED_VERSION = 2,
                      E_TRUNCATED = 3, E_UNKNOWN_MODE = 4, E_CORRUPT = 5,
                      E_LENGTH_MISMATCH = 6, E_UNSUPPORTED_DTYPE = 7,
                      E_DTYPE_MISMATCH = 8, E_UNSUPPORTED = 9,
                      E_NO_ENTROPY_AREA = 10 };  // entropy-coded part, no device area given

constexpr int kSub = 1024;              // FastLanes sub-block (reference bitpack.rs:22)
constexpr int kMaxBlock = 131072;       // reference format.rs:44
constexpr int kBaseQuantum = 32768;     // reference encoder.rs:144

__host__ __device__ inline uint64_t qmin(uint64_t a, uint64_t b) { return a < b ? a : b; }
__host__ __device__ inline uint64_t qmax(uint64_t a, uint64_t b) { return a > b ? a : b; }

__host__ __device__ inline uint32_t lane_bytes(int dt) {
  return (dt == DT_I32 || dt == DT_U32 || dt == DT_F32) ? 4u : 8u;
}
__host__ __device__ inline bool dtype_signed(int dt) { return dt == DT_I32 || dt == DT_I64; }
__host__ __device__ inline bool dtype_float(int dt) { return dt == DT_F64 || dt == DT_F32; }

__host__ __device__ inline uint32_t varint_len(uint64_t v) {
#ifdef __CUDA_ARCH__
  uint32_t bits = 64u - (uint32_t)__clzll((long long)(v | 1ull));
#else
  uint32_t bits = 64u - (uint32_t)__builtin_clzll(v | 1ull);
#endif
  return (bits + 6u) / 7u;
}
__host__ __device__ inline uint64_t zigzag64(uint64_t n) { return (n << 1) ^ (uint64_t)((int64_t)n >> 63); }
__host__ __device__ inline uint64_t unzigzag64(uint64_t z) { return (z >> 1) ^ (0ull - (z & 1ull)); }

__device__ inline uint32_t bit_width64(uint64_t range) {
  return range == 0 ? 0u : 64u - (uint32_t)__clzll((long long)range);
}

// Runs f() once per device and process: kernel attributes belong to the
// device's context, so each device is configured on first use, and the calls
// (driver calls that take the context's lock) stay off the per-column path.
template <class F>
inline void once_per_device(std::atomic<unsigned long long>& done, F f) {
  int dev = 0;
  cudaGetDevice(&dev);
  unsigned long long bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return;
  f();
  done.fetch_or(bit, std::memory_order_release);
}

// ---------------------------------------------------------------------------
// Unaligned little-endian loads from a byte stream.  Each helper touches only
// the naturally aligned words that overlap the requested bytes, so a load of
// the last bytes of a buffer never reaches past the word holding its last byte.
// ---------------------------------------------------------------------------
__device__ inline uint32_t ld_u32(const uint8_t* p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  uint32_t s = (uint32_t)(a & 3u);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~(uintptr_t)3);
  uint32_t lo = __ldg(w);
  if (s == 0) return lo;
  uint32_t hi = __ldg(w + 1);
  return __funnelshift_r(lo, hi, s * 8u);
}
__device__ inline uint64_t ld_u64(const uint8_t* p) {
  uintptr_t a = reinterpret_cast<uintptr_t>(p);
  uint32_t s = (uint32_t)(a & 3u);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~(uintptr_t)3);
  uint32_t w0 = __ldg(w), w1 = __ldg(w + 1);
  if (s == 0) return (uint64_t)w0 | ((uint64_t)w1 << 32);
  uint32_t w2 = __ldg(w + 2);
  uint32_t lo = __funnelshift_r(w0, w1, s * 8u), hi = __funnelshift_r(w1, w2, s * 8u);
  return (uint64_t)lo | ((uint64_t)hi << 32);
}
__device__ inline uint16_t ld_u16(const uint8_t* p) {
  return (uint16_t)(p[0] | ((uint32_t)p[1] << 8));
}

// Bounded LEB128 read (reference varint.rs:24-39).  Returns E_OK/E_TRUNCATED/E_CORRUPT.
__device__ inline uint32_t rd_varint(const uint8_t* p, uint64_t len, uint64_t* pos, uint64_t* out) {
  uint64_t r = 0;
  uint32_t shift = 0;
  for (;;) {
    if (*pos >= len) return E_TRUNCATED;
    uint8_t b = p[(*pos)++];
    r |= (uint64_t)(b & 0x7f) << shift;
    if (!(b & 0x80)) { *out = r; return E_OK; }
    shift += 7;
    if (shift >= 64) return E_CORRUPT;
  }
}

// ---------------------------------------------------------------------------
// Exact FP64 helpers.
// ---------------------------------------------------------------------------
__device__ inline double as_f64(uint64_t b) { return __longlong_as_double((long long)b); }
__device__ inline uint64_t f64_bits(double d) { return (uint64_t)__double_as_longlong(d); }

// Powers of ten as correctly rounded doubles (reference codecs/alp.rs:23-30).
__constant__ static double kExp10[19] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8, 1e9,
                                         1e10, 1e11, 1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18};
__constant__ static double kFrac10[19] = {1e0,   1e-1,  1e-2,  1e-3,  1e-4,  1e-5,  1e-6,
                                          1e-7,  1e-8,  1e-9,  1e-10, 1e-11, 1e-12, 1e-13,
                                          1e-14, 1e-15, 1e-16, 1e-17, 1e-18};
__constant__ static double kFmScales[7] = {10.0, 100.0, 1000.0, 10000.0, 100000.0, 1000000.0, 10000000.0};

// Rust `f64 as i64`: truncate toward zero, saturate, NaN -> 0.
__device__ inline int64_t f64_as_i64(double x) {
  if (x != x) return 0;
  if (x >= 9223372036854775808.0) return INT64_MAX;
  if (x < -9223372036854775808.0) return INT64_MIN;
  return __double2ll_rz(x);
}
__device__ inline bool is_finite_f64(double x) { return (f64_bits(x) & 0x7FF0000000000000ull) != 0x7FF0000000000000ull; }

// ALP digit encode/decode (reference codecs/alp.rs:32-44), evaluated left to right.
__device__ inline bool alp_encode_value(double v, int e, int f, int64_t* d) {
  double tmp = __dmul_rn(__dmul_rn(v, kExp10[e]), kFrac10[f]);
  const double kUpper = 9.223372036854776e18, kMagic = 6755399441055744.0;
  if (!is_finite_f64(tmp) || tmp >= kUpper || tmp <= -kUpper) return false;
  *d = f64_as_i64(__dadd_rn(__dadd_rn(tmp, kMagic), -kMagic));
  return true;
}
__device__ inline double alp_decode_value(int64_t d, int e, int f) {
  return __dmul_rn(__dmul_rn(__ll2double_rn(d), kExp10[f]), kFrac10[e]);
}
__device__ inline bool alp_roundtrips(uint64_t bits, int e, int f, int64_t* d) {
  return alp_encode_value(as_f64(bits), e, f, d) && f64_bits(alp_decode_value(*d, e, f)) == bits;
}

// alp_roundtrips without the integer conversions: the digit is kept as the
// integral double r it is cast from.  |r| <= 2^63, and (f64)(r as i64) == r
// (r = 2^63 saturates to i64::MAX, whose f64 is 2^63 again), so decoding from
// r equals decoding from the digit, and r orders like the digit.
__device__ inline bool alp_roundtrips_r(uint64_t bits, int e, int f, double* r) {
  double tmp = __dmul_rn(__dmul_rn(as_f64(bits), kExp10[e]), kFrac10[f]);
  const double kUpper = 9.223372036854776e18, kMagic = 6755399441055744.0;
  if (!is_finite_f64(tmp) || tmp >= kUpper || tmp <= -kUpper) return false;
  double rr = __dadd_rn(__dadd_rn(tmp, kMagic), -kMagic);
  *r = rr;
  return f64_bits(__dmul_rn(__dmul_rn(rr, kExp10[f]), kFrac10[e])) == bits;
}

// f64::round (half away from zero), written from its definition: trunc, then
// step away from zero when the discarded fraction is at least one half.  The
// subtraction x - trunc(x) is exact for every finite double.
__device__ inline double round_half_away(double x) {
  double t = trunc(x);
  double frac = __dadd_rn(x, -t);
  if (fabs(frac) >= 0.5) t = __dadd_rn(t, copysign(1.0, x));
  return t;
}

// f32 -> f64 widening and f64 -> f32 narrowing with the x86-64 SSE NaN rules
// the reference's `as` casts compile to: a NaN keeps its payload (shifted) and
// gets its quiet bit set.  Non-NaN values use the exact hardware conversions.
__device__ inline uint64_t f32bits_to_f64bits(uint32_t b) {
  if ((b & 0x7F800000u) == 0x7F800000u && (b & 0x007FFFFFu)) {
    uint64_t sign = (uint64_t)(b >> 31) << 63;
    uint64_t mant = (uint64_t)(b & 0x007FFFFFu) << 29;
    return sign | 0x7FF0000000000000ull | mant | 0x0008000000000000ull;
  }
  return f64_bits((double)__uint_as_float(b));
}
__device__ inline uint32_t f64bits_to_f32bits(uint64_t w) {
  if ((w & 0x7FF0000000000000ull) == 0x7FF0000000000000ull && (w & 0x000FFFFFFFFFFFFFull)) {
    uint32_t sign = (uint32_t)(w >> 63) << 31;
    uint32_t mant = (uint32_t)((w & 0x000FFFFFFFFFFFFFull) >> 29);
    return sign | 0x7F800000u | 0x00400000u | mant;
  }
  return __float_as_uint(__double2float_rn(as_f64(w)));
}

// ---------------------------------------------------------------------------
// Warp / block reductions.
// ---------------------------------------------------------------------------
template <typename T>
__device__ inline T warp_min(T v) {
  for (int o = 16; o; o >>= 1) { T u = __shfl_xor_sync(0xffffffffu, v, o); v = u < v ? u : v; }
  return v;
}
template <typename T>
__device__ inline T warp_max(T v) {
  for (int o = 16; o; o >>= 1) { T u = __shfl_xor_sync(0xffffffffu, v, o); v = u > v ? u : v; }
  return v;
}
template <typename T>
__device__ inline T warp_sum(T v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline uint32_t warp_and(uint32_t v) {
  for (int o = 16; o; o >>= 1) v &= __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Inclusive warp prefix sum.
template <typename T>
__device__ inline T warp_incl_scan(T v) {
  int lane = threadIdx.x & 31;
  for (int o = 1; o < 32; o <<= 1) {
    T u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  return v;
}

}  // namespace qb
