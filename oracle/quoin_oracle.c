/*
 * quoin oracle — plain-C CPU restatement of the reference's in-path
 * algorithm.  TEST INFRASTRUCTURE ONLY: the checker for the GPU product and
 * the timed CPU baseline.  The product never links or calls this file.
 *
 * Parity status: "parity unpinned" at the byte level — no Rust toolchain or
 * crate cache exists here, and the reference's tests carry no golden streams.
 * The restatement follows each cited reference line; the reference's
 * known-answer tests (header bytes, Fastest ratio floors, codec size bounds,
 * round trips) are ported in tests/ and pin what they can.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the reference project root).  Build: make -C oracle  (gcc -O2
 * -ffp-contract=off; FP64 must not be contracted, matching rustc).
 */
#define _GNU_SOURCE
#include "quoin_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Growable buffers                                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint8_t *p;
    size_t len, cap;
} buf_t;

static void b_reserve(buf_t *b, size_t add) {
    if (b->len + add <= b->cap) return;
    size_t nc = b->cap ? b->cap : 64;
    while (nc < b->len + add) nc *= 2;
    b->p = (uint8_t *)realloc(b->p, nc);
    b->cap = nc;
}
static void b_push(buf_t *b, uint8_t v) {
    b_reserve(b, 1);
    b->p[b->len++] = v;
}
static void b_write(buf_t *b, const void *src, size_t n) {
    if (!n) return;
    b_reserve(b, n);
    memcpy(b->p + b->len, src, n);
    b->len += n;
}
static void b_u16(buf_t *b, uint16_t v) {
    uint8_t t[2] = {(uint8_t)v, (uint8_t)(v >> 8)};
    b_write(b, t, 2);
}
static void b_u32(buf_t *b, uint32_t v) {
    uint8_t t[4];
    for (int i = 0; i < 4; i++) t[i] = (uint8_t)(v >> (8 * i));
    b_write(b, t, 4);
}
static void b_u64(buf_t *b, uint64_t v) {
    uint8_t t[8];
    for (int i = 0; i < 8; i++) t[i] = (uint8_t)(v >> (8 * i));
    b_write(b, t, 8);
}
static void b_free(buf_t *b) {
    free(b->p);
    b->p = NULL;
    b->len = b->cap = 0;
}

static uint64_t rd_u64(const uint8_t *p) {
    uint64_t v = 0;
    for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
    return v;
}
static uint32_t rd_u32(const uint8_t *p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static uint16_t rd_u16(const uint8_t *p) { return (uint16_t)(p[0] | (p[1] << 8)); }

static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static uint32_t bit_width(uint64_t range) { return range == 0 ? 0 : (uint32_t)(64 - clz64(range)); }

/* ------------------------------------------------------------------------ */
/* varint — src/varint.rs:9-39                                               */
/* ------------------------------------------------------------------------ */

static void b_varint(buf_t *b, uint64_t v) {
    for (;;) {
        uint8_t byte = (uint8_t)(v & 0x7f);
        v >>= 7;
        if (v) {
            b_push(b, byte | 0x80);
        } else {
            b_push(b, byte);
            return;
        }
    }
}
static size_t varint_len(uint64_t v) {
    size_t n = 1;
    while (v >= 0x80) {
        v >>= 7;
        n++;
    }
    return n;
}
/* src/varint.rs:24-39 */
static int varint_read(const uint8_t *in, size_t len, size_t *pos, uint64_t *out) {
    uint64_t r = 0;
    unsigned shift = 0;
    for (;;) {
        if (*pos >= len) return OQ_TRUNCATED;
        uint8_t byte = in[(*pos)++];
        r |= (uint64_t)(byte & 0x7f) << shift;
        if (!(byte & 0x80)) {
            *out = r;
            return OQ_OK;
        }
        shift += 7;
        if (shift >= 64) return OQ_CORRUPT;
    }
}

/* ------------------------------------------------------------------------ */
/* FastLanes bit-packing — src/bitpack.rs:48-161                             */
/* ------------------------------------------------------------------------ */

static uint32_t mask32(uint32_t w) { return w >= 32 ? 0xFFFFFFFFu : ((1u << w) - 1); }
static uint64_t mask64(uint32_t w) { return w >= 64 ? ~0ull : ((1ull << w) - 1); }

/* bitpack.rs:49-75 */
void oq_pack32(const uint32_t *values, uint32_t width, uint32_t *out) {
    memset(out, 0, sizeof(uint32_t) * 32 * width);
    if (width == 0) return;
    uint32_t m = mask32(width);
    for (uint32_t r = 0; r < 32; r++) {
        uint32_t bit_off = r * width, word = bit_off / 32, shift = bit_off % 32;
        for (uint32_t l = 0; l < 32; l++) {
            uint32_t v = values[r * 32 + l] & m;
            out[word * 32 + l] |= v << shift;
            if (shift + width > 32) out[(word + 1) * 32 + l] |= v >> (32 - shift);
        }
    }
}
/* bitpack.rs:79-103 */
void oq_unpack32(const uint32_t *packed, uint32_t width, uint32_t *out) {
    if (width == 0) {
        memset(out, 0, 4096);
        return;
    }
    uint32_t m = mask32(width);
    for (uint32_t r = 0; r < 32; r++) {
        uint32_t bit_off = r * width, word = bit_off / 32, shift = bit_off % 32;
        for (uint32_t l = 0; l < 32; l++) {
            uint32_t lo = packed[word * 32 + l];
            uint32_t v;
            if (shift + width > 32)
                v = (lo >> shift) | (packed[(word + 1) * 32 + l] << (32 - shift));
            else
                v = lo >> shift;
            out[r * 32 + l] = v & m;
        }
    }
}
/* bitpack.rs:107-133 */
void oq_pack64(const uint64_t *values, uint32_t width, uint64_t *out) {
    memset(out, 0, sizeof(uint64_t) * 16 * width);
    if (width == 0) return;
    uint64_t m = mask64(width);
    for (uint32_t r = 0; r < 64; r++) {
        uint32_t bit_off = r * width, word = bit_off / 64, shift = bit_off % 64;
        for (uint32_t l = 0; l < 16; l++) {
            uint64_t v = values[r * 16 + l] & m;
            out[word * 16 + l] |= v << shift;
            if (shift + width > 64) out[(word + 1) * 16 + l] |= v >> (64 - shift);
        }
    }
}
/* bitpack.rs:137-161 */
void oq_unpack64(const uint64_t *packed, uint32_t width, uint64_t *out) {
    if (width == 0) {
        memset(out, 0, 8192);
        return;
    }
    uint64_t m = mask64(width);
    for (uint32_t r = 0; r < 64; r++) {
        uint32_t bit_off = r * width, word = bit_off / 64, shift = bit_off % 64;
        for (uint32_t l = 0; l < 16; l++) {
            uint64_t lo = packed[word * 16 + l];
            uint64_t v;
            if (shift + width > 64)
                v = (lo >> shift) | (packed[(word + 1) * 16 + l] << (64 - shift));
            else
                v = lo >> shift;
            out[r * 16 + l] = v & m;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* FOR_BITPACK — src/codecs/for_bitpack.rs:25-157                            */
/* ------------------------------------------------------------------------ */

/* for_bitpack.rs:47-96 */
static void for_encode_sub(const uint64_t *sub, size_t n, bool is_signed, buf_t *out) {
    uint64_t min, range;
    if (is_signed) {
        int64_t mn = INT64_MAX, mx = INT64_MIN;
        for (size_t i = 0; i < n; i++) {
            int64_t s = (int64_t)sub[i];
            if (s < mn) mn = s;
            if (s > mx) mx = s;
        }
        min = (uint64_t)mn;
        range = (uint64_t)mx - (uint64_t)mn;
    } else {
        uint64_t mn = ~0ull, mx = 0;
        for (size_t i = 0; i < n; i++) {
            if (sub[i] < mn) mn = sub[i];
            if (sub[i] > mx) mx = sub[i];
        }
        min = mn;
        range = mx - mn;
    }
    uint32_t width = bit_width(range);
    b_push(out, (uint8_t)width);
    b_u64(out, min);
    if (width == 0) return;
    if (width <= 32) {
        uint32_t res[1024] = {0};
        uint32_t packed[32 * 32];
        for (size_t k = 0; k < n; k++) res[k] = (uint32_t)(sub[k] - min);
        oq_pack32(res, width, packed);
        for (uint32_t w = 0; w < 32 * width; w++) b_u32(out, packed[w]);
    } else {
        uint64_t res[1024] = {0};
        uint64_t packed[16 * 64];
        for (size_t k = 0; k < n; k++) res[k] = sub[k] - min;
        oq_pack64(res, width, packed);
        for (uint32_t w = 0; w < 16 * width; w++) b_u64(out, packed[w]);
    }
}
/* for_bitpack.rs:25-35 */
static void for_encode(const uint64_t *vals, size_t n, bool is_signed, buf_t *out) {
    b_varint(out, n);
    for (size_t i = 0; i < n; i += 1024) {
        size_t end = i + 1024 < n ? i + 1024 : n;
        for_encode_sub(vals + i, end - i, is_signed, out);
    }
}
/* for_bitpack.rs:108-157.  `out` must hold n_values words. */
static int for_decode(const uint8_t *p, size_t plen, size_t n_values, bool is_signed, uint64_t *out) {
    (void)is_signed; /* unresidual is the same wrapping add either way */
    size_t pos = 0;
    uint64_t n64;
    int rc = varint_read(p, plen, &pos, &n64);
    if (rc) return rc;
    if (n64 != (uint64_t)n_values) return OQ_CORRUPT;
    size_t n = n_values, got = 0;
    while (got < n) {
        if (pos >= plen) return OQ_TRUNCATED;
        uint8_t width = p[pos++];
        if (width > 64) return OQ_CORRUPT;
        size_t count = n - got < 1024 ? n - got : 1024;
        if (plen - pos < 8) return OQ_TRUNCATED;
        uint64_t min = rd_u64(p + pos);
        pos += 8;
        if (width == 0) {
            for (size_t k = 0; k < count; k++) out[got + k] = min;
        } else if (width <= 32) {
            size_t nwords = 32 * (size_t)width;
            if (plen - pos < nwords * 4) return OQ_TRUNCATED;
            uint32_t packed[32 * 32], res[1024];
            for (size_t k = 0; k < nwords; k++) packed[k] = rd_u32(p + pos + 4 * k);
            pos += nwords * 4;
            oq_unpack32(packed, width, res);
            for (size_t k = 0; k < count; k++) out[got + k] = min + (uint64_t)res[k];
        } else {
            size_t nwords = 16 * (size_t)width;
            if (plen - pos < nwords * 8) return OQ_TRUNCATED;
            uint64_t packed[16 * 64], res[1024];
            for (size_t k = 0; k < nwords; k++) packed[k] = rd_u64(p + pos + 8 * k);
            pos += nwords * 8;
            oq_unpack64(packed, width, res);
            for (size_t k = 0; k < count; k++) out[got + k] = min + res[k];
        }
        got += count;
    }
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* DELTA_BITPACK — src/codecs/delta_bitpack.rs:32-64                         */
/* ------------------------------------------------------------------------ */

static uint64_t zigzag64(uint64_t n) { return (n << 1) ^ (uint64_t)((int64_t)n >> 63); }
static uint64_t unzigzag64(uint64_t z) { return (z >> 1) ^ (0 - (z & 1)); }

/* delta_bitpack.rs:32-46 */
static void delta_encode(const uint64_t *vals, size_t n, buf_t *out) {
    uint64_t base = n ? vals[0] : 0;
    b_u64(out, base);
    uint64_t *d = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    uint64_t prev = base;
    for (size_t i = 0; i < n; i++) {
        d[i] = zigzag64(vals[i] - prev);
        prev = vals[i];
    }
    for_encode(d, n, false, out);
    free(d);
}
/* delta_bitpack.rs:48-64 */
static int delta_decode(const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    if (plen < 8) return OQ_TRUNCATED;
    uint64_t base = rd_u64(p);
    int rc = for_decode(p + 8, plen - 8, n, false, out);
    if (rc) return rc;
    uint64_t prev = base;
    for (size_t i = 0; i < n; i++) {
        prev += unzigzag64(out[i]);
        out[i] = prev;
    }
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* RAW / CONST / STRIDE / XORZ — src/codecs/{raw,const_block,stride,xorz}.rs */
/* ------------------------------------------------------------------------ */

static size_t lane_bytes(int dtype) {
    return (dtype == OQ_I32 || dtype == OQ_U32 || dtype == OQ_F32) ? 4 : 8; /* dtype.rs:110-115 */
}
static bool dtype_signed(int dtype) { return dtype == OQ_I32 || dtype == OQ_I64; } /* dtype.rs:121-123 */
static bool dtype_float(int dtype) { return dtype == OQ_F64 || dtype == OQ_F32; }  /* dtype.rs:95-102 */

static uint32_t f64bits_to_f32bits(uint64_t w) {
    double d;
    memcpy(&d, &w, 8);
    float f = (float)d; /* Rust `as f32`: cvtsd2ss on x86-64 */
    uint32_t r;
    memcpy(&r, &f, 4);
    return r;
}
static uint64_t f32bits_to_f64bits(uint32_t b) {
    float f;
    memcpy(&f, &b, 4);
    double d = (double)f; /* Rust `as f64`: cvtss2sd on x86-64 */
    uint64_t r;
    memcpy(&r, &d, 8);
    return r;
}

/* raw.rs:12-28 */
static void raw_encode(const uint64_t *v, size_t n, int dtype, buf_t *out) {
    if (dtype == OQ_F32) {
        for (size_t i = 0; i < n; i++) b_u32(out, f64bits_to_f32bits(v[i]));
        return;
    }
    size_t lb = lane_bytes(dtype);
    b_reserve(out, n * lb);
    for (size_t i = 0; i < n; i++)
        for (size_t k = 0; k < lb; k++) out->p[out->len++] = (uint8_t)(v[i] >> (8 * k));
}
/* raw.rs:30-48 */
static int raw_decode(const uint8_t *p, size_t plen, size_t n, int dtype, uint64_t *out) {
    size_t lb = lane_bytes(dtype);
    if (plen != n * lb) return OQ_CORRUPT;
    for (size_t i = 0; i < n; i++) {
        if (dtype == OQ_F32)
            out[i] = f32bits_to_f64bits(rd_u32(p + 4 * i));
        else if (lb == 4)
            out[i] = rd_u32(p + 4 * i);
        else
            out[i] = rd_u64(p + 8 * i);
    }
    return OQ_OK;
}
/* const_block.rs:5-12 */
static bool const_encode(const uint64_t *v, size_t n, buf_t *out) {
    if (n == 0) return false;
    for (size_t i = 1; i < n; i++)
        if (v[i] != v[0]) return false;
    b_u64(out, v[0]);
    return true;
}
/* stride.rs:6-22 */
static bool stride_encode(const uint64_t *v, size_t n, buf_t *out) {
    if (n < 2) return false;
    uint64_t first = v[0], stride = v[1] - v[0];
    for (size_t i = 0; i < n; i++)
        if (v[i] != first + (uint64_t)i * stride) return false;
    b_u64(out, first);
    b_u64(out, stride);
    return true;
}
/* xorz.rs:8-16 */
static void xorz_encode(const uint64_t *v, size_t n, buf_t *out) {
    uint64_t prev = 0;
    for (size_t i = 0; i < n; i++) {
        b_varint(out, v[i] ^ prev);
        prev = v[i];
    }
}
/* xorz.rs:18-32 */
static int xorz_decode(const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    uint64_t prev = 0;
    size_t pos = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t x;
        int rc = varint_read(p, plen, &pos, &x);
        if (rc) return rc;
        prev ^= x;
        out[i] = prev;
    }
    if (pos != plen) return OQ_CORRUPT;
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* ALP — src/codecs/alp.rs:18-248                                            */
/* ------------------------------------------------------------------------ */

#define ALP_MAX_EXP 18
static const double ALP_MAGIC = 6755399441055744.0;     /* alp.rs:20 */
static const double ALP_UPPER = 9.223372036854776e18;   /* alp.rs:21 */
static const double EXP10[19] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8, 1e9,
                                 1e10, 1e11, 1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18};
static const double FRAC10[19] = {1e0,   1e-1,  1e-2,  1e-3,  1e-4,  1e-5,  1e-6,
                                  1e-7,  1e-8,  1e-9,  1e-10, 1e-11, 1e-12, 1e-13,
                                  1e-14, 1e-15, 1e-16, 1e-17, 1e-18};

static double as_f64(uint64_t b) {
    double d;
    memcpy(&d, &b, 8);
    return d;
}
static uint64_t f64_bits(double d) {
    uint64_t b;
    memcpy(&b, &d, 8);
    return b;
}
/* Rust `f64 as i64`: truncate, saturate, NaN -> 0. */
static int64_t f64_as_i64(double x) {
    if (x != x) return 0;
    if (x >= 9223372036854775808.0) return INT64_MAX;
    if (x < -9223372036854775808.0) return INT64_MIN;
    return (int64_t)x;
}
/* alp.rs:32-39 */
static bool alp_encode_value(double v, int e, int f, int64_t *d) {
    double tmp = v * EXP10[e] * FRAC10[f];
    if (!isfinite(tmp) || tmp >= ALP_UPPER || tmp <= -ALP_UPPER) return false;
    *d = f64_as_i64(tmp + ALP_MAGIC - ALP_MAGIC);
    return true;
}
/* alp.rs:41-44 */
static double alp_decode_value(int64_t d, int e, int f) { return (double)d * EXP10[f] * FRAC10[e]; }
static bool alp_roundtrips(uint64_t bits, int e, int f, int64_t *d) {
    return alp_encode_value(as_f64(bits), e, f, d) && f64_bits(alp_decode_value(*d, e, f)) == bits;
}
/* alp.rs:49-91 */
static bool alp_find_ef(const uint64_t *sub, size_t n, int *be, int *bf) {
    size_t stride = n / 32 ? n / 32 : 1;
    uint64_t sample[32];
    size_t sl = 0;
    for (size_t i = 0; i < n && sl < 32; i += stride) sample[sl++] = sub[i];
    int bbe = 0, bbf = 0;
    size_t best_cost = SIZE_MAX, best_exc = sl;
    for (int e = 0; e <= ALP_MAX_EXP; e++) {
        for (int f = 0; f <= e; f++) {
            size_t exc = 0;
            int64_t lo = INT64_MAX, hi = INT64_MIN;
            for (size_t k = 0; k < sl; k++) {
                int64_t d;
                if (alp_roundtrips(sample[k], e, f, &d)) {
                    if (d < lo) lo = d;
                    if (d > hi) hi = d;
                } else {
                    exc++;
                }
            }
            size_t width;
            if (exc == sl || hi <= lo)
                width = exc == sl ? 64 : 0;
            else
                width = bit_width((uint64_t)hi - (uint64_t)lo);
            size_t cost = width * sl + exc * 80;
            if (cost < best_cost) {
                best_cost = cost;
                bbe = e;
                bbf = f;
                best_exc = exc;
            }
        }
    }
    if (best_exc * 2 > sl) return false;
    *be = bbe;
    *bf = bbf;
    return true;
}
/* alp.rs:108-166 */
static bool alp_encode_sub(const uint64_t *sub, size_t n, buf_t *out) {
    int e, f;
    if (!alp_find_ef(sub, n, &e, &f)) return false;
    int64_t digits[1024];
    uint16_t exc_pos[1024];
    uint64_t exc_bits[1024];
    size_t nexc = 0;
    bool have_first = false;
    int64_t first = 0;
    for (size_t k = 0; k < n; k++) {
        int64_t d;
        if (alp_roundtrips(sub[k], e, f, &d)) {
            digits[k] = d;
            if (!have_first) {
                have_first = true;
                first = d;
            }
        } else {
            exc_pos[nexc] = (uint16_t)k;
            exc_bits[nexc] = sub[k];
            nexc++;
        }
    }
    int64_t filler = have_first ? first : 0;
    for (size_t x = 0; x < nexc; x++) digits[exc_pos[x]] = filler;
    for (size_t k = n; k < 1024; k++) digits[k] = filler;
    int64_t mn = digits[0], mx = digits[0];
    for (size_t k = 1; k < 1024; k++) {
        if (digits[k] < mn) mn = digits[k];
        if (digits[k] > mx) mx = digits[k];
    }
    uint32_t width = bit_width((uint64_t)mx - (uint64_t)mn);
    if (width > 32) return false;
    b_push(out, (uint8_t)e);
    b_push(out, (uint8_t)f);
    b_u16(out, (uint16_t)nexc);
    b_u64(out, (uint64_t)mn);
    b_push(out, (uint8_t)width);
    if (width > 0) {
        uint32_t res[1024], packed[32 * 32];
        for (size_t k = 0; k < 1024; k++) res[k] = (uint32_t)((uint64_t)digits[k] - (uint64_t)mn);
        oq_pack32(res, width, packed);
        for (uint32_t w = 0; w < 32 * width; w++) b_u32(out, packed[w]);
    }
    for (size_t x = 0; x < nexc; x++) {
        b_u16(out, exc_pos[x]);
        b_u64(out, exc_bits[x]);
    }
    return true;
}
/* alp.rs:93-106 */
static bool alp_encode(const uint64_t *v, size_t n, buf_t *out) {
    if (n == 0) return false;
    b_varint(out, n);
    for (size_t i = 0; i < n; i += 1024) {
        size_t end = i + 1024 < n ? i + 1024 : n;
        if (!alp_encode_sub(v + i, end - i, out)) return false;
    }
    return true;
}
/* alp.rs:168-248 */
static int alp_decode(const uint8_t *p, size_t plen, size_t n_values, uint64_t *out) {
    size_t pos = 0;
    uint64_t n64;
    int rc = varint_read(p, plen, &pos, &n64);
    if (rc) return rc;
    if (n64 != (uint64_t)n_values) return OQ_CORRUPT;
    size_t n = n_values, got = 0;
    while (got < n) {
        if (pos >= plen) return OQ_TRUNCATED;
        int e = p[pos];
        if (pos + 1 >= plen) return OQ_TRUNCATED;
        int f = p[pos + 1];
        if (e > ALP_MAX_EXP || f > e) return OQ_CORRUPT;
        if (plen < pos + 4) return OQ_TRUNCATED;
        size_t exc_count = rd_u16(p + pos + 2);
        if (plen < pos + 12) return OQ_TRUNCATED;
        int64_t min = (int64_t)rd_u64(p + pos + 4);
        if (pos + 12 >= plen) return OQ_TRUNCATED;
        uint32_t width = p[pos + 12];
        pos += 13;
        if (width > 32) return OQ_CORRUPT;
        size_t count = n - got < 1024 ? n - got : 1024;
        int64_t digits[1024];
        if (width > 0) {
            size_t nwords = 32 * (size_t)width;
            if (plen - pos < nwords * 4) return OQ_TRUNCATED;
            uint32_t packed[32 * 32], res[1024];
            for (size_t k = 0; k < nwords; k++) packed[k] = rd_u32(p + pos + 4 * k);
            pos += nwords * 4;
            oq_unpack32(packed, width, res);
            for (size_t k = 0; k < 1024; k++) digits[k] = (int64_t)((uint64_t)min + (uint64_t)res[k]);
        } else {
            for (size_t k = 0; k < 1024; k++) digits[k] = min;
        }
        for (size_t k = 0; k < count; k++) out[got + k] = f64_bits(alp_decode_value(digits[k], e, f));
        for (size_t x = 0; x < exc_count; x++) {
            if (plen < pos + 2) return OQ_TRUNCATED;
            size_t ep = rd_u16(p + pos);
            if (plen < pos + 10) return OQ_TRUNCATED;
            uint64_t bits = rd_u64(p + pos + 2);
            pos += 10;
            if (ep >= count) return OQ_CORRUPT;
            out[got + ep] = bits;
        }
        got += count;
    }
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* Hash map u64 -> u32 (counting / code assignment helper)                   */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t *keys;
    uint32_t *vals;
    uint8_t *used;
    size_t cap, len;
} hmap_t;

static void hm_init(hmap_t *h, size_t expect) {
    size_t cap = 16;
    while (cap < expect * 2) cap *= 2;
    h->cap = cap;
    h->len = 0;
    h->keys = (uint64_t *)malloc(cap * 8);
    h->vals = (uint32_t *)malloc(cap * 4);
    h->used = (uint8_t *)calloc(cap, 1);
}
static void hm_free(hmap_t *h) {
    free(h->keys);
    free(h->vals);
    free(h->used);
}
static size_t hm_slot(const hmap_t *h, uint64_t k) {
    size_t i = (size_t)((k * 0x9E3779B97F4A7C15ull) >> 20) & (h->cap - 1);
    while (h->used[i] && h->keys[i] != k) i = (i + 1) & (h->cap - 1);
    return i;
}
static void hm_grow(hmap_t *h) {
    hmap_t g;
    hm_init(&g, h->cap);
    for (size_t i = 0; i < h->cap; i++)
        if (h->used[i]) {
            size_t s = hm_slot(&g, h->keys[i]);
            g.used[s] = 1;
            g.keys[s] = h->keys[i];
            g.vals[s] = h->vals[i];
            g.len++;
        }
    hm_free(h);
    *h = g;
}
/* Returns pointer to the value slot; *inserted set when the key was new. */
static uint32_t *hm_entry(hmap_t *h, uint64_t k, bool *inserted) {
    if ((h->len + 1) * 2 > h->cap) hm_grow(h);
    size_t s = hm_slot(h, k);
    *inserted = !h->used[s];
    if (!h->used[s]) {
        h->used[s] = 1;
        h->keys[s] = k;
        h->vals[s] = 0;
        h->len++;
    }
    return &h->vals[s];
}
static bool hm_get(const hmap_t *h, uint64_t k, uint32_t *v) {
    size_t s = hm_slot(h, k);
    if (!h->used[s]) return false;
    *v = h->vals[s];
    return true;
}

/* Top-8 keys by (count desc, key asc) — alp_rd.rs:58-68. */
static size_t top8(const hmap_t *h, uint64_t *dict, uint64_t *covered) {
    uint64_t tk[8];
    uint32_t tc[8];
    size_t nt = 0;
    for (size_t i = 0; i < h->cap; i++) {
        if (!h->used[i]) continue;
        uint64_t k = h->keys[i];
        uint32_t c = h->vals[i];
        /* insertion into sorted top list */
        size_t pos = nt;
        while (pos > 0 && (c > tc[pos - 1] || (c == tc[pos - 1] && k < tk[pos - 1]))) pos--;
        if (pos >= 8) continue;
        size_t end = nt < 8 ? nt : 7;
        for (size_t j = end; j > pos; j--) {
            tk[j] = tk[j - 1];
            tc[j] = tc[j - 1];
        }
        tk[pos] = k;
        tc[pos] = c;
        if (nt < 8) nt++;
    }
    uint64_t cov = 0;
    for (size_t j = 0; j < nt; j++) {
        dict[j] = tk[j];
        cov += tc[j];
    }
    *covered = cov;
    return nt;
}

/* ------------------------------------------------------------------------ */
/* rANS — src/entropy/rans.rs:25-175                                         */
/* ------------------------------------------------------------------------ */

#define RANS_SCALE_BITS 12
#define RANS_M (1u << RANS_SCALE_BITS)
#define RANS_L (1u << 23)

/* rans.rs:25-48 (ties: Iterator::max_by_key returns the LAST maximum) */
static void rans_normalize(const uint32_t *counts, uint64_t total, uint32_t *freq) {
    uint32_t sum = 0;
    for (int s = 0; s < 256; s++) {
        freq[s] = 0;
        if (counts[s] > 0) {
            uint32_t f = (uint32_t)(((uint64_t)counts[s] * RANS_M) / total);
            freq[s] = f ? f : 1;
            sum += freq[s];
        }
    }
    while (sum > RANS_M) {
        int best = -1;
        for (int s = 0; s < 256; s++)
            if (freq[s] > 1 && (best < 0 || freq[s] >= freq[best])) best = s;
        freq[best]--;
        sum--;
    }
    if (sum < RANS_M) {
        int best = 0;
        for (int s = 0; s < 256; s++)
            if (freq[s] >= freq[best]) best = s;
        freq[best] += RANS_M - sum;
    }
}
/* rans.rs:52-108 */
static bool rans_compress(const uint8_t *data, size_t n, buf_t *out) {
    if (n == 0) return false;
    uint32_t counts[256] = {0}, freq[256], cum[257];
    for (size_t i = 0; i < n; i++) counts[data[i]]++;
    rans_normalize(counts, n, freq);
    cum[0] = 0;
    for (int s = 0; s < 256; s++) cum[s + 1] = cum[s] + freq[s];
    size_t blen = 2 * n + 16 + 64;
    uint8_t *buf = (uint8_t *)malloc(blen);
    size_t p = blen;
    uint32_t x[4] = {RANS_L, RANS_L, RANS_L, RANS_L};
    for (size_t i = n; i > 0;) {
        i--;
        uint32_t s = data[i], f = freq[s], c = cum[s];
        size_t idx = i & 3;
        uint32_t xi = x[idx];
        uint32_t x_max = ((RANS_L >> RANS_SCALE_BITS) << 8) * f;
        while (xi >= x_max) {
            buf[--p] = (uint8_t)xi;
            xi >>= 8;
        }
        x[idx] = ((xi / f) << RANS_SCALE_BITS) + (xi % f) + c;
    }
    for (int idx = 3; idx >= 0; idx--) {
        p -= 4;
        for (int k = 0; k < 4; k++) buf[p + k] = (uint8_t)(x[idx] >> (8 * k));
    }
    b_varint(out, n);
    size_t present = 0;
    for (int s = 0; s < 256; s++) present += freq[s] > 0;
    b_varint(out, present);
    for (int s = 0; s < 256; s++)
        if (freq[s] > 0) {
            b_push(out, (uint8_t)s);
            b_varint(out, freq[s]);
        }
    b_write(out, buf + p, blen - p);
    free(buf);
    return true;
}
/* rans.rs:110-175 */
static int rans_decompress(const uint8_t *p, size_t plen, size_t max_len, buf_t *out) {
    size_t pos = 0;
    uint64_t n64, ns64;
    int rc = varint_read(p, plen, &pos, &n64);
    if (rc) return rc;
    if (n64 > (uint64_t)max_len) return OQ_CORRUPT;
    rc = varint_read(p, plen, &pos, &ns64);
    if (rc) return rc;
    if (ns64 == 0 || ns64 > 256) return OQ_CORRUPT;
    uint32_t freq[256] = {0}, cum[257], sum = 0;
    for (uint64_t k = 0; k < ns64; k++) {
        if (pos >= plen) return OQ_TRUNCATED;
        uint8_t s = p[pos++];
        uint64_t f64v;
        rc = varint_read(p, plen, &pos, &f64v);
        if (rc) return rc;
        uint32_t f = (uint32_t)f64v;
        if (f == 0 || f > RANS_M) return OQ_CORRUPT;
        freq[s] = f;
        sum += f;
    }
    if (sum != RANS_M) return OQ_CORRUPT;
    cum[0] = 0;
    for (int s = 0; s < 256; s++) cum[s + 1] = cum[s] + freq[s];
    uint8_t slot_to_sym[RANS_M];
    memset(slot_to_sym, 0, sizeof slot_to_sym);
    for (int s = 0; s < 256; s++)
        for (uint32_t slot = cum[s]; slot < cum[s + 1] && slot < RANS_M; slot++) slot_to_sym[slot] = (uint8_t)s;
    uint32_t x[4];
    for (int k = 0; k < 4; k++) {
        if (plen < pos + 4) return OQ_TRUNCATED;
        x[k] = rd_u32(p + pos);
        pos += 4;
    }
    size_t n = (size_t)n64;
    b_reserve(out, n);
    for (size_t i = 0; i < n; i++) {
        size_t idx = i & 3;
        uint32_t xi = x[idx], slot = xi & (RANS_M - 1);
        uint8_t s = slot_to_sym[slot];
        out->p[out->len++] = s;
        uint32_t xn = freq[s] * (xi >> RANS_SCALE_BITS) + slot - cum[s];
        while (xn < RANS_L) {
            if (pos >= plen) return OQ_TRUNCATED;
            xn = (xn << 8) | p[pos++];
        }
        x[idx] = xn;
    }
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* Entropy stage (rANS branch) — src/entropy/mod.rs:49-75,127-178            */
/* ------------------------------------------------------------------------ */

#define TAG_RC 0
#define TAG_TANS 1
#define TAG_RANS 2
#define TAG_LZ 3

/* entropy/mod.rs:49-60 + 127-150 for lambda >= 2 and no LZ cascade: rANS
 * always compresses non-empty input, and every in-path caller passes a
 * non-empty stream. */
static void code_residuals(const uint8_t *res, size_t n, buf_t *out) {
    b_push(out, TAG_RANS);
    rans_compress(res, n, out);
}
/* ------------------------------------------------------------------------ */
/* Range coder — src/entropy/rc.rs: a binary LZMA-style coder (11-bit         */
/* probabilities adapted by shift 5, a 32-bit range renormalised a byte at a  */
/* time, carries through a cached byte) under an order-1 byte model: 256      */
/* contexts (the previous byte) x a 256-node bit tree, MSB first.             */
/* ------------------------------------------------------------------------ */
#define RC_PROB_BITS 11
#define RC_PROB_INIT 1024
#define RC_MOVE_BITS 5
#define RC_TOP (1u << 24)

typedef struct {
    uint64_t low;
    uint32_t range;
    uint8_t cache;
    uint64_t cache_size;
    buf_t *out;
} rc_enc_t;

/* rc.rs:40-57 */
static void rc_shift_low(rc_enc_t *e) {
    if ((e->low >> 32) != 0 || e->low < 0xFF000000ull) {
        uint8_t carry = (uint8_t)(e->low >> 32);
        uint8_t temp = e->cache;
        do {
            b_push(e->out, (uint8_t)(temp + carry));
            temp = 0xFF;
        } while (--e->cache_size != 0);
        e->cache = (uint8_t)((e->low >> 24) & 0xFF);
    }
    e->cache_size++;
    e->low = (e->low & 0x00FFFFFFull) << 8;
}

/* rc.rs:59-79 (the branchless form selects exactly these updates) */
static void rc_encode_bit(rc_enc_t *e, uint16_t *prob, uint32_t bit) {
    uint32_t bound = (e->range >> RC_PROB_BITS) * (uint32_t)*prob;
    uint32_t p = *prob;
    if (bit) {
        e->low += bound;
        e->range -= bound;
        *prob = (uint16_t)(p - (p >> RC_MOVE_BITS));
    } else {
        e->range = bound;
        *prob = (uint16_t)(p + (((1u << RC_PROB_BITS) - p) >> RC_MOVE_BITS));
    }
    while (e->range < RC_TOP) {
        e->range <<= 8;
        rc_shift_low(e);
    }
}

typedef struct {
    uint32_t code, range;
    const uint8_t *in;
    size_t len, pos;
} rc_dec_t;

/* rc.rs:113-120: reads past the end give 0 */
static uint32_t rc_next(rc_dec_t *d) {
    uint32_t b = d->pos < d->len ? d->in[d->pos] : 0;
    d->pos++;
    return b;
}

/* rc.rs:122-142 */
static uint32_t rc_decode_bit(rc_dec_t *d, uint16_t *prob) {
    uint32_t bound = (d->range >> RC_PROB_BITS) * (uint32_t)*prob;
    uint32_t p = *prob;
    uint32_t bit = d->code >= bound;
    if (bit) {
        d->code -= bound;
        d->range -= bound;
        *prob = (uint16_t)(p - (p >> RC_MOVE_BITS));
    } else {
        d->range = bound;
        *prob = (uint16_t)(p + (((1u << RC_PROB_BITS) - p) >> RC_MOVE_BITS));
    }
    while (d->range < RC_TOP) {
        d->range <<= 8;
        d->code = (d->code << 8) | rc_next(d);
    }
    return bit;
}

/* rc.rs:193-206: varint(len) ++ coded bytes */
static void rc_compress(const uint8_t *src, size_t n, buf_t *out) {
    b_varint(out, n);
    rc_enc_t e = {0, 0xFFFFFFFFu, 0, 1, out};
    uint16_t *probs = (uint16_t *)malloc(65536 * sizeof(uint16_t));
    for (size_t i = 0; i < 65536; i++) probs[i] = RC_PROB_INIT;
    size_t ctx = 0;
    for (size_t i = 0; i < n; i++) {
        uint32_t node = 1;
        for (int k = 7; k >= 0; k--) {
            uint32_t bit = (src[i] >> k) & 1u;
            rc_encode_bit(&e, &probs[ctx * 256 + node], bit);
            node = (node << 1) | bit;
        }
        ctx = src[i];
    }
    for (int k = 0; k < 5; k++) rc_shift_low(&e);
    free(probs);
}

/* rc.rs:208-225 */
static int rc_decompress(const uint8_t *p, size_t plen, size_t max_len, buf_t *out) {
    size_t pos = 0;
    uint64_t len = 0;
    int rc = varint_read(p, plen, &pos, &len);
    if (rc) return rc;
    if (len > max_len) return OQ_CORRUPT;
    rc_dec_t d = {0, 0xFFFFFFFFu, p + pos, plen - pos, 0};
    rc_next(&d);  /* the encoder's leading cache byte */
    for (int k = 0; k < 4; k++) d.code = (d.code << 8) | rc_next(&d);
    uint16_t *probs = (uint16_t *)malloc(65536 * sizeof(uint16_t));
    for (size_t i = 0; i < 65536; i++) probs[i] = RC_PROB_INIT;
    b_reserve(out, (size_t)len);
    size_t ctx = 0;
    for (uint64_t i = 0; i < len; i++) {
        uint32_t node = 1;
        for (int k = 0; k < 8; k++) node = (node << 1) | rc_decode_bit(&d, &probs[ctx * 256 + node]);
        uint8_t b = (uint8_t)(node & 0xFF);
        b_push(out, b);
        ctx = b;
    }
    free(probs);
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* LZ — src/codecs/lz.rs: byte LZ77 with LZSS framing (a control byte of 8    */
/* flags, MSB first; 1 = match (varint offset, varint length - 4), 0 = a     */
/* literal byte) after varint(original length).  Mode LZ (4) codes a block's  */
/* little-endian bytes; the Max cascade (entropy tag 3) codes residual bytes. */
/* ------------------------------------------------------------------------ */
#define LZ_MIN_MATCH 4
#define LZ_HASH_BITS 17
#define LZ_MAX_CHAIN 64

/* lz.rs:19-23 */
static size_t lz_hash4(const uint8_t *w) {
    uint32_t v = (uint32_t)w[0] | ((uint32_t)w[1] << 8) | ((uint32_t)w[2] << 16) | ((uint32_t)w[3] << 24);
    return (size_t)((uint32_t)(v * 2654435761u) >> (32 - LZ_HASH_BITS));
}

/* lz.rs:30-117: greedy matching over hash chains of at most 64 candidates */
static void lz_compress(const uint8_t *in, size_t n, buf_t *out) {
    int64_t *head = (int64_t *)malloc(((size_t)1 << LZ_HASH_BITS) * sizeof(int64_t));
    int64_t *prev = (int64_t *)malloc((n ? n : 1) * sizeof(int64_t));
    for (size_t i = 0; i < ((size_t)1 << LZ_HASH_BITS); i++) head[i] = -1;
    for (size_t i = 0; i < n; i++) prev[i] = -1;
    /* tokens: off = 0 marks a literal (matches always have off >= 1) */
    uint32_t *toff = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    uint32_t *tval = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    size_t nt = 0, i = 0;
    while (i < n) {
        size_t best_len = 0, best_off = 0;
        if (i + LZ_MIN_MATCH <= n) {
            size_t h = lz_hash4(in + i), max_len = n - i;
            int64_t cand = head[h];
            int chain = LZ_MAX_CHAIN;
            while (cand >= 0 && chain > 0) {
                size_t c = (size_t)cand;
                if (best_len == 0 || (c + best_len < n && in[c + best_len] == in[i + best_len])) {
                    size_t l = 0;
                    while (l < max_len && in[c + l] == in[i + l]) l++;
                    if (l > best_len) {
                        best_len = l;
                        best_off = i - c;
                        if (l == max_len) break;
                    }
                }
                cand = prev[c];
                chain--;
            }
        }
        if (best_len >= LZ_MIN_MATCH) {
            toff[nt] = (uint32_t)best_off;
            tval[nt++] = (uint32_t)best_len;
            size_t end = i + best_len;
            for (; i < end; i++)
                if (i + LZ_MIN_MATCH <= n) {
                    size_t h = lz_hash4(in + i);
                    prev[i] = head[h];
                    head[h] = (int64_t)i;
                }
        } else {
            toff[nt] = 0;
            tval[nt++] = in[i];
            if (i + LZ_MIN_MATCH <= n) {
                size_t h = lz_hash4(in + i);
                prev[i] = head[h];
                head[h] = (int64_t)i;
            }
            i++;
        }
    }
    b_varint(out, n);
    for (size_t g = 0; g < nt; g += 8) {
        uint8_t ctrl = 0;
        size_t ge = g + 8 < nt ? g + 8 : nt;
        for (size_t k = g; k < ge; k++)
            if (toff[k]) ctrl |= (uint8_t)(1u << (7 - (k - g)));
        b_push(out, ctrl);
        for (size_t k = g; k < ge; k++) {
            if (toff[k]) {
                b_varint(out, toff[k]);
                b_varint(out, tval[k] - LZ_MIN_MATCH);
            } else {
                b_push(out, (uint8_t)tval[k]);
            }
        }
    }
    free(head);
    free(prev);
    free(toff);
    free(tval);
}

/* lz.rs:119-155 */
static int lz_decompress(const uint8_t *p, size_t len, size_t expected, buf_t *out) {
    size_t pos = 0;
    uint64_t n;
    int rc = varint_read(p, len, &pos, &n);
    if (rc) return rc;
    if (n != expected) return OQ_CORRUPT;
    b_reserve(out, (size_t)n);
    while (out->len < n) {
        if (pos >= len) return OQ_TRUNCATED;
        uint8_t ctrl = p[pos++];
        for (int k = 0; k < 8 && out->len < n; k++) {
            if ((ctrl >> (7 - k)) & 1) {
                uint64_t off, ml;
                if ((rc = varint_read(p, len, &pos, &off))) return rc;
                if ((rc = varint_read(p, len, &pos, &ml))) return rc;
                ml += LZ_MIN_MATCH;
                if (off == 0 || off > out->len) return OQ_CORRUPT;
                if (ml > n - out->len) return OQ_CORRUPT; /* out.len() + len > n, without wrapping */
                size_t start = out->len - (size_t)off;
                for (uint64_t j = 0; j < ml; j++) b_push(out, out->p[start + j]);
            } else {
                if (pos >= len) return OQ_TRUNCATED;
                b_push(out, p[pos++]);
            }
        }
    }
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* tANS — src/entropy/tans.rs, src/bitio.rs (entropy tag 1: the reference    */
/* still decodes it and no longer produces it; the encoder here only makes   */
/* test streams)                                                             */
/* ------------------------------------------------------------------------ */
/* A 1,024-entry state table (states 1024..2047).  Wire: varint(len) ++
 * u8(distinct - 1) ++ the distinct symbols ++ their u16 LE weights (sum 1024)
 * ++ u32 LE final encoder state ++ the renormalisation bits, MSB first. */
#define TANS_SIZE 1024u
#define TANS_LOG 10u

/* tans.rs:85-99: weight w of symbol s fills w table slots, visited with the
 * odd stride 615 (3 * 1024 / 5 made odd), so every slot is written once. */
static void tans_spread(const uint16_t *w, const uint8_t *syms, int num, uint8_t *table) {
    uint32_t stride = (3u * TANS_SIZE) / 5u;
    if (!(stride & 1u)) stride++;
    uint32_t step = 0;
    for (int s = 0; s < num; s++)
        for (uint32_t k = 0; k < w[s]; k++, step++) table[(stride * step) & (TANS_SIZE - 1u)] = syms[s];
}

/* tans.rs:28-78: f32 weights, one extra table slot per symbol kept back and
 * the rest shared by (count * 1024 / total - 1); then +-1 round-robin nudges
 * (at most 8 * num + 16 each way) to a sum of exactly 1024, else no coder. */
static int tans_quantize(const uint32_t *counts, const uint8_t *syms, int num, uint64_t total, uint16_t *w) {
    if (num <= 0 || num > 256) return 0;
    float mult = total ? (float)TANS_SIZE / (float)total : 0.0f;
    float want[256], want_sum = 0.0f;
    for (int i = 0; i < num; i++) {
        float x = (float)counts[syms[i]] * mult - 1.0f;
        if (x < 0.0f) x = 0.0f;
        want[i] = x;
        want_sum += x;
    }
    float share = want_sum > 0.0f ? ((float)TANS_SIZE - (float)num) / want_sum : 0.0f;
    int64_t sum = 0;
    for (int i = 0; i < num; i++) {
        float x = 1.0f + want[i] * share + 0.5f;
        uint16_t q = x >= 65535.0f ? 65535 : (uint16_t)x;
        w[i] = q ? q : 1;
        sum += w[i];
    }
    int guard = num * 8 + 16, i = 0;
    for (; sum > (int64_t)TANS_SIZE && guard > 0; guard--, i = (i + 1) % num)
        if (w[i] > 1) {
            w[i]--;
            sum--;
        }
    guard = num * 8 + 16;
    i = 0;
    for (; sum < (int64_t)TANS_SIZE && guard > 0; guard--, i = (i + 1) % num) {
        w[i]++;
        sum++;
    }
    return sum == (int64_t)TANS_SIZE;
}

/* tans.rs:108-191.  Returns 0 (no stream) for empty input or when the weights
 * cannot be made to sum to 1024. */
static int tans_compress(const uint8_t *src, size_t n, buf_t *out) {
    if (n == 0) return 0;
    uint32_t counts[256] = {0};
    for (size_t i = 0; i < n; i++) counts[src[i]]++;
    uint8_t syms[256];
    int num = 0, slot[256];
    for (int b = 0; b < 256; b++)
        if (counts[b]) {
            slot[b] = num;
            syms[num++] = (uint8_t)b;
        }
    uint16_t w[256];
    if (!tans_quantize(counts, syms, num, n, w)) return 0;
    uint8_t table[TANS_SIZE];
    tans_spread(w, syms, num, table);
    /* per symbol: the renormalisation bit count (min_bits, +1 at or above
     * cutoff) and the first of its next-state entries (start) */
    uint32_t cutoff[256] = {0}, start[256] = {0}, fill[256];
    uint8_t min_bits[256] = {0};
    uint32_t cum = 0;
    for (int s = 0; s < num; s++) {
        uint32_t top = 2u * w[s] - 1u, lg = 0;
        while ((top >> lg) > 1u) lg++;
        min_bits[syms[s]] = (uint8_t)(TANS_LOG - lg);
        cutoff[syms[s]] = (2u * w[s]) << (TANS_LOG - lg);
        start[syms[s]] = cum;
        fill[s] = cum;
        cum += w[s];
    }
    uint32_t next[TANS_SIZE];
    for (uint32_t i = 0; i < TANS_SIZE; i++) next[fill[slot[table[i]]]++] = TANS_SIZE + i;
    /* encode last symbol first; the bits of symbol k go out in symbol order */
    uint16_t *low = (uint16_t *)malloc(n * sizeof(uint16_t));
    uint8_t *nb = (uint8_t *)malloc(n);
    uint32_t state = TANS_SIZE;
    for (size_t k = n; k-- > 0;) {
        uint8_t c = src[k];
        uint32_t bits = min_bits[c] + (state >= cutoff[c] ? 1u : 0u);
        low[k] = (uint16_t)(bits ? (state & ((1u << bits) - 1u)) : 0u);
        nb[k] = (uint8_t)bits;
        state = next[start[c] + (state >> bits) - w[slot[c]]];
    }
    b_varint(out, n);
    b_push(out, (uint8_t)(num - 1));
    b_write(out, syms, (size_t)num);
    for (int s = 0; s < num; s++) b_u16(out, w[s]);
    b_u32(out, state);
    uint64_t acc = 0;
    unsigned have = 0;
    for (size_t k = 0; k < n; k++) {
        if (!nb[k]) continue;
        acc = (acc << nb[k]) | low[k];
        have += nb[k];
        while (have >= 8) {
            have -= 8;
            b_push(out, (uint8_t)(acc >> have));
        }
        acc &= (1ull << have) - 1ull;
    }
    if (have) b_push(out, (uint8_t)(acc << (8 - have)));
    free(low);
    free(nb);
    return 1;
}

/* tans.rs:193-283: header checks in the reference's order, then one table
 * lookup and one MSB-first bit read per byte; reads past the end give 0. */
static int tans_decompress(const uint8_t *p, size_t plen, size_t max_len, buf_t *out) {
    size_t pos = 0;
    uint64_t len;
    int rc = varint_read(p, plen, &pos, &len);
    if (rc) return rc;
    if (len > max_len) return OQ_CORRUPT;
    if (pos >= plen) return OQ_TRUNCATED;
    int num = p[pos++] + 1;
    if (plen - pos < (size_t)num) return OQ_TRUNCATED;
    const uint8_t *syms = p + pos;
    pos += (size_t)num;
    uint16_t w[256];
    for (int s = 0; s < num; s++) {
        if (plen - pos < 2) return OQ_TRUNCATED;
        w[s] = (uint16_t)(p[pos] | (p[pos + 1] << 8));
        pos += 2;
    }
    if (plen - pos < 4) return OQ_TRUNCATED;
    uint32_t state = (uint32_t)p[pos] | ((uint32_t)p[pos + 1] << 8) | ((uint32_t)p[pos + 2] << 16) |
                     ((uint32_t)p[pos + 3] << 24);
    pos += 4;
    if (state < TANS_SIZE || state >= 2u * TANS_SIZE) return OQ_CORRUPT;
    uint8_t seen[256] = {0};
    uint32_t wsum = 0;
    for (int s = 0; s < num; s++) {
        if (!w[s] || seen[syms[s]]) return OQ_CORRUPT;
        seen[syms[s]] = 1;
        wsum += w[s];
    }
    if (wsum != TANS_SIZE) return OQ_CORRUPT;
    uint8_t table[TANS_SIZE], bits_of[TANS_SIZE];
    uint16_t base_of[TANS_SIZE];
    tans_spread(w, syms, num, table);
    /* the k-th slot of a symbol of weight w continues from x = w + k: it
     * reads enough bits to bring x << bits into [1024, 2048) */
    uint32_t x[256] = {0};
    for (int s = 0; s < num; s++) x[syms[s]] = w[s];
    for (uint32_t i = 0; i < TANS_SIZE; i++) {
        uint32_t b = x[table[i]]++;
        if (!b) return OQ_CORRUPT;
        uint32_t bits = (uint32_t)(__builtin_clz(b) - __builtin_clz(TANS_SIZE));
        base_of[i] = (uint16_t)((b << bits) - TANS_SIZE);
        bits_of[i] = (uint8_t)bits;
    }
    const uint8_t *in = p + pos;
    size_t inlen = plen - pos, ip = 0;
    uint64_t acc = 0;
    unsigned have = 0;
    b_reserve(out, (size_t)len);
    for (uint64_t k = 0; k < len; k++) {
        uint32_t idx = state - TANS_SIZE;
        if (idx >= TANS_SIZE) return OQ_CORRUPT;
        uint32_t bits = bits_of[idx], extra = 0;
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
        out->p[out->len++] = table[idx];
        state = TANS_SIZE + base_of[idx] + extra;
    }
    return OQ_OK;
}

/* entropy/mod.rs:152-163: tag 2 rANS, tag 0 the range coder, tag 1 tANS. */
static int decode_entropy_only(const uint8_t *p, size_t plen, size_t max_len, buf_t *out) {
    if (plen == 0) return OQ_TRUNCATED;
    switch (p[0]) {
        case TAG_RANS: return rans_decompress(p + 1, plen - 1, max_len, out);
        case TAG_RC: return rc_decompress(p + 1, plen - 1, max_len, out);
        case TAG_TANS: return tans_decompress(p + 1, plen - 1, max_len, out);
        default: return OQ_CORRUPT;
    }
}
/* entropy/mod.rs:165-178: tag 3 is the LZ cascade (Max): varint(residual
 * length) ++ an entropy-coded LZ stream of at most 2 * length + 64 bytes. */
static int decode_residuals(const uint8_t *p, size_t plen, size_t max_len, buf_t *out) {
    if (plen && p[0] == TAG_LZ) {
        size_t pos = 0;
        uint64_t orig;
        int rc = varint_read(p + 1, plen - 1, &pos, &orig);
        if (rc) return rc;
        if (orig > max_len) return OQ_CORRUPT;
        buf_t lzs = {0};
        rc = decode_entropy_only(p + 1 + pos, plen - 1 - pos, (size_t)orig * 2 + 64, &lzs);
        if (!rc) rc = lz_decompress(lzs.p, lzs.len, (size_t)orig, out);
        b_free(&lzs);
        return rc;
    }
    return decode_entropy_only(p, plen, max_len, out);
}

/* ------------------------------------------------------------------------ */
/* BYTE_TRANSPOSE — src/codecs/transpose.rs:10-32, src/transform.rs:24-47    */
/* ------------------------------------------------------------------------ */

static uint8_t *transpose_encode(const uint64_t *v, size_t n) {
    uint8_t *soa = (uint8_t *)malloc(n * 8 + 1);
    for (int plane = 0; plane < 8; plane++)
        for (size_t i = 0; i < n; i++) soa[plane * n + i] = (uint8_t)(v[i] >> (8 * plane));
    return soa;
}
static int transpose_decode(const uint8_t *soa, size_t len, size_t n, uint64_t *out) {
    if (len != n * 8) return OQ_CORRUPT;
    for (size_t i = 0; i < n; i++) {
        uint64_t w = 0;
        for (int plane = 0; plane < 8; plane++) w |= (uint64_t)soa[plane * n + i] << (8 * plane);
        out[i] = w;
    }
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* ALP-RD — src/codecs/alp_rd.rs:80-285                                      */
/* ------------------------------------------------------------------------ */

static uint32_t rd_code_bits(size_t dict_len) { /* alp_rd.rs:70-76 */
    if (dict_len <= 1) return 1;
    uint32_t b = bit_width((uint64_t)(dict_len - 1));
    return b ? b : 1;
}
/* alp_rd.rs:80-107 */
static bool rd_choose_cut(const uint64_t *v, size_t n, uint32_t *cut) {
    size_t step = n / 2048 ? n / 2048 : 1;
    size_t sn = (n + step - 1) / step;
    uint32_t best_cut = 0;
    double best_bits = INFINITY;
    hmap_t h;
    for (uint32_t lbw = 1; lbw <= 24; lbw++) {
        uint32_t rbw = 64 - lbw;
        hm_init(&h, 64);
        for (size_t i = 0; i < n; i += step) {
            bool ins;
            (*hm_entry(&h, v[i] >> rbw, &ins))++;
        }
        uint64_t dict[8], covered;
        size_t dl = top8(&h, dict, &covered);
        hm_free(&h);
        uint64_t exc = (uint64_t)sn - covered;
        double per_value = (double)((uint64_t)sn * (uint64_t)(rbw + rd_code_bits(dl)) + exc * 96) / (double)sn;
        if (per_value < best_bits) {
            best_bits = per_value;
            best_cut = lbw;
        }
    }
    if (best_cut == 0 || best_bits >= 63.0) return false;
    *cut = best_cut;
    return true;
}
/* alp_rd.rs:132-206 */
static bool alprd_encode(const uint64_t *v, size_t n, bool entropy, buf_t *out) {
    if (n == 0) return false;
    uint32_t lbw;
    if (!rd_choose_cut(v, n, &lbw)) return false;
    uint32_t rbw = 64 - lbw;
    uint64_t rmask = mask64(rbw);
    hmap_t h;
    hm_init(&h, 64);
    for (size_t i = 0; i < n; i++) {
        bool ins;
        (*hm_entry(&h, v[i] >> rbw, &ins))++;
    }
    uint64_t dict[8], cov;
    size_t dl = top8(&h, dict, &cov);
    hm_free(&h);
    uint64_t *codes = (uint64_t *)malloc(n * 8), *rights = (uint64_t *)malloc(n * 8);
    size_t *exc_pos = (size_t *)malloc(n * sizeof(size_t));
    uint64_t *exc_left = (uint64_t *)malloc(n * 8);
    size_t nexc = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t left = v[i] >> rbw;
        rights[i] = v[i] & rmask;
        size_t c = 0;
        bool found = false;
        for (size_t j = 0; j < dl; j++)
            if (dict[j] == left) {
                c = j;
                found = true;
                break;
            }
        if (found) {
            codes[i] = c;
        } else {
            codes[i] = 0;
            exc_pos[nexc] = i;
            exc_left[nexc] = left;
            nexc++;
        }
    }
    bool ok = nexc * 4 <= n;
    if (ok) {
        b_push(out, (uint8_t)lbw);
        b_push(out, (uint8_t)dl);
        for (size_t j = 0; j < dl; j++) b_u64(out, dict[j]);
        b_varint(out, nexc);
        for (size_t x = 0; x < nexc; x++) {
            b_varint(out, exc_pos[x]);
            b_u64(out, exc_left[x]);
        }
        buf_t cbp = {0}, rbp = {0};
        for_encode(codes, n, false, &cbp);
        uint8_t ctag = 0;
        buf_t *cblob = &cbp;
        buf_t cent = {0}, rent = {0};
        if (entropy) {
            uint8_t *cb = (uint8_t *)malloc(n);
            for (size_t i = 0; i < n; i++) cb[i] = (uint8_t)codes[i];
            code_residuals(cb, n, &cent);
            free(cb);
            if (cent.len < cbp.len) {
                ctag = 1;
                cblob = &cent;
            }
        }
        for_encode(rights, n, false, &rbp);
        uint8_t rtag = 0;
        buf_t *rblob = &rbp;
        if (entropy) {
            code_residuals(rbp.p, rbp.len, &rent);
            if (rent.len < rbp.len) {
                rtag = 1;
                rblob = &rent;
            }
        }
        b_push(out, ctag);
        b_varint(out, cblob->len);
        b_write(out, cblob->p, cblob->len);
        b_push(out, rtag);
        b_write(out, rblob->p, rblob->len);
        b_free(&cbp);
        b_free(&rbp);
        b_free(&cent);
        b_free(&rent);
    }
    free(codes);
    free(rights);
    free(exc_pos);
    free(exc_left);
    return ok;
}
/* alp_rd.rs:208-285 */
static int alprd_decode(const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    size_t pos = 0;
    if (pos >= plen) return OQ_TRUNCATED;
    uint32_t lbw = p[pos++];
    if (lbw < 1 || lbw > 63) return OQ_CORRUPT;
    uint32_t rbw = 64 - lbw;
    if (pos >= plen) return OQ_TRUNCATED;
    size_t dsz = p[pos++];
    if (dsz > 8) return OQ_CORRUPT;
    uint64_t dict[8];
    for (size_t j = 0; j < dsz; j++) {
        if (plen < pos + 8) return OQ_TRUNCATED;
        dict[j] = rd_u64(p + pos);
        pos += 8;
    }
    uint64_t nexc64;
    int rc = varint_read(p, plen, &pos, &nexc64);
    if (rc) return rc;
    if (nexc64 > (uint64_t)n) return OQ_CORRUPT;
    size_t nexc = (size_t)nexc64;
    size_t *ep = (size_t *)malloc((nexc ? nexc : 1) * sizeof(size_t));
    uint64_t *el = (uint64_t *)malloc((nexc ? nexc : 1) * 8);
    uint64_t *codes = NULL, *rights = NULL;
    buf_t tmp = {0};
    for (size_t x = 0; x < nexc; x++) {
        uint64_t pp;
        rc = varint_read(p, plen, &pos, &pp);
        if (rc) goto done;
        if (plen < pos + 8) {
            rc = OQ_TRUNCATED;
            goto done;
        }
        uint64_t l = rd_u64(p + pos);
        pos += 8;
        if (pp >= (uint64_t)n) {
            rc = OQ_CORRUPT;
            goto done;
        }
        ep[x] = (size_t)pp;
        el[x] = l;
    }
    if (pos >= plen) {
        rc = OQ_TRUNCATED;
        goto done;
    }
    uint8_t ctag = p[pos++];
    uint64_t clen64;
    rc = varint_read(p, plen, &pos, &clen64);
    if (rc) goto done;
    if (clen64 > (uint64_t)(plen - pos)) {
        rc = OQ_TRUNCATED;
        goto done;
    }
    const uint8_t *cblob = p + pos;
    size_t clen = (size_t)clen64;
    pos += clen;
    if (pos >= plen) {
        rc = OQ_TRUNCATED;
        goto done;
    }
    uint8_t rtag = p[pos++];
    const uint8_t *rblob = p + pos;
    size_t rlen = plen - pos;
    codes = (uint64_t *)malloc((n ? n : 1) * 8);
    rights = (uint64_t *)malloc((n ? n : 1) * 8);
    if (ctag == 0) {
        rc = for_decode(cblob, clen, n, false, codes);
        if (rc) goto done;
    } else if (ctag == 1) {
        rc = decode_residuals(cblob, clen, n, &tmp);
        if (rc) goto done;
        if (tmp.len != n) {
            rc = OQ_CORRUPT;
            goto done;
        }
        for (size_t i = 0; i < n; i++) codes[i] = tmp.p[i];
        tmp.len = 0;
    } else {
        rc = OQ_CORRUPT;
        goto done;
    }
    if (rtag == 0) {
        rc = for_decode(rblob, rlen, n, false, rights);
        if (rc) goto done;
    } else if (rtag == 1) {
        rc = decode_residuals(rblob, rlen, n * 8 + 64, &tmp);
        if (rc) goto done;
        rc = for_decode(tmp.p, tmp.len, n, false, rights);
        if (rc) goto done;
    } else {
        rc = OQ_CORRUPT;
        goto done;
    }
    for (size_t i = 0; i < n; i++) {
        if (codes[i] >= dsz) {
            rc = OQ_CORRUPT;
            goto done;
        }
        out[i] = (dict[codes[i]] << rbw) | rights[i];
    }
    for (size_t x = 0; x < nexc; x++) out[ep[x]] = (el[x] << rbw) | rights[ep[x]];
    rc = OQ_OK;
done:
    free(ep);
    free(el);
    free(codes);
    free(rights);
    b_free(&tmp);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* FLOAT_MULT — src/codecs/float_mult.rs:45-133                              */
/* ------------------------------------------------------------------------ */

static const double FM_SCALES[7] = {10.0, 100.0, 1000.0, 10000.0, 100000.0, 1000000.0, 10000000.0};

/* float_mult.rs:45-64 */
static bool fm_find_scale(const uint64_t *v, size_t n, int *idx_out, int64_t *ks) {
    for (int idx = 0; idx < 7; idx++) {
        double scale = FM_SCALES[idx];
        bool ok = true;
        for (size_t i = 0; i < n; i++) {
            double x = as_f64(v[i]);
            double k = round(x * scale);
            if (!isfinite(k) || fabs(k) >= 9.0e18) {
                ok = false;
                break;
            }
            int64_t ki = (int64_t)k;
            if (f64_bits((double)ki / scale) != v[i]) {
                ok = false;
                break;
            }
            ks[i] = ki;
        }
        if (ok) {
            *idx_out = idx;
            return true;
        }
    }
    return false;
}
/* float_mult.rs:66-98 */
static bool fm_encode(const uint64_t *v, size_t n, bool entropy, buf_t *out) {
    if (n == 0) return false;
    int64_t *ks = (int64_t *)malloc(n * 8);
    int idx;
    if (!fm_find_scale(v, n, &idx, ks)) {
        free(ks);
        return false;
    }
    buf_t bp = {0};
    for_encode((const uint64_t *)ks, n, true, &bp);
    uint8_t tag = 0;
    buf_t *blob = &bp;
    buf_t coded = {0};
    if (entropy) {
        buf_t delta = {0};
        int64_t prev = 0;
        for (size_t i = 0; i < n; i++) {
            b_varint(&delta, zigzag64((uint64_t)ks[i] - (uint64_t)prev));
            prev = ks[i];
        }
        code_residuals(delta.p, delta.len, &coded);
        b_free(&delta);
        if (coded.len < bp.len) {
            tag = 1;
            blob = &coded;
        }
    }
    b_push(out, tag);
    b_push(out, (uint8_t)idx);
    b_write(out, blob->p, blob->len);
    b_free(&bp);
    b_free(&coded);
    free(ks);
    return true;
}
/* float_mult.rs:100-133 */
static int fm_decode(const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    if (plen < 1) return OQ_TRUNCATED;
    uint8_t tag = p[0];
    if (plen < 2) return OQ_TRUNCATED;
    uint8_t si = p[1];
    if (si >= 7) return OQ_CORRUPT;
    double scale = FM_SCALES[si];
    const uint8_t *rest = p + 2;
    size_t rlen = plen - 2;
    if (tag == 0) {
        int rc = for_decode(rest, rlen, n, true, out);
        if (rc) return rc;
    } else if (tag == 1) {
        buf_t d = {0};
        int rc = decode_residuals(rest, rlen, n * 10 + 16, &d);
        if (rc) {
            b_free(&d);
            return rc;
        }
        int64_t prev = 0;
        size_t pos = 0;
        for (size_t i = 0; i < n; i++) {
            uint64_t z;
            rc = varint_read(d.p, d.len, &pos, &z);
            if (rc) {
                b_free(&d);
                return rc;
            }
            prev = (int64_t)((uint64_t)prev + unzigzag64(z));
            out[i] = (uint64_t)prev;
        }
        bool trailing = pos != d.len;
        b_free(&d);
        if (trailing) return OQ_CORRUPT;
    } else {
        return OQ_CORRUPT;
    }
    for (size_t i = 0; i < n; i++) out[i] = f64_bits((double)(int64_t)out[i] / scale);
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* DICT — src/codecs/dict.rs:40-207                                          */
/* ------------------------------------------------------------------------ */

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}
/* dict.rs:40-61 */
static void dict_encode_values(const uint64_t *sorted, size_t card, bool entropy, uint8_t *tag, buf_t *blob) {
    buf_t raw = {0};
    for (size_t i = 0; i < card; i++) b_u64(&raw, sorted[i]);
    *tag = 0;
    *blob = raw;
    buf_t delta = {0};
    delta_encode(sorted, card, &delta);
    if (delta.len < blob->len) {
        b_free(blob);
        *tag = 1;
        *blob = delta;
    } else {
        b_free(&delta);
    }
    if (entropy) {
        uint8_t *tr = transpose_encode(sorted, card);
        buf_t c = {0};
        code_residuals(tr, card * 8, &c);
        free(tr);
        if (c.len < blob->len) {
            b_free(blob);
            *tag = 2;
            *blob = c;
        } else {
            b_free(&c);
        }
    }
}
/* dict.rs:87-152 */
static bool dict_encode(const uint64_t *v, size_t n, bool entropy, buf_t *out) {
    if (n == 0) return false;
    size_t max_card = n / 2 + 1;
    hmap_t h;
    hm_init(&h, 1024);
    uint64_t *dict = (uint64_t *)malloc(sizeof(uint64_t) * (max_card + 2));
    size_t card = 0;
    for (size_t i = 0; i < n; i++) {
        bool ins;
        uint32_t *slot = hm_entry(&h, v[i], &ins);
        if (ins) {
            dict[card] = v[i];
            card++;
            if (card > max_card) {
                hm_free(&h);
                free(dict);
                return false;
            }
        }
        (void)slot;
    }
    qsort(dict, card, 8, cmp_u64);
    for (size_t r = 0; r < card; r++) {
        bool ins;
        *hm_entry(&h, dict[r], &ins) = (uint32_t)r;
    }
    uint64_t *codes = (uint64_t *)malloc(n * 8);
    for (size_t i = 0; i < n; i++) {
        uint32_t r = 0;
        hm_get(&h, v[i], &r);
        codes[i] = r;
    }
    hm_free(&h);
    uint8_t vtag;
    buf_t vblob;
    dict_encode_values(dict, card, entropy, &vtag, &vblob);
    uint8_t ctag = 0;
    buf_t cblob = {0};
    for_encode(codes, n, false, &cblob);
    if (entropy && card <= (1u << 16)) {
        size_t nb = card <= 256 ? 1 : 2;
        buf_t e = {0};
        b_push(&e, (uint8_t)nb);
        uint8_t *plane = (uint8_t *)malloc(n);
        for (size_t pl = 0; pl < nb; pl++) {
            for (size_t i = 0; i < n; i++) plane[i] = (uint8_t)(codes[i] >> (8 * pl));
            buf_t c = {0};
            code_residuals(plane, n, &c);
            b_varint(&e, c.len);
            b_write(&e, c.p, c.len);
            b_free(&c);
        }
        free(plane);
        if (e.len < cblob.len) {
            b_free(&cblob);
            ctag = 1;
            cblob = e;
        } else {
            b_free(&e);
        }
    }
    b_varint(out, card);
    b_push(out, vtag);
    b_varint(out, vblob.len);
    b_write(out, vblob.p, vblob.len);
    b_push(out, ctag);
    b_write(out, cblob.p, cblob.len);
    b_free(&vblob);
    b_free(&cblob);
    free(codes);
    free(dict);
    return true;
}
/* dict.rs:64-85 */
static int dict_decode_values(uint8_t tag, const uint8_t *blob, size_t blen, size_t card, uint64_t *dict) {
    if (tag == 0) {
        if (blen != card * 8) return OQ_CORRUPT;
        for (size_t i = 0; i < card; i++) dict[i] = rd_u64(blob + 8 * i);
        return OQ_OK;
    }
    if (tag == 1) return delta_decode(blob, blen, card, dict);
    if (tag == 2) {
        buf_t b = {0};
        int rc = decode_residuals(blob, blen, card * 8, &b);
        if (!rc) rc = b.len != card * 8 ? OQ_CORRUPT : transpose_decode(b.p, b.len, card, dict);
        b_free(&b);
        return rc;
    }
    return OQ_CORRUPT;
}
/* dict.rs:154-207 */
static int dict_decode(const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    size_t pos = 0;
    uint64_t card64;
    int rc = varint_read(p, plen, &pos, &card64);
    if (rc) return rc;
    if (card64 > (uint64_t)n) return OQ_CORRUPT;
    size_t card = (size_t)card64;
    if (pos >= plen) return OQ_TRUNCATED;
    uint8_t vtag = p[pos++];
    uint64_t vlen;
    rc = varint_read(p, plen, &pos, &vlen);
    if (rc) return rc;
    if (vlen > (uint64_t)(plen - pos)) return OQ_TRUNCATED;
    uint64_t *dict = (uint64_t *)malloc((card ? card : 1) * 8);
    uint64_t *codes = (uint64_t *)calloc(n ? n : 1, 8);
    buf_t pl = {0};
    rc = dict_decode_values(vtag, p + pos, (size_t)vlen, card, dict);
    if (rc) goto done;
    pos += (size_t)vlen;
    if (pos >= plen) {
        rc = OQ_TRUNCATED;
        goto done;
    }
    uint8_t ctag = p[pos++];
    if (ctag == 0) {
        rc = for_decode(p + pos, plen - pos, n, false, codes);
        if (rc) goto done;
    } else if (ctag == 1) {
        if (pos >= plen) {
            rc = OQ_TRUNCATED;
            goto done;
        }
        size_t nb = p[pos++];
        if (nb < 1 || nb > 2) {
            rc = OQ_CORRUPT;
            goto done;
        }
        for (size_t k = 0; k < nb; k++) {
            uint64_t l;
            rc = varint_read(p, plen, &pos, &l);
            if (rc) goto done;
            if (l > (uint64_t)(plen - pos)) {
                rc = OQ_TRUNCATED;
                goto done;
            }
            pl.len = 0;
            rc = decode_residuals(p + pos, (size_t)l, n, &pl);
            if (rc) goto done;
            pos += (size_t)l;
            if (pl.len != n) {
                rc = OQ_CORRUPT;
                goto done;
            }
            for (size_t i = 0; i < n; i++) codes[i] |= (uint64_t)pl.p[i] << (8 * k);
        }
    } else {
        rc = OQ_CORRUPT;
        goto done;
    }
    for (size_t i = 0; i < n; i++) {
        if (codes[i] >= card) {
            rc = OQ_CORRUPT;
            goto done;
        }
        out[i] = dict[codes[i]];
    }
    rc = OQ_OK;
done:
    free(dict);
    free(codes);
    b_free(&pl);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* RLE — src/codecs/rle.rs:10-75                                             */
/* ------------------------------------------------------------------------ */

/* rle.rs:10-42 */
static bool rle_encode(const uint64_t *v, size_t n, buf_t *out) {
    if (n == 0) return false;
    size_t max_runs = n / 2 + 1;
    uint64_t *rv = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1));
    uint64_t *rl = (uint64_t *)malloc(sizeof(uint64_t) * (n + 1));
    size_t nr = 0;
    uint64_t prev = v[0], len = 0;
    for (size_t i = 0; i < n; i++) {
        if (v[i] == prev) {
            len++;
        } else {
            rv[nr] = prev;
            rl[nr] = len;
            nr++;
            prev = v[i];
            len = 1;
            if (nr > max_runs) {
                free(rv);
                free(rl);
                return false;
            }
        }
    }
    rv[nr] = prev;
    rl[nr] = len;
    nr++;
    b_varint(out, nr);
    for (size_t r = 0; r < nr; r++) b_u64(out, rv[r]);
    for_encode(rl, nr, false, out);
    free(rv);
    free(rl);
    return true;
}
/* rle.rs:44-75 */
static int rle_decode(const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    size_t pos = 0;
    uint64_t nr64;
    int rc = varint_read(p, plen, &pos, &nr64);
    if (rc) return rc;
    if (nr64 > (uint64_t)n) return OQ_CORRUPT;
    size_t nr = (size_t)nr64;
    uint64_t *rv = (uint64_t *)malloc((nr ? nr : 1) * 8), *rl = (uint64_t *)malloc((nr ? nr : 1) * 8);
    for (size_t r = 0; r < nr; r++) {
        if (plen < pos + 8) {
            free(rv);
            free(rl);
            return OQ_TRUNCATED;
        }
        rv[r] = rd_u64(p + pos);
        pos += 8;
    }
    rc = for_decode(p + pos, plen - pos, nr, false, rl);
    if (rc) {
        free(rv);
        free(rl);
        return rc;
    }
    size_t got = 0;
    for (size_t r = 0; r < nr; r++) {
        uint64_t l = rl[r];
        if (l > (uint64_t)(n - got)) {
            free(rv);
            free(rl);
            return OQ_CORRUPT;
        }
        for (uint64_t k = 0; k < l; k++) out[got++] = rv[r];
    }
    free(rv);
    free(rl);
    if (got != n) return OQ_LENGTH_MISMATCH;
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* Validity bitmap — src/validity.rs:17-146                                  */
/* ------------------------------------------------------------------------ */

static bool bm_is_set(const uint8_t *bm, size_t i) { return (bm[i >> 3] >> (i & 7)) & 1; }

/* validity.rs:28-37 */
static size_t count_valid(const uint8_t *bm, size_t n) {
    size_t c = 0, full = n / 8;
    for (size_t i = 0; i < full; i++) c += (size_t)__builtin_popcount(bm[i]);
    size_t rem = n & 7;
    if (rem) c += (size_t)__builtin_popcount(bm[full] & ((1u << rem) - 1));
    return c;
}
/* validity.rs:40-70 */
static void validity_encode(const uint8_t *bm, size_t n, buf_t *out) {
    buf_t rle = {0};
    uint8_t cur = 0;
    uint64_t run = 0;
    for (size_t i = 0; i < n; i++) {
        uint8_t bit = bm_is_set(bm, i);
        if (bit == cur) {
            run++;
        } else {
            b_varint(&rle, run);
            cur ^= 1;
            run = 1;
        }
    }
    b_varint(&rle, run);
    size_t raw_len = (n + 7) / 8;
    if (rle.len < raw_len) {
        b_push(out, 1);
        b_write(out, rle.p, rle.len);
    } else {
        b_push(out, 0);
        b_write(out, bm, raw_len);
    }
    b_free(&rle);
}
/* validity.rs:73-119.  `bm` must hold ceil(n/8) bytes. */
static int validity_decode(const uint8_t *blob, size_t blen, size_t n, uint8_t *bm) {
    size_t raw_len = (n + 7) / 8;
    memset(bm, 0, raw_len);
    if (blen == 0) return OQ_TRUNCATED;
    uint8_t tag = blob[0];
    const uint8_t *rest = blob + 1;
    size_t rlen = blen - 1;
    if (tag == 0) {
        if (rlen < raw_len) return OQ_TRUNCATED;
        memcpy(bm, rest, raw_len);
        if (n & 7) bm[raw_len - 1] &= (uint8_t)((1u << (n & 7)) - 1);
        return OQ_OK;
    }
    if (tag == 1) {
        size_t pos = 0, i = 0;
        uint8_t cur = 0;
        while (i < n) {
            uint64_t run;
            int rc = varint_read(rest, rlen, &pos, &run);
            if (rc) return rc;
            if (run > (uint64_t)(n - i)) return OQ_CORRUPT;
            size_t end = i + (size_t)run;
            if (cur == 1)
                for (size_t k = i; k < end; k++) bm[k >> 3] |= (uint8_t)(1u << (k & 7));
            i = end;
            cur ^= 1;
        }
        return OQ_OK;
    }
    return OQ_CORRUPT;
}

/* ------------------------------------------------------------------------ */
/* Block planning + competition — src/encoder.rs                             */
/* ------------------------------------------------------------------------ */

enum {
    M_PRED = 0, M_CONST = 1, M_STRIDE = 2, M_XORZ = 3, M_LZ = 4, M_RAW = 5, M_ORDERED_DELTA = 7,
    M_ALP = 9, M_BYTE_TRANSPOSE = 11, M_FLOAT_MULT = 17, M_DICT = 19, M_DELTA2 = 20,
    M_PRED2 = 25, M_PRED_RC = 29, M_DELTA_DP = 45, M_FOR_BITPACK = 50, M_DELTA_BITPACK = 51,
    M_ALP_RD = 52, M_RLE = 53, M_PCO = 54
};

static _Atomic uint64_t g_wins[64]; /* src/diag.rs:8-23 */

/* mode.rs:60-84 */
static bool mode_known(int id) {
    switch (id) {
        case 0: case 1: case 2: case 3: case 4: case 5: case 7: case 9: case 11: case 17:
        case 19: case 20: case 25: case 29: case 45: case 50: case 51: case 52: case 53: case 54:
            return true;
        default: return false;
    }
}
/* encoder.rs:79-89 */
static uint64_t decode_weight(int m) {
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
static uint64_t level_lambda(int level) { return level == 0 ? 16 : level == 1 ? 4 : level == 2 ? 2 : 0; } /* lib.rs:126-138 */

typedef struct {
    uint32_t exp_range;
    bool distinct_low, repeats;
} feats_t;

/* encoder.rs:705-750 */
static feats_t probe_block_features(const uint64_t *b, size_t n) {
    feats_t f;
    if (n == 0) {
        f.exp_range = 0;
        f.distinct_low = true;
        f.repeats = false;
        return f;
    }
    uint32_t min_exp = UINT32_MAX, max_exp = 0, consec_eq = 0;
    uint64_t prev = b[0];
    for (size_t i = 0; i < n; i++) {
        uint32_t e = (uint32_t)((b[i] >> 52) & 0x7FF);
        if (e < min_exp) min_exp = e;
        if (e > max_exp) max_exp = e;
        consec_eq += b[i] == prev;
        prev = b[i];
    }
    uint64_t seen[256] = {0};
    uint32_t distinct = 0;
    size_t stride = n / 4096 ? n / 4096 : 1;
    for (size_t k = 0; k < n; k += stride) {
        uint64_t h = b[k] * 0x9E3779B97F4A7C15ull;
        size_t bucket = (size_t)((h >> 50) & 0x3FFF);
        uint64_t bit = 1ull << (bucket & 63);
        if (!(seen[bucket >> 6] & bit)) {
            seen[bucket >> 6] |= bit;
            distinct++;
        }
    }
    f.exp_range = max_exp - min_exp;
    f.distinct_low = distinct < 2048;
    uint64_t c2 = (uint64_t)consec_eq * 2;
    if (c2 > UINT32_MAX) c2 = UINT32_MAX; /* saturating_mul on u32 */
    f.repeats = c2 > (uint64_t)(uint32_t)n;
    return f;
}
/* encoder.rs:655-683 */
static bool looks_incompressible(const uint64_t *b, size_t n, const feats_t *f, size_t lb) {
    if (f->distinct_low || f->repeats || n < 256) return false;
    uint32_t lane_bits = (uint32_t)(lb * 8);
    uint32_t thr = lane_bits >= 4 ? lane_bits - 4 : 0;
    size_t step = n / 2048 ? n / 2048 : 1;
    uint64_t vmin = b[0], vmax = b[0], dmax = 0;
    for (size_t i = step; i < n; i += step) {
        uint64_t v = b[i];
        if (v < vmin) vmin = v;
        if (v > vmax) vmax = v;
        uint64_t zz = zigzag64(v - b[i - 1]);
        if (zz > dmax) dmax = zz;
    }
    uint32_t vw = (uint32_t)(64 - clz64(vmax - vmin));
    uint32_t dw = dmax == 0 ? 0 : (uint32_t)(64 - clz64(dmax));
    return vw >= thr && dw >= thr;
}
/* encoder.rs:644-646 */
static bool looks_compressible(size_t res, size_t raw) { return (uint64_t)res * 20 < (uint64_t)raw * 19; }

typedef struct {
    int mode;
    buf_t payload;
    uint64_t score;
    uint64_t lambda, decoded_bytes;
} best_t;

static uint64_t penalty(int mode, uint64_t lambda, uint64_t db) { return (lambda * decode_weight(mode) * db) >> 8; } /* encoder.rs:94-97 */

/* encoder.rs:126-139 (runner-up bookkeeping only feeds the Max-level cascade) */
static void consider(best_t *b, int mode, buf_t *payload) {
    uint64_t s = payload->len + penalty(mode, b->lambda, b->decoded_bytes);
    if (s < b->score) {
        b_free(&b->payload);
        b->payload = *payload;
        b->mode = mode;
        b->score = s;
        payload->p = NULL;
        payload->len = payload->cap = 0;
    } else {
        b_free(payload);
    }
}

static void frame_bytes(int mode, size_t n, const buf_t *payload, buf_t *out) { /* encoder.rs:752-759 */
    b_push(out, (uint8_t)mode);
    b_u32(out, (uint32_t)n);
    b_u32(out, (uint32_t)payload->len);
    b_write(out, payload->p, payload->len);
}

/* encoder.rs:275-469 for Fastest / Fast / Balanced (Lz, Pco, predictors and
 * the LZ cascade are outside the in-path pool and never reached at these
 * levels except Lz/Pco at Balanced, which are skipped). */
static void encode_block_full(const uint64_t *b, size_t n, int dtype, int level, buf_t *out) {
    bool fam_float = dtype_float(dtype);
    bool entropy = level >= 2, reduced = level == 0;
    uint64_t lambda = level_lambda(level);
    size_t lb = lane_bytes(dtype);
    uint64_t decoded_bytes = (uint64_t)n * lb, raw_bytes = (uint64_t)n * 8;
    feats_t feats = probe_block_features(b, n);
    if (!fam_float && looks_incompressible(b, n, &feats, lb)) {
        atomic_fetch_add(&g_wins[M_RAW], 1);
        buf_t r = {0};
        raw_encode(b, n, dtype, &r);
        frame_bytes(M_RAW, n, &r, out);
        b_free(&r);
        return;
    }
    best_t best = {0};
    best.lambda = lambda;
    best.decoded_bytes = decoded_bytes;
    best.mode = M_RAW;
    raw_encode(b, n, dtype, &best.payload);
    best.score = best.payload.len + penalty(M_RAW, lambda, decoded_bytes);
    buf_t p = {0};
    if (const_encode(b, n, &p)) consider(&best, M_CONST, &p); else b_free(&p);
    if (stride_encode(b, n, &p)) consider(&best, M_STRIDE, &p); else b_free(&p);
    if (!reduced) {
        xorz_encode(b, n, &p);
        consider(&best, M_XORZ, &p);
    }
    for_encode(b, n, dtype_signed(dtype), &p);
    consider(&best, M_FOR_BITPACK, &p);
    delta_encode(b, n, &p);
    consider(&best, M_DELTA_BITPACK, &p);
    if (fam_float && !reduced) {
        if (fm_encode(b, n, entropy, &p)) consider(&best, M_FLOAT_MULT, &p); else b_free(&p);
        if (alp_encode(b, n, &p)) consider(&best, M_ALP, &p); else b_free(&p);
        if (alprd_encode(b, n, entropy, &p)) consider(&best, M_ALP_RD, &p); else b_free(&p);
    }
    bool block_compressible = looks_compressible(best.payload.len, raw_bytes);
    if (entropy && block_compressible && (feats.exp_range <= 64 || feats.repeats)) {
        uint8_t *tr = transpose_encode(b, n);
        code_residuals(tr, n * 8, &p);
        free(tr);
        consider(&best, M_BYTE_TRANSPOSE, &p);
    }
    if (block_compressible && !reduced) {
        if (dict_encode(b, n, entropy, &p)) consider(&best, M_DICT, &p); else b_free(&p);
        if (rle_encode(b, n, &p)) consider(&best, M_RLE, &p); else b_free(&p);
    }
    atomic_fetch_add(&g_wins[best.mode], 1);
    frame_bytes(best.mode, n, &best.payload, out);
    b_free(&best.payload);
}

/* ------------------------------------------------------------------------ */
/* Selection::Sample — encoder.rs:470-620, mode gates encoder.rs:24-60        */
/* ------------------------------------------------------------------------ */

/* The in-pool members of SAMPLE_MODES (encoder.rs:479-495), in its order; the
 * predictor modes between Xorz and FloatMult run only at High/Max. */
static const int SAMPLE_POOL[] = {M_XORZ, M_FLOAT_MULT, M_BYTE_TRANSPOSE, M_FOR_BITPACK, M_DELTA_BITPACK,
                                  M_ALP, M_ALP_RD, M_DICT, M_RLE};
#define SAMPLE_RUNS 8
#define SAMPLE_RUN_LEN 64

/* mode_runs (encoder.rs:50-60): float-only modes, and the entropy modes at
 * Balanced and above. */
static bool sample_mode_runs(int mode, bool fam_float, int level) {
    if ((mode == M_FLOAT_MULT || mode == M_ALP || mode == M_ALP_RD) && !fam_float) return false;
    if ((mode == M_FLOAT_MULT || mode == M_BYTE_TRANSPOSE) && level < 2) return false;
    return true;
}

/* encode_mode (encoder.rs:543-572) for the in-pool modes; false when the mode
 * does not apply. */
static bool sample_encode_mode(int mode, const uint64_t *b, size_t n, int dtype, int level, buf_t *out) {
    bool entropy = level >= 2;
    switch (mode) {
        case M_XORZ: xorz_encode(b, n, out); return true;
        case M_FOR_BITPACK: for_encode(b, n, dtype_signed(dtype), out); return true;
        case M_DELTA_BITPACK: delta_encode(b, n, out); return true;
        case M_FLOAT_MULT: return fm_encode(b, n, entropy, out);
        case M_ALP: return alp_encode(b, n, out);
        case M_ALP_RD: return alprd_encode(b, n, entropy, out);
        case M_DICT: return dict_encode(b, n, entropy, out);
        case M_RLE: return rle_encode(b, n, out);
        case M_BYTE_TRANSPOSE: {
            if (n == 0) return false;
            uint8_t *tr = transpose_encode(b, n);
            code_residuals(tr, n * 8, out);
            free(tr);
            return true;
        }
        default: return false;
    }
}

/* encoder.rs:574-620 for the in-pool modes (Lz and Pco, which Balanced would
 * try on the full block, are outside the pool): RAW, then CONST and STRIDE on
 * the full block, then the winner of the sample estimates encoded in full. */
static void encode_block_sampled(const uint64_t *b, size_t n, int dtype, int level, buf_t *out) {
    bool fam_float = dtype_float(dtype);
    best_t best = {0};
    best.lambda = level_lambda(level);
    best.decoded_bytes = (uint64_t)n * lane_bytes(dtype);
    best.mode = M_RAW;
    raw_encode(b, n, dtype, &best.payload);
    best.score = best.payload.len + penalty(M_RAW, best.lambda, best.decoded_bytes);
    buf_t p = {0};
    if (const_encode(b, n, &p)) consider(&best, M_CONST, &p); else b_free(&p);
    if (stride_encode(b, n, &p)) consider(&best, M_STRIDE, &p); else b_free(&p);
    /* build_sample (encoder.rs:503-516): 8 runs of 64 spread over the block */
    size_t total = SAMPLE_RUNS * SAMPLE_RUN_LEN, m = n;
    uint64_t *smp = (uint64_t *)malloc((n < total ? n : total) * 8 + 8);
    if (n <= total) {
        memcpy(smp, b, n * 8);
    } else {
        m = total;
        for (size_t r = 0; r < SAMPLE_RUNS; r++) {
            size_t start = r * (n - SAMPLE_RUN_LEN) / (SAMPLE_RUNS - 1);
            memcpy(smp + r * SAMPLE_RUN_LEN, b + start, SAMPLE_RUN_LEN * 8);
        }
    }
    int win = -1;
    size_t win_est = SIZE_MAX;
    for (size_t k = 0; k < sizeof SAMPLE_POOL / sizeof SAMPLE_POOL[0]; k++) {
        int mode = SAMPLE_POOL[k];
        if (!sample_mode_runs(mode, fam_float, level)) continue;
        buf_t e = {0};
        if (sample_encode_mode(mode, smp, m, dtype, level, &e) && e.len < win_est) {
            win_est = e.len;
            win = mode;
        }
        b_free(&e);
    }
    free(smp);
    if (win >= 0 && sample_encode_mode(win, b, n, dtype, level, &p)) consider(&best, win, &p); else b_free(&p);
    atomic_fetch_add(&g_wins[best.mode], 1);
    frame_bytes(best.mode, n, &best.payload, out);
    b_free(&best.payload);
}

/* encoder.rs:244-256: the level argument carries OQ_SELECT_SAMPLE for
 * Selection::Sample. */
static void encode_block(const uint64_t *b, size_t n, int dtype, int level, buf_t *out) {
    if (level & OQ_SELECT_SAMPLE) encode_block_sampled(b, n, dtype, level & 0xFF, out);
    else encode_block_full(b, n, dtype, level, out);
}

/* encoder.rs:154-178 */
/* plan_blocks' probe (encoder.rs:168-170) for every 32,768-value window of a
 * lane: flags[w] = 1 where a block starting at window w grows to MAX_QUANTUM. */
void oq_probe_windows(const uint64_t *v, size_t n, uint8_t *flags) {
    for (size_t w = 0; w * 32768 < n; w++) {
        size_t s = w * 32768, e = s + 32768 < n ? s + 32768 : n;
        feats_t f = probe_block_features(v + s, e - s);
        flags[w] = (f.distinct_low || f.repeats) ? 1 : 0;
    }
}

static size_t plan_blocks(const uint64_t *v, size_t n, long block_size, size_t **starts_out) {
    size_t cap = n / 32768 + 2, nb = 0;
    if (block_size > 0) {
        size_t bs = (size_t)block_size;
        if (bs > 131072) bs = 131072;
        cap = n / bs + 2;
    }
    size_t *st = (size_t *)malloc(sizeof(size_t) * (cap + 1));
    size_t s = 0;
    while (s < n) {
        size_t end;
        if (block_size > 0) {
            size_t bs = (size_t)block_size;
            if (bs > 131072) bs = 131072;
            end = s + bs < n ? s + bs : n;
        } else {
            size_t base_end = s + 32768 < n ? s + 32768 : n;
            feats_t f = probe_block_features(v + s, base_end - s);
            if (f.distinct_low || f.repeats)
                end = s + 131072 < n ? s + 131072 : n;
            else
                end = base_end;
        }
        st[nb++] = s;
        s = end;
    }
    st[nb] = n;
    *starts_out = st;
    return nb;
}

typedef struct {
    const uint64_t *vals;
    const size_t *starts;
    size_t nb;
    int dtype, level;
    buf_t *frames;
    _Atomic size_t next;
} enc_job_t;

static void *enc_worker(void *arg) {
    enc_job_t *j = (enc_job_t *)arg;
    for (;;) {
        size_t k = atomic_fetch_add(&j->next, 1);
        if (k >= j->nb) break;
        encode_block(j->vals + j->starts[k], j->starts[k + 1] - j->starts[k], j->dtype, j->level, &j->frames[k]);
    }
    return NULL;
}

static uint8_t clamp_plog2(int p) { return (uint8_t)(p < 10 ? 10 : p > 16 ? 16 : p); }

/* encoder.rs:184-214 (+ build_frames 216-242) */
static void compress_lane_buf(const uint64_t *vals, size_t n_valid, int dtype, size_t logical_n,
                              const uint8_t *validity, int level, long block_size, int plog2,
                              int threads, buf_t *out) {
    size_t *starts;
    size_t nb = plan_blocks(vals, n_valid, block_size, &starts);
    buf_t *frames = (buf_t *)calloc(nb ? nb : 1, sizeof(buf_t));
    enc_job_t job = {vals, starts, nb, dtype, level, frames, 0};
    if (threads > 1 && nb > 1) {
        int t = threads;
        pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)t);
        for (int i = 0; i < t; i++) pthread_create(&th[i], NULL, enc_worker, &job);
        for (int i = 0; i < t; i++) pthread_join(th[i], NULL);
        free(th);
    } else {
        enc_worker(&job);
    }
    b_write(out, "FCR1", 4);
    b_push(out, 2);
    b_push(out, validity ? 1 : 0);
    b_push(out, clamp_plog2(plog2));
    b_push(out, (uint8_t)dtype);
    b_u64(out, logical_n);
    if (validity) {
        buf_t vb = {0};
        validity_encode(validity, logical_n, &vb);
        b_varint(out, vb.len);
        b_write(out, vb.p, vb.len);
        b_free(&vb);
    }
    for (size_t k = 0; k < nb; k++) {
        b_write(out, frames[k].p, frames[k].len);
        b_free(&frames[k]);
    }
    free(frames);
    free(starts);
}

/* ------------------------------------------------------------------------ */
/* Stream decoder — src/decoder.rs:43-190, src/format.rs:65-94               */
/* ------------------------------------------------------------------------ */

/* decoder.rs:145-190 (in-path modes) */
/* ------------------------------------------------------------------------ */
/* Linear recurrences — src/codecs/linear.rs (High / Max modes): ORDERED_DELTA */
/* (second difference of the u64 patterns, zigzag LEB128), DELTA2 (XOR with a */
/* polynomial extrapolation in f64) and DELTA_DP (the f64 residual, verified  */
/* invertible).  The frame payload is the entropy-coded residual bytes.        */
/* ------------------------------------------------------------------------ */

/* linear.rs:31-45 */
static void idelta2_encode(const uint64_t *v, size_t n, buf_t *out) {
    uint64_t p1 = 0, p2 = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t pred = i == 0 ? 0 : i == 1 ? p1 : p1 * 2 - p2;
        b_varint(out, zigzag64(v[i] - pred));
        p2 = p1;
        p1 = v[i];
    }
}
/* linear.rs:47-66 */
static int idelta2_decode(const uint8_t *p, size_t len, size_t n, uint64_t *out) {
    uint64_t p1 = 0, p2 = 0;
    size_t pos = 0;
    for (size_t i = 0; i < n; i++) {
        uint64_t pred = i == 0 ? 0 : i == 1 ? p1 : p1 * 2 - p2, r;
        int rc = varint_read(p, len, &pos, &r);
        if (rc) return rc;
        uint64_t v = pred + unzigzag64(r);
        out[i] = v;
        p2 = p1;
        p1 = v;
    }
    return pos == len ? OQ_OK : OQ_CORRUPT;
}

static uint64_t f64_to_bits(double d);
static double bits_to_f64(uint64_t b);
/* f64 arithmetic with NaN operands propagated as x86 SSE does in source
 * order (the first NaN operand, quieted; an invalid operation gives the
 * default NaN 0xFFF8...), written out so the result does not depend on how a
 * compiler orders the operands. */
static double nan_op(double a, double b, double r) {
    if (isnan(a)) return bits_to_f64(f64_to_bits(a) | 0x0008000000000000ull);
    if (isnan(b)) return bits_to_f64(f64_to_bits(b) | 0x0008000000000000ull);
    if (isnan(r)) return bits_to_f64(0xFFF8000000000000ull);
    return r;
}
static double x_mul(double a, double b) { return nan_op(a, b, a * b); }
static double x_add(double a, double b) { return nan_op(a, b, a + b); }
static double x_sub(double a, double b) { return nan_op(a, b, a - b); }

/* linear.rs:75-100: Newton extrapolation, most recent first; the effective
 * order drops to the history available.  pred = 0.0 + c0*h0 + c1*h1 + ...,
 * each product and sum rounded on its own (no FMA). */
static double lin_predict(const double *h, size_t avail, int order) {
    static const int coef[5][4] = {{0}, {1}, {2, -1}, {3, -3, 1}, {4, -6, 4, -1}};
    int eff = (size_t)order < avail ? order : (int)avail;
    if (eff == 0) return 0.0;
    double pred = 0.0;
    for (int k = 0; k < eff; k++) pred = x_add(pred, x_mul((double)coef[eff][k], h[k]));
    return pred;
}
static void lin_push(double *h, double v) {
    h[3] = h[2];
    h[2] = h[1];
    h[1] = h[0];
    h[0] = v;
}
static uint64_t f64_to_bits(double d) {
    uint64_t b;
    memcpy(&b, &d, 8);
    return b;
}
static double bits_to_f64(uint64_t b) {
    double d;
    memcpy(&d, &b, 8);
    return d;
}

/* linear.rs:121-140: the order whose order-th difference of a 1,024-value
 * window from the middle of the block has the smallest mean magnitude. */
static int lin_select_order(const uint64_t *v, size_t n) {
    if (n < 8) return 2;
    size_t win = n < 1024 ? n : 1024, start = (n - win) / 2, len = win;
    double *d = (double *)malloc(win * sizeof(double));
    for (size_t i = 0; i < win; i++) d[i] = bits_to_f64(v[start + i]);
    int best = 1;
    double best_mag = INFINITY;
    for (int order = 1; order <= 4; order++) {
        for (size_t i = 0; i + 1 < len; i++) d[i] = d[i + 1] - d[i];
        if (len) len--;
        double mag = INFINITY;
        if (len) {
            double sum = -0.0;
            for (size_t i = 0; i < len; i++) sum += fabs(d[i]);
            mag = sum / (double)len;
        }
        if (isfinite(mag) && mag < best_mag) {
            best_mag = mag;
            best = order;
        }
    }
    free(d);
    return best;
}

/* linear.rs:146-157 */
static void delta2_encode(const uint64_t *v, size_t n, int order, buf_t *out) {
    b_push(out, (uint8_t)order);
    double h[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < n; i++) {
        uint64_t pred = f64_to_bits(lin_predict(h, i < 4 ? i : 4, order));
        b_varint(out, v[i] ^ pred);
        lin_push(h, bits_to_f64(v[i]));
    }
}
/* linear.rs:159-179 */
static int delta2_decode(const uint8_t *p, size_t len, size_t n, uint64_t *out) {
    if (len == 0) return OQ_TRUNCATED;
    int order = p[0];
    if (order < 1 || order > 4) return OQ_CORRUPT;
    double h[4] = {0, 0, 0, 0};
    size_t pos = 1;
    for (size_t i = 0; i < n; i++) {
        uint64_t pred = f64_to_bits(lin_predict(h, i < 4 ? i : 4, order)), r;
        int rc = varint_read(p, len, &pos, &r);
        if (rc) return rc;
        out[i] = r ^ pred;
        lin_push(h, bits_to_f64(out[i]));
    }
    return pos == len ? OQ_OK : OQ_CORRUPT;
}

/* linear.rs:190-213: false when some value does not survive pred + (v - pred) */
static bool dp_encode(const uint64_t *v, size_t n, int order, buf_t *out) {
    if (n == 0) return false;
    b_push(out, (uint8_t)order);
    double h[4] = {0, 0, 0, 0};
    uint64_t prev = 0;
    for (size_t i = 0; i < n; i++) {
        double x = bits_to_f64(v[i]), pred = lin_predict(h, i < 4 ? i : 4, order), r = x_sub(x, pred);
        if (f64_to_bits(x_add(pred, r)) != v[i]) return false;
        uint64_t rb = f64_to_bits(r);
        b_varint(out, rb ^ prev);
        prev = rb;
        lin_push(h, x);
    }
    return true;
}
/* linear.rs:215-237 */
static int dp_decode(const uint8_t *p, size_t len, size_t n, uint64_t *out) {
    if (len == 0) return OQ_TRUNCATED;
    int order = p[0];
    if (order < 1 || order > 4) return OQ_CORRUPT;
    double h[4] = {0, 0, 0, 0};
    uint64_t prev = 0;
    size_t pos = 1;
    for (size_t i = 0; i < n; i++) {
        double pred = lin_predict(h, i < 4 ? i : 4, order);
        uint64_t r;
        int rc = varint_read(p, len, &pos, &r);
        if (rc) return rc;
        uint64_t rb = r ^ prev;
        double x = x_add(pred, bits_to_f64(rb));
        out[i] = f64_to_bits(x);
        prev = rb;
        lin_push(h, x);
    }
    return pos == len ? OQ_OK : OQ_CORRUPT;
}

/* ------------------------------------------------------------------------ */
/* FCM / DFCM predictors — src/codecs/pred.rs with src/hash.rs (High / Max):  */
/* a 2^predictor_log2 table indexed by CRC32C(seed, context) predicts the    */
/* value (FCM: the last value seen after the context value; DFCM: the last   */
/* value + the last delta seen after the context delta); residuals are XORs, */
/* LEB128.                                                                   */
/* ------------------------------------------------------------------------ */
#define HASH_SEED 0x9e3779b9u

/* hash.rs:18-31: CRC32C (reflected 0x82F63B78) over the 8 bytes of v */
static uint32_t crc32c_u64(uint32_t crc, uint64_t v) {
    for (int i = 0; i < 8; i++) {
        crc ^= (uint32_t)(v & 0xff);
        v >>= 8;
        for (int k = 0; k < 8; k++) crc = (crc >> 1) ^ (0x82F63B78u & (0u - (crc & 1u)));
    }
    return crc;
}

/* pred.rs:23-35 */
static void fcm_encode(const uint64_t *v, size_t n, int plog2, buf_t *out) {
    size_t mask = ((size_t)1 << plog2) - 1, ctx = 0;
    uint64_t *table = (uint64_t *)calloc(mask + 1, 8);
    for (size_t i = 0; i < n; i++) {
        b_varint(out, v[i] ^ table[ctx]);
        table[ctx] = v[i];
        ctx = crc32c_u64(HASH_SEED, v[i]) & mask;
    }
    free(table);
}
/* pred.rs:37-58 */
static int fcm_decode(const uint8_t *p, size_t len, size_t n, int plog2, uint64_t *out) {
    size_t mask = ((size_t)1 << plog2) - 1, ctx = 0, pos = 0;
    uint64_t *table = (uint64_t *)calloc(mask + 1, 8);
    int rc = OQ_OK;
    for (size_t i = 0; i < n && !rc; i++) {
        uint64_t r;
        rc = varint_read(p, len, &pos, &r);
        if (rc) break;
        uint64_t v = r ^ table[ctx];
        out[i] = v;
        table[ctx] = v;
        ctx = crc32c_u64(HASH_SEED, v) & mask;
    }
    free(table);
    if (rc) return rc;
    return pos == len ? OQ_OK : OQ_CORRUPT;
}
/* pred.rs:60-76 */
static void dfcm_encode(const uint64_t *v, size_t n, int plog2, buf_t *out) {
    size_t mask = ((size_t)1 << plog2) - 1, dctx = 0;
    uint64_t *table = (uint64_t *)calloc(mask + 1, 8), last = 0;
    for (size_t i = 0; i < n; i++) {
        b_varint(out, v[i] ^ (last + table[dctx]));
        uint64_t delta = v[i] - last;
        table[dctx] = delta;
        dctx = crc32c_u64(HASH_SEED, delta) & mask;
        last = v[i];
    }
    free(table);
}
/* pred.rs:78-98 */
static int dfcm_decode(const uint8_t *p, size_t len, size_t n, int plog2, uint64_t *out) {
    size_t mask = ((size_t)1 << plog2) - 1, dctx = 0, pos = 0;
    uint64_t *table = (uint64_t *)calloc(mask + 1, 8), last = 0;
    int rc = OQ_OK;
    for (size_t i = 0; i < n; i++) {
        uint64_t pred = last + table[dctx], r;
        rc = varint_read(p, len, &pos, &r);
        if (rc) break;
        uint64_t v = r ^ pred;
        out[i] = v;
        uint64_t delta = v - last;
        table[dctx] = delta;
        dctx = crc32c_u64(HASH_SEED, delta) & mask;
        last = v;
    }
    free(table);
    if (rc) return rc;
    return pos == len ? OQ_OK : OQ_CORRUPT;
}

/* decoder.rs:150-171: entropy-coded residuals (bound 10n + 16), then the recurrence */
static int linear_frame_decode(int mode, const uint8_t *p, size_t plen, size_t n, uint64_t *out);

static int pred_frame_decode(int mode, const uint8_t *p, size_t plen, size_t n, int plog2, uint64_t *out);

static int decode_frame(int mode, const uint8_t *p, size_t plen, size_t n, int dtype, int plog2, uint64_t *out) {
    switch (mode) {
        case M_RAW: return raw_decode(p, plen, n, dtype, out);
        case M_CONST:
            if (plen != 8) return OQ_CORRUPT;
            for (size_t i = 0; i < n; i++) out[i] = rd_u64(p);
            return OQ_OK;
        case M_STRIDE: {
            if (plen != 16) return OQ_CORRUPT;
            uint64_t first = rd_u64(p), stride = rd_u64(p + 8);
            for (size_t i = 0; i < n; i++) out[i] = first + (uint64_t)i * stride;
            return OQ_OK;
        }
        case M_XORZ: return xorz_decode(p, plen, n, out);
        case M_BYTE_TRANSPOSE: {
            buf_t b = {0};
            int rc = decode_residuals(p, plen, n * 8 + 16, &b);
            if (!rc) rc = transpose_decode(b.p, b.len, n, out);
            b_free(&b);
            return rc;
        }
        case M_FLOAT_MULT: return fm_decode(p, plen, n, out);
        case M_FOR_BITPACK: return for_decode(p, plen, n, dtype_signed(dtype), out);
        case M_ALP: return alp_decode(p, plen, n, out);
        case M_DELTA_BITPACK: return delta_decode(p, plen, n, out);
        case M_ALP_RD: return alprd_decode(p, plen, n, out);
        case M_DICT: return dict_decode(p, plen, n, out);
        case M_RLE: return rle_decode(p, plen, n, out);
        case M_ORDERED_DELTA:
        case M_DELTA2:
        case M_DELTA_DP: return linear_frame_decode(mode, p, plen, n, out);
        case M_PRED:
        case M_PRED_RC:
        case M_PRED2: return pred_frame_decode(mode, p, plen, n, plog2, out);
        case M_LZ: { /* decoder.rs:172-175, lz.rs:165-172 */
            buf_t b = {0}, o = {0};
            int rc = decode_residuals(p, plen, n * 16 + 1024, &b);
            if (!rc) rc = lz_decompress(b.p, b.len, n * 8, &o);
            if (!rc)
                for (size_t i = 0; i < n; i++) out[i] = rd_u64(o.p + 8 * i);
            b_free(&b);
            b_free(&o);
            return rc;
        }
        default: return OQ_UNSUPPORTED;
    }
}

/* decoder.rs:150-157: PRED reads LEB128 residuals directly, PRED_RC and
 * PRED2 entropy-coded ones (bound 10n + 16) */
static int pred_frame_decode(int mode, const uint8_t *p, size_t plen, size_t n, int plog2, uint64_t *out) {
    if (mode == M_PRED) return fcm_decode(p, plen, n, plog2, out);
    buf_t b = {0};
    int rc = decode_residuals(p, plen, n * 10 + 16, &b);
    if (!rc) rc = mode == M_PRED_RC ? fcm_decode(b.p, b.len, n, plog2, out) : dfcm_decode(b.p, b.len, n, plog2, out);
    b_free(&b);
    return rc;
}

static int linear_frame_decode(int mode, const uint8_t *p, size_t plen, size_t n, uint64_t *out) {
    buf_t b = {0};
    int rc = decode_residuals(p, plen, n * 10 + 16, &b);
    if (!rc) {
        if (mode == M_ORDERED_DELTA) rc = idelta2_decode(b.p, b.len, n, out);
        else if (mode == M_DELTA2) rc = delta2_decode(b.p, b.len, n, out);
        else rc = dp_decode(b.p, b.len, n, out);
    }
    b_free(&b);
    return rc;
}

typedef struct {
    int mode;
    size_t n, off;
    const uint8_t *payload;
    size_t plen;
} frame_t;

typedef struct {
    const frame_t *frames;
    size_t nf;
    int dtype;
    int plog2; /* the header's predictor_log2 (format.rs:56-94) */
    uint64_t *lane;
    int *rcs;
    _Atomic size_t next;
} dec_job_t;

static void *dec_worker(void *arg) {
    dec_job_t *j = (dec_job_t *)arg;
    for (;;) {
        size_t k = atomic_fetch_add(&j->next, 1);
        if (k >= j->nf) break;
        const frame_t *f = &j->frames[k];
        j->rcs[k] = decode_frame(f->mode, f->payload, f->plen, f->n, j->dtype, j->plog2, j->lane + f->off);
    }
    return NULL;
}

#define MAX_BITMAP_BYTES ((size_t)1 << 36)

/* format.rs:65-94 */
static int header_read(const uint8_t *src, size_t len, int *dtype, bool *hv, uint64_t *n) {
    if (len < 16) return OQ_TRUNCATED;
    if (memcmp(src, "FCR1", 4) != 0) return OQ_BAD_MAGIC;
    if (src[4] != 2) return OQ_UNSUPPORTED_VERSION;
    if (src[5] & ~1u) return OQ_CORRUPT;
    if (src[6] < 10 || src[6] > 16) return OQ_CORRUPT;
    if (src[7] > 7) return OQ_UNSUPPORTED_DTYPE;
    *hv = src[5] & 1;
    *dtype = src[7];
    *n = rd_u64(src + 8);
    return OQ_OK;
}

/* decoder.rs:43-118.  On success *lane_out holds logical_n words (null slots
 * 0) and *bm_out the bitmap or NULL. */
static int decompress_lane(const uint8_t *src, size_t len, int threads, int *dtype_out, size_t *n_out,
                           uint64_t **lane_out, uint8_t **bm_out) {
    int dtype;
    bool hv;
    uint64_t n64;
    int rc = header_read(src, len, &dtype, &hv, &n64);
    if (rc) return rc;
    /* The reference fails the logical-length allocation (decoder.rs:105-106,
     * validity.rs:135-136) and reports CorruptPayload for absurd lengths. */
    if (n64 > ((uint64_t)1 << 36)) return OQ_CORRUPT;
    size_t logical_n = (size_t)n64;
    size_t pos = 16;
    uint8_t *bm = NULL;
    size_t n_total = logical_n;
    if (hv) {
        uint64_t vlen;
        rc = varint_read(src, len, &pos, &vlen);
        if (rc) return rc;
        if (vlen > (uint64_t)(len - pos)) return OQ_TRUNCATED;
        size_t raw_len = (size_t)((n64 + 7) / 8);
        if (n64 > UINT64_MAX - 7 || raw_len > MAX_BITMAP_BYTES) return OQ_CORRUPT;
        bm = (uint8_t *)malloc(raw_len ? raw_len : 1);
        rc = validity_decode(src + pos, (size_t)vlen, logical_n, bm);
        if (rc) {
            free(bm);
            return rc;
        }
        pos += (size_t)vlen;
        n_total = count_valid(bm, logical_n);
    }
    size_t fcap = 16, nf = 0, counted = 0;
    frame_t *frames = (frame_t *)malloc(sizeof(frame_t) * fcap);
    while (counted < n_total) {
        if (len - pos < 9) {
            rc = OQ_TRUNCATED;
            goto fail;
        }
        int mode = src[pos];
        if (!mode_known(mode)) {
            rc = OQ_UNKNOWN_MODE;
            goto fail;
        }
        size_t fn = rd_u32(src + pos + 1), plen = rd_u32(src + pos + 5);
        pos += 9;
        if (fn > 131072) {
            rc = OQ_CORRUPT;
            goto fail;
        }
        if (len - pos < plen) {
            rc = OQ_TRUNCATED;
            goto fail;
        }
        if (nf == fcap) {
            fcap *= 2;
            frames = (frame_t *)realloc(frames, sizeof(frame_t) * fcap);
        }
        frames[nf].mode = mode;
        frames[nf].n = fn;
        frames[nf].off = counted;
        frames[nf].payload = src + pos;
        frames[nf].plen = plen;
        nf++;
        pos += plen;
        counted += fn;
        if (counted > n_total) {
            rc = OQ_CORRUPT;
            goto fail;
        }
    }
    {
        uint64_t *vals = (uint64_t *)malloc(sizeof(uint64_t) * (n_total ? n_total : 1));
        int *rcs = (int *)calloc(nf ? nf : 1, sizeof(int));
        dec_job_t job = {frames, nf, dtype, src[6], vals, rcs, 0};
        if (threads > 1 && nf > 1) {
            pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
            for (int i = 0; i < threads; i++) pthread_create(&th[i], NULL, dec_worker, &job);
            for (int i = 0; i < threads; i++) pthread_join(th[i], NULL);
            free(th);
        } else {
            dec_worker(&job);
        }
        rc = OQ_OK;
        for (size_t k = 0; k < nf; k++)
            if (rcs[k]) {
                rc = rcs[k];
                break;
            }
        free(rcs);
        if (rc) {
            free(vals);
            goto fail;
        }
        uint64_t *lane = vals;
        if (bm) { /* validity.rs:130-146 */
            lane = (uint64_t *)calloc(logical_n ? logical_n : 1, 8);
            size_t j = 0;
            for (size_t i = 0; i < logical_n; i++)
                if (bm_is_set(bm, i)) lane[i] = vals[j++];
            free(vals);
        }
        free(frames);
        *dtype_out = dtype;
        *n_out = logical_n;
        *lane_out = lane;
        *bm_out = bm;
        return OQ_OK;
    }
fail:
    free(frames);
    free(bm);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Decimal container — src/decimal.rs:39-408                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t l[4];
} limb4_t;

/* decimal.rs:56-85 (assemble) */
static void decimal_assemble(int dtype, size_t logical_n, int8_t scale, uint8_t precision,
                             const uint8_t *vmin_le, size_t nlimbs, const uint8_t *validity,
                             uint64_t **limbs, size_t n_valid, int level, long block_size, int plog2,
                             int threads, buf_t *out) {
    bool hv = validity && count_valid(validity, logical_n) < logical_n;
    b_write(out, "FCR1", 4);
    b_push(out, 2);
    b_push(out, (uint8_t)(2 | (hv ? 1 : 0)));
    b_push(out, 0);
    b_push(out, (uint8_t)dtype);
    b_u64(out, logical_n);
    b_push(out, (uint8_t)scale);
    b_push(out, precision);
    b_push(out, (uint8_t)nlimbs);
    b_write(out, vmin_le, nlimbs * 8);
    if (hv) {
        buf_t vb = {0};
        validity_encode(validity, logical_n, &vb);
        b_varint(out, vb.len);
        b_write(out, vb.p, vb.len);
        b_free(&vb);
    }
    for (size_t k = 0; k < nlimbs; k++) {
        buf_t sub = {0};
        compress_lane_buf(limbs[k], n_valid, OQ_U64, n_valid, NULL, level, block_size, plog2, threads, &sub);
        b_varint(out, sub.len);
        b_write(out, sub.p, sub.len);
        b_free(&sub);
    }
}

static bool lt_signed4(const limb4_t *a, const limb4_t *b) { /* decimal.rs:254-269 */
    uint64_t sa = a->l[3] >> 63, sb = b->l[3] >> 63;
    if (sa != sb) return sa == 1;
    for (int i = 3; i >= 0; i--)
        if (a->l[i] != b->l[i]) return a->l[i] < b->l[i];
    return false;
}

/* decimal.rs:174-212 (128) and 339-377 (256): `nl` limbs per value. */
static void decimal_compress(int dtype, size_t n, const uint8_t *values, const uint8_t *validity, int8_t scale,
                             uint8_t precision, int level, long block_size, int plog2, int threads, buf_t *out) {
    size_t nl = dtype == OQ_DEC128 ? 2 : 4;
    bool has_nulls = validity && count_valid(validity, n) < n;
    size_t nv = 0;
    limb4_t *valid = (limb4_t *)malloc(sizeof(limb4_t) * (n ? n : 1));
    for (size_t i = 0; i < n; i++) {
        if (has_nulls && !bm_is_set(validity, i)) continue;
        limb4_t v;
        for (size_t k = 0; k < 4; k++) {
            if (k < nl)
                v.l[k] = rd_u64(values + i * nl * 8 + k * 8);
            else /* a 128-bit value sign-extends into the unused limbs */
                v.l[k] = (uint64_t)((int64_t)v.l[nl - 1] >> 63);
        }
        valid[nv++] = v;
    }
    limb4_t vmin;
    memset(&vmin, 0, sizeof vmin);
    if (nv) {
        vmin = valid[0];
        for (size_t i = 1; i < nv; i++)
            if (lt_signed4(&valid[i], &vmin)) vmin = valid[i];
    }
    uint64_t *limbs[4];
    for (size_t k = 0; k < nl; k++) limbs[k] = (uint64_t *)malloc(sizeof(uint64_t) * (nv ? nv : 1));
    for (size_t i = 0; i < nv; i++) { /* decimal.rs:281-293 sub_limbs */
        unsigned borrow = 0;
        for (size_t k = 0; k < nl; k++) {
            uint64_t a = valid[i].l[k], b = vmin.l[k];
            uint64_t d1 = a - b;
            unsigned b1 = a < b;
            uint64_t d2 = d1 - borrow;
            unsigned b2 = d1 < (uint64_t)borrow;
            limbs[k][i] = d2;
            borrow = b1 | b2;
        }
    }
    uint8_t vmin_le[32];
    for (size_t k = 0; k < nl; k++)
        for (int b = 0; b < 8; b++) vmin_le[k * 8 + b] = (uint8_t)(vmin.l[k] >> (8 * b));
    decimal_assemble(dtype, n, scale, precision, vmin_le, nl, validity, limbs, nv, level, block_size, plog2,
                     threads, out);
    for (size_t k = 0; k < nl; k++) free(limbs[k]);
    free(valid);
}

/* decimal.rs:100-168 (parse_shell) + 218-246 / 379-408 (recombine, scatter).
 * Writes n native values (16 or 32 B each). */
static int decimal_decompress(const uint8_t *src, size_t len, int expect, int threads, size_t *n_out,
                              uint8_t **values_out, uint8_t **bm_out, int8_t *scale, uint8_t *precision) {
    if (len < 19) return OQ_TRUNCATED;
    if (memcmp(src, "FCR1", 4) != 0) return OQ_BAD_MAGIC;
    if (src[4] != 2) return OQ_UNSUPPORTED_VERSION;
    if (!(src[5] & 2)) return OQ_CORRUPT;
    bool hv = src[5] & 1;
    if (src[7] > 7) return OQ_UNSUPPORTED_DTYPE;
    if (src[7] != expect) return OQ_DTYPE_MISMATCH;
    uint64_t n64 = rd_u64(src + 8);
    if (n64 > ((uint64_t)1 << 36)) return OQ_CORRUPT;
    size_t logical_n = (size_t)n64;
    *scale = (int8_t)src[16];
    *precision = src[17];
    size_t nl = src[18];
    if (nl == 0 || nl > 4) return OQ_CORRUPT;
    size_t vmin_off = 19, pos = 19 + nl * 8;
    if (pos > len) return OQ_TRUNCATED;
    uint8_t *bm = NULL;
    size_t n_valid = logical_n;
    if (hv) {
        uint64_t vlen;
        int rc = varint_read(src, len, &pos, &vlen);
        if (rc) return rc;
        if (vlen > (uint64_t)(len - pos)) return OQ_TRUNCATED;
        size_t raw_len = (size_t)((n64 + 7) / 8);
        if (n64 > UINT64_MAX - 7 || raw_len > MAX_BITMAP_BYTES) return OQ_CORRUPT;
        bm = (uint8_t *)malloc(raw_len ? raw_len : 1);
        rc = validity_decode(src + pos, (size_t)vlen, logical_n, bm);
        if (rc) {
            free(bm);
            return rc;
        }
        pos += (size_t)vlen;
        n_valid = count_valid(bm, logical_n);
    }
    uint64_t *limbs[4] = {0};
    int rc = OQ_OK;
    size_t got_limbs = 0;
    for (size_t k = 0; k < nl; k++) {
        uint64_t sl;
        rc = varint_read(src, len, &pos, &sl);
        if (rc) break;
        if (sl > (uint64_t)(len - pos)) {
            rc = OQ_TRUNCATED;
            break;
        }
        int dt;
        size_t ln;
        uint8_t *sbm = NULL;
        rc = decompress_lane(src + pos, (size_t)sl, threads, &dt, &ln, &limbs[k], &sbm);
        free(sbm);
        if (rc) break;
        got_limbs++;
        pos += (size_t)sl;
        if (ln != n_valid) {
            rc = OQ_CORRUPT;
            break;
        }
    }
    size_t want = expect == OQ_DEC128 ? 2 : 4;
    if (!rc && nl != want) rc = OQ_CORRUPT;
    if (rc) {
        for (size_t k = 0; k < got_limbs; k++) free(limbs[k]);
        free(bm);
        return rc;
    }
    size_t w = want * 8;
    uint8_t *vals = (uint8_t *)calloc(logical_n ? logical_n : 1, w);
    uint64_t vmin[4];
    for (size_t k = 0; k < want; k++) vmin[k] = rd_u64(src + vmin_off + 8 * k);
    size_t j = 0;
    for (size_t i = 0; i < logical_n; i++) {
        if (bm && !bm_is_set(bm, i)) continue;
        unsigned __int128 carry = 0;
        for (size_t k = 0; k < want; k++) {
            unsigned __int128 cur = (unsigned __int128)vmin[k] + limbs[k][j] + carry;
            uint64_t lw = (uint64_t)cur;
            carry = cur >> 64;
            for (int b = 0; b < 8; b++) vals[i * w + k * 8 + b] = (uint8_t)(lw >> (8 * b));
        }
        j++;
    }
    for (size_t k = 0; k < nl; k++) free(limbs[k]);
    *n_out = logical_n;
    *values_out = vals;
    *bm_out = bm;
    return OQ_OK;
}

/* ------------------------------------------------------------------------ */
/* Column API — src/lib.rs:389-508                                           */
/* ------------------------------------------------------------------------ */

static size_t native_width(int dtype) {
    switch (dtype) {
        case OQ_I32: case OQ_U32: case OQ_F32: return 4;
        case OQ_DEC128: return 16;
        case OQ_DEC256: return 32;
        default: return 8;
    }
}

/* lib.rs:389-403 (to_lane) */
static uint64_t *to_lane(int dtype, size_t n, const void *values) {
    uint64_t *lane = (uint64_t *)malloc(sizeof(uint64_t) * (n ? n : 1));
    const uint8_t *v = (const uint8_t *)values;
    for (size_t i = 0; i < n; i++) {
        switch (dtype) {
            case OQ_I32: lane[i] = (uint64_t)(int64_t)(int32_t)rd_u32(v + 4 * i); break;
            case OQ_U32: lane[i] = rd_u32(v + 4 * i); break;
            case OQ_F32: lane[i] = f32bits_to_f64bits(rd_u32(v + 4 * i)); break;
            default: lane[i] = rd_u64(v + 8 * i); break;
        }
    }
    return lane;
}

static int compress_column_impl(int dtype, size_t n, const void *values, const uint8_t *validity, int8_t scale,
                                uint8_t precision, int level, long block_size, int plog2, int threads,
                                uint8_t **out, size_t *out_len) {
    if (level < 0 || (level & ~(OQ_SELECT_SAMPLE | 0xFF)) || (level & 0xFF) > 2 || dtype < 0 || dtype > 7)
        return OQ_BAD_ARG;
    buf_t b = {0};
    if (dtype == OQ_DEC128 || dtype == OQ_DEC256) { /* lib.rs:431-443 */
        decimal_compress(dtype, n, (const uint8_t *)values, validity, scale, precision, level, block_size, plog2,
                         threads, &b);
    } else {
        bool has_nulls = validity && count_valid(validity, n) < n; /* lib.rs:446 */
        uint64_t *lane = to_lane(dtype, n, values);
        if (!has_nulls) {
            compress_lane_buf(lane, n, dtype, n, NULL, level, block_size, plog2, threads, &b);
        } else { /* validity.rs:122-127 compact */
            size_t j = 0;
            for (size_t i = 0; i < n; i++)
                if (bm_is_set(validity, i)) lane[j++] = lane[i];
            compress_lane_buf(lane, j, dtype, n, validity, level, block_size, plog2, threads, &b);
        }
        free(lane);
    }
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return OQ_OK;
}

int oq_compress_column(int dtype, size_t n, const void *values, const uint8_t *validity, int8_t scale,
                       uint8_t precision, int level, long block_size, int plog2, uint8_t **out, size_t *out_len) {
    return compress_column_impl(dtype, n, values, validity, scale, precision, level, block_size, plog2, 1, out,
                                out_len);
}

int oq_compress_column_mt(int dtype, size_t n, const void *values, const uint8_t *validity, int8_t scale,
                          uint8_t precision, int level, long block_size, int threads, uint8_t **out,
                          size_t *out_len) {
    return compress_column_impl(dtype, n, values, validity, scale, precision, level, block_size, 16, threads, out,
                                out_len);
}

int oq_compress_lane(const uint64_t *vals, size_t n_valid, int dtype, size_t logical_n, const uint8_t *validity,
                     int level, long block_size, int plog2, uint8_t **out, size_t *out_len) {
    if (level < 0 || (level & ~(OQ_SELECT_SAMPLE | 0xFF)) || (level & 0xFF) > 2) return OQ_BAD_ARG;
    buf_t b = {0};
    compress_lane_buf(vals, n_valid, dtype, logical_n, validity, level, block_size, plog2, 1, &b);
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return OQ_OK;
}

int oq_stream_info(const uint8_t *src, size_t len, int *dtype, uint64_t *n, int *hv, int8_t *scale,
                   uint8_t *precision) {
    if (len > 5 && (src[5] & 2)) {
        if (len < 19) return OQ_TRUNCATED;
        if (src[7] > 7) return OQ_UNSUPPORTED_DTYPE;
        *dtype = src[7];
        *n = rd_u64(src + 8);
        *hv = src[5] & 1;
        *scale = (int8_t)src[16];
        *precision = src[17];
        return OQ_OK;
    }
    bool h;
    int rc = header_read(src, len, dtype, &h, n);
    if (rc) return rc;
    *hv = h;
    *scale = 0;
    *precision = 0;
    return OQ_OK;
}

/* lib.rs:462-508 */
static int decompress_column_impl(const uint8_t *src, size_t len, int threads, int *dtype, size_t *n,
                                  void **values, uint8_t **validity, int8_t *scale, uint8_t *precision) {
    *scale = 0;
    *precision = 0;
    if (len > 5 && (src[5] & 2)) { /* decimal.rs:39-41 */
        if (len < 8) return OQ_TRUNCATED;
        if (src[7] > 7) return OQ_UNSUPPORTED_DTYPE;
        int expect = src[7] == OQ_DEC256 ? OQ_DEC256 : OQ_DEC128;
        uint8_t *vals;
        int rc = decimal_decompress(src, len, expect, threads, n, &vals, validity, scale, precision);
        if (rc) return rc;
        *dtype = expect;
        *values = vals;
        return OQ_OK;
    }
    uint64_t *lane;
    uint8_t *bm;
    int dt;
    size_t ln;
    int rc = decompress_lane(src, len, threads, &dt, &ln, &lane, &bm);
    if (rc) return rc;
    if (dt == OQ_DEC128 || dt == OQ_DEC256) {
        free(lane);
        free(bm);
        return OQ_CORRUPT;
    }
    size_t w = native_width(dt);
    uint8_t *out = (uint8_t *)malloc((ln ? ln : 1) * w);
    for (size_t i = 0; i < ln; i++) {
        uint64_t x = lane[i];
        if (dt == OQ_I32 || dt == OQ_U32) {
            uint32_t t = (uint32_t)x;
            memcpy(out + 4 * i, &t, 4);
        } else if (dt == OQ_F32) {
            uint32_t t = f64bits_to_f32bits(x);
            memcpy(out + 4 * i, &t, 4);
        } else {
            memcpy(out + 8 * i, &x, 8);
        }
    }
    free(lane);
    *dtype = dt;
    *n = ln;
    *values = out;
    *validity = bm;
    return OQ_OK;
}

int oq_decompress_column(const uint8_t *src, size_t len, int *dtype, size_t *n, void **values, uint8_t **validity,
                         int8_t *scale, uint8_t *precision) {
    return decompress_column_impl(src, len, 1, dtype, n, values, validity, scale, precision);
}

int oq_decompress_column_mt(const uint8_t *src, size_t len, int threads, int *dtype, size_t *n, void **values,
                            uint8_t **validity, int8_t *scale, uint8_t *precision) {
    return decompress_column_impl(src, len, threads, dtype, n, values, validity, scale, precision);
}

void oq_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Test hooks                                                                */
/* ------------------------------------------------------------------------ */

int oq_rans_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    if (!rans_compress(data, n, &b)) {
        *out = NULL;
        *out_len = 0;
        return OQ_OK;
    }
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}

int oq_rans_decompress(const uint8_t *payload, size_t len, size_t max_len, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    int rc = rans_decompress(payload, len, max_len, &b);
    if (rc) {
        b_free(&b);
        return rc;
    }
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return OQ_OK;
}

int oq_encode_mode(int mode, const uint64_t *v, size_t n, int dtype, int level, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    bool ok = true, entropy = level >= 2;
    switch (mode) {
        case M_RAW: raw_encode(v, n, dtype, &b); break;
        case M_CONST: ok = const_encode(v, n, &b); break;
        case M_STRIDE: ok = stride_encode(v, n, &b); break;
        case M_XORZ: xorz_encode(v, n, &b); break;
        case M_FOR_BITPACK: for_encode(v, n, dtype_signed(dtype), &b); break;
        case M_DELTA_BITPACK: delta_encode(v, n, &b); break;
        case M_FLOAT_MULT: ok = fm_encode(v, n, entropy, &b); break;
        case M_ALP: ok = alp_encode(v, n, &b); break;
        case M_ALP_RD: ok = alprd_encode(v, n, entropy, &b); break;
        case M_DICT: ok = dict_encode(v, n, entropy, &b); break;
        case M_RLE: ok = rle_encode(v, n, &b); break;
        case M_BYTE_TRANSPOSE: {
            if (n == 0) {
                ok = false;
                break;
            }
            uint8_t *tr = transpose_encode(v, n);
            code_residuals(tr, n * 8, &b);
            free(tr);
            break;
        }
        default: return OQ_UNSUPPORTED;
    }
    if (!ok) {
        b_free(&b);
        *out = NULL;
        *out_len = 0;
        return OQ_OK;
    }
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return OQ_OK;
}

/* `tag` ++ the bytes coded by the range coder (0), tANS (1) or rANS (2).
 * 0 when that coder makes no stream for these bytes. */
static int code_tagged(const uint8_t *r, size_t n, int tag, buf_t *b) {
    b_push(b, (uint8_t)tag);
    if (tag == TAG_RC) {
        rc_compress(r, n, b);
        return 1;
    }
    if (tag == TAG_TANS) return tans_compress(r, n, b);
    if (tag == TAG_RANS && n) {
        rans_compress(r, n, b);
        return 1;
    }
    return 0;
}

/* A High / Max linear-mode payload (linear.rs) with the residual bytes coded
 * by `tag` (TAG_RC, TAG_TANS or TAG_RANS, entropy/mod.rs:24-29); order 0 picks it as
 * the reference's encoder does (linear.rs:121-140).  *out = NULL when
 * DELTA_DP does not apply. */
int oq_linear_payload(int mode, const uint64_t *v, size_t n, int order, int tag, uint8_t **out, size_t *out_len) {
    buf_t r = {0}, b = {0};
    *out = NULL;
    *out_len = 0;
    if (order == 0) order = lin_select_order(v, n);
    if (mode == M_ORDERED_DELTA) {
        idelta2_encode(v, n, &r);
    } else if (mode == M_DELTA2) {
        delta2_encode(v, n, order, &r);
    } else if (mode == M_DELTA_DP) {
        if (!dp_encode(v, n, order, &r)) {
            b_free(&r);
            return OQ_OK;
        }
    } else {
        return OQ_UNSUPPORTED;
    }
    if (!code_tagged(r.p, r.len, tag, &b)) {
        b_free(&r);
        b_free(&b);
        return OQ_UNSUPPORTED;
    }
    b_free(&r);
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}

int oq_linear_select_order(const uint64_t *v, size_t n) { return lin_select_order(v, n); }

/* A PRED (0, LEB128 residuals), PRED_RC (29) or PRED2 (25) frame payload
 * (codecs/pred.rs) at predictor_log2 plog2; the residual bytes of 29 and 25
 * are coded by `tag` (TAG_RC, TAG_TANS or TAG_RANS). */
int oq_pred_payload(int mode, const uint64_t *v, size_t n, int plog2, int tag, uint8_t **out, size_t *out_len) {
    buf_t r = {0}, b = {0};
    *out = NULL;
    *out_len = 0;
    if (plog2 < 10 || plog2 > 16) return OQ_CORRUPT;
    if (mode == M_PRED2) dfcm_encode(v, n, plog2, &r);
    else if (mode == M_PRED || mode == M_PRED_RC) fcm_encode(v, n, plog2, &r);
    else return OQ_UNSUPPORTED;
    if (mode == M_PRED) {
        *out = r.p ? r.p : (uint8_t *)malloc(1);
        *out_len = r.len;
        return OQ_OK;
    }
    if (!code_tagged(r.p, r.len, tag, &b)) {
        b_free(&r);
        b_free(&b);
        return OQ_UNSUPPORTED;
    }
    b_free(&r);
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}

/* tans.rs compress_bytes / decompress_bytes (the coded bytes, no tag);
 * oq_tans_compress gives OQ_UNSUPPORTED where the reference returns None. */
int oq_tans_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    *out = NULL;
    *out_len = 0;
    if (!tans_compress(data, n, &b)) {
        b_free(&b);
        return OQ_UNSUPPORTED;
    }
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}
int oq_tans_decompress(const uint8_t *src, size_t len, size_t max_len, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    int rc = tans_decompress(src, len, max_len, &b);
    if (rc) {
        b_free(&b);
        return rc;
    }
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return OQ_OK;
}

uint32_t oq_crc32c_u64(uint32_t crc, uint64_t v) { return crc32c_u64(crc, v); }

/* lz.rs: the LZ stream of `data` (lz_compress) and its inverse */
int oq_lz_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    lz_compress(data, n, &b);
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}
int oq_lz_decompress(const uint8_t *stream, size_t len, size_t expected, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    int rc = lz_decompress(stream, len, expected, &b);
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return rc;
}

int oq_rc_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    rc_compress(data, n, &b);
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}

int oq_rc_decompress(const uint8_t *payload, size_t len, size_t max_len, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    int rc = rc_decompress(payload, len, max_len, &b);
    *out = b.p ? b.p : (uint8_t *)malloc(1);
    *out_len = b.len;
    return rc;
}

int oq_decode_mode(int mode, const uint8_t *payload, size_t plen, size_t n, int dtype, uint64_t *out) {
    return decode_frame(mode, payload, plen, n, dtype, 16, out);
}

int oq_validity_encode(const uint8_t *bitmap, size_t n, uint8_t **out, size_t *out_len) {
    buf_t b = {0};
    validity_encode(bitmap, n, &b);
    *out = b.p;
    *out_len = b.len;
    return OQ_OK;
}

int oq_validity_decode(const uint8_t *blob, size_t len, size_t n, uint8_t *bitmap_out) {
    return validity_decode(blob, len, n, bitmap_out);
}

void oq_mode_win_counts(uint64_t out[64]) {
    for (int i = 0; i < 64; i++) out[i] = atomic_load(&g_wins[i]);
}
void oq_reset_mode_win_counts(void) {
    for (int i = 0; i < 64; i++) atomic_store(&g_wins[i], 0);
}
