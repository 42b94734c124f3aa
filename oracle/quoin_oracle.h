/*
 * quoin oracle — a plain-C CPU restatement of the reference compressor's
 * in-path algorithm (okhsunrog/quoin, Rust).  TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker: the tests, the package's smoke() check and
 * bench.py's CPU-baseline leg call it to produce expected streams/values and
 * to time the reference's CPU algorithm.  The product (quoin_b200) never
 * links, loads or calls it.
 *
 * Parity status: the reference cannot be built here (no Rust toolchain and
 * unvendored crates), and its tests hold no golden byte streams.  The oracle
 * is pinned only by the reference's own known-answer behaviour (header bytes,
 * ratio floors at Level::Fastest, round trips, codec size bounds); byte-level
 * stream parity is otherwise "parity unpinned" — it follows the cited source
 * line by line.
 *
 * Levels: 0 = Fastest, 1 = Fast (both run entirely inside the path and are the
 * byte-identical levels), 2 = Balanced restricted to the in-path pool (the Lz
 * and Pco candidates are skipped), used to produce rANS-tagged streams for
 * decoder tests.
 */
#ifndef QUOIN_ORACLE_H
#define QUOIN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error kinds, mirroring src/error.rs:5-25 (plus UNSUPPORTED for modes and
 * entropy tags outside the in-path pool). */
enum {
    OQ_OK = 0,
    OQ_BAD_MAGIC = 1,
    OQ_UNSUPPORTED_VERSION = 2,
    OQ_TRUNCATED = 3,
    OQ_UNKNOWN_MODE = 4,
    OQ_CORRUPT = 5,
    OQ_LENGTH_MISMATCH = 6,
    OQ_UNSUPPORTED_DTYPE = 7,
    OQ_DTYPE_MISMATCH = 8,
    OQ_UNSUPPORTED = 9,
    OQ_BAD_ARG = 10
};

/* Stream dtype wire ids (src/dtype.rs:68-78). */
enum { OQ_F64 = 0, OQ_I64 = 1, OQ_U64 = 2, OQ_I32 = 3, OQ_U32 = 4, OQ_F32 = 5,
       OQ_DEC128 = 6, OQ_DEC256 = 7 };

/* Added to a level: Selection::Sample instead of Selection::Full (reference
 * src/lib.rs:65-73, src/encoder.rs:470-620). */
#define OQ_SELECT_SAMPLE 0x100

/* Compress a typed column.  `values` holds n native values (8 B for
 * f64/i64/u64, 4 B for i32/u32/f32, 16 B for dec128, 32 B for dec256).
 * `validity` is an Arrow bitmap of ceil(n/8) bytes or NULL.  `block_size` <= 0
 * selects adaptive blocks.  The result is malloc'd into *out (free with
 * oq_free).  Returns an OQ_* code. */
int oq_compress_column(int dtype, size_t n, const void *values, const uint8_t *validity,
                       int8_t scale, uint8_t precision, int level, long block_size,
                       int predictor_log2, uint8_t **out, size_t *out_len);

/* Parse a stream header: dtype, logical n, has_validity, decimal scale and
 * precision (0 for non-decimal streams). */
int oq_stream_info(const uint8_t *src, size_t len, int *dtype, uint64_t *n,
                   int *has_validity, int8_t *scale, uint8_t *precision);

/* Decompress into malloc'd buffers.  *values holds n native values; *validity
 * is a ceil(n/8) bitmap or NULL when the stream has none. */
int oq_decompress_column(const uint8_t *src, size_t len, int *dtype, size_t *n,
                         void **values, uint8_t **validity, int8_t *scale,
                         uint8_t *precision);

void oq_free(void *p);

/* Lane-level entry points (u64 lane, already compacted). */
int oq_compress_lane(const uint64_t *vals, size_t n_valid, int dtype, size_t logical_n,
                     const uint8_t *validity, int level, long block_size, int predictor_log2,
                     uint8_t **out, size_t *out_len);

/* Kernel-level entry points used by unit tests. */
void oq_pack32(const uint32_t *values1024, uint32_t width, uint32_t *out);
void oq_unpack32(const uint32_t *packed, uint32_t width, uint32_t *out1024);
void oq_pack64(const uint64_t *values1024, uint32_t width, uint64_t *out);
void oq_unpack64(const uint64_t *packed, uint32_t width, uint64_t *out1024);
/* rANS over bytes (src/entropy/rans.rs).  compress returns 0 on empty input. */
int oq_rans_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len);
int oq_rans_decompress(const uint8_t *payload, size_t len, size_t max_len, uint8_t **out,
                       size_t *out_len);
/* Per-mode encode of one block (payload only, no frame header); returns 0 and
 * sets *out to NULL when the mode does not apply.  mode = wire id. */
int oq_encode_mode(int mode, const uint64_t *vals, size_t n, int dtype, int level,
                   uint8_t **out, size_t *out_len);
/* Decode one frame payload of `mode` into n lane words. */
int oq_decode_mode(int mode, const uint8_t *payload, size_t plen, size_t n, int dtype,
                   uint64_t *out);
/* plan_blocks' probe for every 32,768-value window of a lane (encoder.rs:154-178). */
void oq_probe_windows(const uint64_t *lane, size_t n, uint8_t *flags);
/* Validity blob (src/validity.rs). */
int oq_validity_encode(const uint8_t *bitmap, size_t n, uint8_t **out, size_t *out_len);
int oq_validity_decode(const uint8_t *blob, size_t len, size_t n, uint8_t *bitmap_out);
/* Diagnostics: per-mode win counters (src/diag.rs). */
void oq_mode_win_counts(uint64_t out[64]);
void oq_reset_mode_win_counts(void);

/* Multi-threaded compress/decompress of a column (std thread pool over
 * plan_blocks ranges / frames, mirroring the reference's rayon split).
 * threads <= 1 runs serially.  Used for the CPU baseline timing. */
int oq_compress_column_mt(int dtype, size_t n, const void *values, const uint8_t *validity,
                          int8_t scale, uint8_t precision, int level, long block_size,
                          int threads, uint8_t **out, size_t *out_len);
int oq_decompress_column_mt(const uint8_t *src, size_t len, int threads, int *dtype,
                            size_t *n, void **values, uint8_t **validity, int8_t *scale,
                            uint8_t *precision);

/* High / Max linear modes (src/codecs/linear.rs): a frame payload of mode 7
 * (ORDERED_DELTA), 20 (DELTA2) or 45 (DELTA_DP) with the residual bytes coded
 * by tag 0 (range coder), 1 (tANS) or 2 (rANS); order 0 = the reference's choice.
 * *out = NULL when DELTA_DP does not apply to the values. */
int oq_linear_payload(int mode, const uint64_t *vals, size_t n, int order, int tag,
                      uint8_t **out, size_t *out_len);
/* FCM / DFCM predictor payloads (src/codecs/pred.rs): mode 0 (PRED), 29
 * (PRED_RC) or 25 (PRED2) at predictor_log2 plog2 (10..16); tag as above for
 * 29 and 25.  And the predictor hash (src/hash.rs). */
int oq_pred_payload(int mode, const uint64_t *vals, size_t n, int plog2, int tag,
                    uint8_t **out, size_t *out_len);
uint32_t oq_crc32c_u64(uint32_t crc, uint64_t v);
/* tANS (src/entropy/tans.rs, entropy tag 1): the coded bytes without the tag. */
int oq_tans_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len);
int oq_tans_decompress(const uint8_t *src, size_t len, size_t max_len, uint8_t **out,
                       size_t *out_len);
/* The LZ stream of src/codecs/lz.rs (lz_compress / lz_decompress). */
int oq_lz_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len);
int oq_lz_decompress(const uint8_t *stream, size_t len, size_t expected, uint8_t **out,
                     size_t *out_len);
/* linear.rs:121-140: the extrapolation order the reference's encoder picks. */
int oq_linear_select_order(const uint64_t *vals, size_t n);
/* The range coder (src/entropy/rc.rs): varint(len) ++ coded bytes. */
int oq_rc_compress(const uint8_t *data, size_t n, uint8_t **out, size_t *out_len);
int oq_rc_decompress(const uint8_t *payload, size_t len, size_t max_len, uint8_t **out,
                     size_t *out_len);

#ifdef __cplusplus
}
#endif
#endif
