/*
 * quoin — C ABI of the B200-native quoin library (libquoin_b200.so).
 *
 * Lossless compressor for typed numeric columns.  The first part of this header
 * is the reference C ABI, symbol for symbol, with the same codes, ownership
 * and buffer rules; the second part adds the B200-specific entry points
 * (typed column with a level/block-size knob, device-resident buffers and CUDA
 * streams, a reusable decode index and the per-mode win counters).
 *
 * Each declaration cites the reference interface it replaces
 * (capi/include/quoin.h, capi/src/lib.rs, capi/src/typed.rs, src/lib.rs).
 *
 * Differences from the reference, by design:
 *  - compression runs on the GPU (sm_100a); the competition pool covers
 *    Level::Fastest and Level::Fast, whose streams are byte-identical to the
 *    reference encoder's.  The reference symbols compress at Level::Fast
 *    (the reference default, Level::Max, needs Pco, Lz, the range coder and
 *    the FCM/DFCM predictors, which are outside this library);
 *  - decompression accepts every stream whose block modes and entropy tags
 *    are in the covered pool; blocks outside it return QUOIN_ERR_CORRUPT
 *    (reference symbols) or QUOIN_ERR_UNSUPPORTED (extended symbols).
 *  - a "context" owns a CUDA stream and device arenas instead of a thread pool.
 *
 * Threading: every call is synchronous with respect to the caller's buffers.
 * Not async-signal-safe; do not fork after first use.
 */
#ifndef QUOIN_H
#define QUOIN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return / error codes (capi/include/quoin.h:28-33). */
#define QUOIN_OK                    0
#define QUOIN_ERR_NULL             (-1) /* a required pointer argument was NULL  */
#define QUOIN_ERR_BUFFER_TOO_SMALL (-2) /* dst too small; needed size in out_*   */
#define QUOIN_ERR_CORRUPT          (-3) /* malformed / truncated input stream    */
#define QUOIN_ERR_PANIC            (-4) /* internal error caught at the boundary  */

/* Extended codes, returned only by the quoin_b200_* symbols (the error kinds
 * of src/error.rs:5-25, plus device and scope errors). */
#define QUOIN_ERR_BAD_MAGIC           (-10)
#define QUOIN_ERR_UNSUPPORTED_VERSION (-11)
#define QUOIN_ERR_TRUNCATED           (-12)
#define QUOIN_ERR_UNKNOWN_MODE        (-13)
#define QUOIN_ERR_CORRUPT_PAYLOAD     (-14)
#define QUOIN_ERR_LENGTH_MISMATCH     (-15)
#define QUOIN_ERR_UNSUPPORTED_DTYPE   (-16)
#define QUOIN_ERR_DTYPE_MISMATCH      (-17)
#define QUOIN_ERR_UNSUPPORTED         (-18) /* mode / entropy tag / level outside the pool */
#define QUOIN_ERR_CUDA                (-19) /* a CUDA call failed (no device, OOM, ...)   */
#define QUOIN_ERR_BAD_ARG             (-20)
#define QUOIN_ERR_NOALLOC_LIMIT       (-21) /* stream outside quoin_b200_decompress_device_noalloc's limits */
#define QUOIN_ERR_UNSUPPORTED_ARROW_TYPE (-22) /* Error::UnsupportedArrowType (src/error.rs) */

/* ---------------- reference ABI (capi/include/quoin.h:35-142) ---------------- */

/* capi/include/quoin.h:36 — NUL-terminated version string (static). */
const char *quoin_version(void);

/* capi/include/quoin.h:39, capi/src/lib.rs:39-41 — 9n + 1024. */
size_t quoin_compress_bound(size_t n_values);

/* capi/include/quoin.h:47-48, capi/src/lib.rs:117-125 (Level::Fast on the GPU). */
int quoin_compress(const double *src, size_t n_values,
                   uint8_t *dst, size_t dst_cap, size_t *out_len);

/* capi/include/quoin.h:56-57, capi/src/lib.rs:132-140. */
int quoin_decompress(const uint8_t *src, size_t src_len,
                     double *dst, size_t dst_cap_values, size_t *out_values);

/* capi/include/quoin.h:64, capi/src/lib.rs:145-158. */
ptrdiff_t quoin_decompressed_value_count(const uint8_t *src, size_t src_len);

/* capi/include/quoin.h:67-81, capi/src/lib.rs:161-224.  A context owns a CUDA
 * stream and device/pinned arenas; `threads` selects nothing on the GPU and is
 * kept for source compatibility.  NULL ctx = the lazily created default. */
typedef struct QuoinCtx QuoinCtx;
QuoinCtx *quoin_ctx_create(size_t threads);
void quoin_ctx_free(QuoinCtx *ctx);
int quoin_compress_ctx(const QuoinCtx *ctx, const double *src, size_t n_values,
                       uint8_t *dst, size_t dst_cap, size_t *out_len);
int quoin_decompress_ctx(const QuoinCtx *ctx, const uint8_t *src, size_t src_len,
                         double *dst, size_t dst_cap_values, size_t *out_values);

/* Arrow-native dtype tags (capi/include/quoin.h:96-114). */
typedef enum {
    QUOIN_DTYPE_BOOL = 0,
    QUOIN_DTYPE_I8   = 1,
    QUOIN_DTYPE_I16  = 2,
    QUOIN_DTYPE_I32  = 3,
    QUOIN_DTYPE_I64  = 4,
    QUOIN_DTYPE_U8   = 5,
    QUOIN_DTYPE_U16  = 6,
    QUOIN_DTYPE_U32  = 7,
    QUOIN_DTYPE_U64  = 8,
    QUOIN_DTYPE_F32  = 9,
    QUOIN_DTYPE_F64  = 10,
    QUOIN_DTYPE_DECIMAL32  = 11,
    QUOIN_DTYPE_DECIMAL64  = 12,
    QUOIN_DTYPE_DECIMAL128 = 13,
    QUOIN_DTYPE_DECIMAL256 = 14
} QuoinDType;

/* capi/include/quoin.h:118, capi/src/typed.rs:50-61. */
size_t quoin_dtype_width(int32_t dtype);
/* capi/include/quoin.h:121, capi/src/typed.rs:65-69 — n*(max(w,8)+1)+1024. */
size_t quoin_typed_compress_bound(int32_t dtype, size_t n);
/* capi/include/quoin.h:126-127, capi/src/typed.rs:125-174 — bytes, 0 on failure. */
size_t quoin_typed_compress(int32_t dtype, size_t n, const void *values,
                            const uint8_t *validity, uint8_t *dst, size_t dst_cap);
/* capi/include/quoin.h:133-135, capi/src/typed.rs:183-227. */
size_t quoin_typed_compress_decimal(int32_t dtype, size_t n, const void *values,
                                    const uint8_t *validity, int8_t scale,
                                    uint8_t precision, uint8_t *dst, size_t dst_cap);
/* capi/include/quoin.h:141-142, capi/src/typed.rs:311-338. */
int quoin_typed_decompress(int32_t dtype, size_t n, const uint8_t *src,
                           size_t src_len, void *values_out, uint8_t *validity_out);

/* ---------------- B200 extensions ---------------- */

/* Speed/ratio levels (src/lib.rs:93-119).  The GPU competition covers
 * FASTEST and FAST; higher levels return QUOIN_ERR_UNSUPPORTED.
 * QUOIN_B200_LEVEL_BALANCED_INPOOL runs Balanced's competition (lambda 2,
 * rANS-coded FLOAT_MULT / ALP-RD / DICT parts, BYTE_TRANSPOSE; encoder.rs:
 * 275-469) without its Lz and Pco candidates: its streams are reference
 * streams (any quoin decoder reads them) and equal Level::Balanced's bytes
 * wherever neither Lz nor Pco would win a block. */
#define QUOIN_LEVEL_FASTEST  0
#define QUOIN_LEVEL_FAST     1
#define QUOIN_LEVEL_BALANCED 2
#define QUOIN_LEVEL_HIGH     3
#define QUOIN_LEVEL_MAX      4
#define QUOIN_B200_LEVEL_BALANCED_INPOOL 258

/* Stream dtype wire ids (src/dtype.rs:68-78). */
#define QUOIN_WIRE_F64 0
#define QUOIN_WIRE_I64 1
#define QUOIN_WIRE_U64 2
#define QUOIN_WIRE_I32 3
#define QUOIN_WIRE_U32 4
#define QUOIN_WIRE_F32 5
#define QUOIN_WIRE_DECIMAL128 6
#define QUOIN_WIRE_DECIMAL256 7

/* Mode selection (src/lib.rs:65-73): FULL sizes every candidate on the whole
 * block; SAMPLE sizes them on a stratified sample of the block and encodes
 * only the winner in full (src/encoder.rs:470-620), at FASTEST and FAST. */
#define QUOIN_B200_SELECTION_FULL   0
#define QUOIN_B200_SELECTION_SAMPLE 1

/* Encoder configuration (src/lib.rs:195-245): predictor_log2 (clamped 10..16,
 * recorded in the header), level, block_size (0 = adaptive; else clamped to
 * [1, 131072]), selection (QUOIN_B200_SELECTION_*). */
typedef struct {
    int32_t level;
    int64_t block_size;
    int32_t predictor_log2;
    int32_t selection;
} QuoinConfig;

/* Replaces compress_column(ColumnRef, Option<&[u8]>, Config) (src/lib.rs:429-455)
 * for host buffers: `values` holds n values of the wire dtype's native width
 * (8 B f64/i64/u64, 4 B i32/u32/f32, 16 B Decimal128, 32 B Decimal256,
 * little-endian), `validity` an Arrow bitmap or NULL; scale/precision are used
 * by the decimal dtypes.  Writes the stream to dst and its length to *out_len
 * (the needed size with QUOIN_ERR_BUFFER_TOO_SMALL). */
int quoin_b200_compress_column(QuoinCtx *ctx, int32_t wire_dtype, size_t n, const void *values,
                               const uint8_t *validity, int8_t scale, uint8_t precision,
                               const QuoinConfig *cfg, uint8_t *dst, size_t dst_cap,
                               size_t *out_len);

/* Header of a stream (src/format.rs:65-94, src/decimal.rs:100-168): wire
 * dtype, logical n, validity flag, decimal scale/precision (0 otherwise). */
int quoin_b200_stream_info(const uint8_t *src, size_t src_len, int32_t *wire_dtype,
                           uint64_t *n, int32_t *has_validity, int8_t *scale,
                           uint8_t *precision);

/* Host-only validation of a whole stream: header, validity blob and frame
 * table walk (src/decoder.rs:43-94, src/decimal.rs:100-168), no device work.
 * Returns the wire dtype, logical n and validity flag, or the error kind. */
int quoin_b200_parse(const uint8_t *src, size_t src_len, int32_t *wire_dtype, uint64_t *n,
                     int32_t *has_validity);

/* Replaces decompress_column(&[u8]) (src/lib.rs:462-508) for host buffers:
 * writes n native values to values_out (null slots 0) and, when the stream has
 * a validity bitmap and validity_out is non-NULL, ceil(n/8) bitmap bytes. */
int quoin_b200_decompress_column(QuoinCtx *ctx, const uint8_t *src, size_t src_len,
                                 void *values_out, uint8_t *validity_out);

/* Device-resident variants: every pointer is device memory on the context's
 * device; `stream` is a cudaStream_t (NULL = the context's own stream).  The
 * call returns after the work on `stream` has completed. */
int quoin_b200_compress_column_device(QuoinCtx *ctx, int32_t wire_dtype, size_t n,
                                      const void *d_values, const uint8_t *d_validity,
                                      int8_t scale, uint8_t precision, const QuoinConfig *cfg,
                                      uint8_t *d_dst, size_t dst_cap, size_t *out_len,
                                      void *stream);

/* Parts of a compress, for a column split across devices (one process per
 * GPU; blocks are independent, reference src/encoder.rs:7-8).
 *
 * quoin_b200_probe_windows_device: the block plan's probe (src/encoder.rs:154-178,
 * probe_block_features src/encoder.rs:705-750) over the column's valid values:
 * grow_out[w] = 1 where plan_blocks grows a block that starts at 32,768-value
 * window w to 131,072 values, else 0; *n_windows = ceil(valid values / 32,768)
 * (QUOIN_ERR_BUFFER_TOO_SMALL when it exceeds grow_cap).  grow_out is HOST
 * memory.  A part of a column that starts at a window boundary of the valid
 * values probes that part's windows, so the plan of the whole column is the
 * plan_blocks scan over the concatenated bytes.
 *
 * quoin_b200_stream_prefix_device: the bytes before a stream's first frame
 * (src/encoder.rs:184-214): the 16-byte header for n values and, when the
 * bitmap has a null, the validity blob.  The stream of the whole column is
 * this prefix followed by the frames of its blocks in order, and the frames of
 * a run of whole blocks are the stream of those blocks' valid values (no
 * validity) without its 16-byte header.
 *
 * Decimal dtypes return QUOIN_ERR_UNSUPPORTED (their container holds limb
 * streams). */
int quoin_b200_probe_windows_device(QuoinCtx *ctx, int32_t wire_dtype, size_t n,
                                    const void *d_values, const uint8_t *d_validity,
                                    uint8_t *grow_out, size_t grow_cap, uint64_t *n_windows,
                                    void *stream);
int quoin_b200_stream_prefix_device(QuoinCtx *ctx, int32_t wire_dtype, size_t n,
                                    const uint8_t *d_validity, const QuoinConfig *cfg,
                                    uint8_t *d_dst, size_t dst_cap, size_t *out_len, void *stream);

/* A decode index: the header, validity and frame table of a stream, parsed
 * and validated once on the host (src/decoder.rs:43-94) and kept resident on
 * the device so the stream can be decoded again without re-walking it. */
typedef struct QuoinDecodeIndex QuoinDecodeIndex;
int quoin_b200_index_create(QuoinCtx *ctx, const uint8_t *src, size_t src_len,
                            QuoinDecodeIndex **out);
void quoin_b200_index_free(QuoinDecodeIndex *idx);
/* n and wire dtype of an indexed stream. */
int quoin_b200_index_info(const QuoinDecodeIndex *idx, int32_t *wire_dtype, uint64_t *n,
                          int32_t *has_validity);
/* Decimal scale and precision (0 for other dtypes) and the number of valid values. */
int quoin_b200_index_decimal(const QuoinDecodeIndex *idx, int8_t *scale, uint8_t *precision,
                             uint64_t *n_valid);
/* Decode the device copy d_src of the indexed stream into d_values_out (and
 * d_validity_out when non-NULL and the stream has a bitmap). */
int quoin_b200_decompress_indexed_device(QuoinCtx *ctx, const QuoinDecodeIndex *idx,
                                         const uint8_t *d_src, void *d_values_out,
                                         uint8_t *d_validity_out, void *stream);

/* Decode a device-resident stream d_src[0 .. src_len) into device memory
 * (replaces decompress_column, src/lib.rs:462-508, for a caller whose stream
 * is already on the GPU; the reader is src/decoder.rs:43-118 and
 * src/format.rs:65-94).  The header, the validity blob and the frame table
 * are read on the device, so the host never copies the stream (streams the
 * device reader does not take, such as damaged ones or an RLE validity blob,
 * are read from a host copy by the host reader, with the same error codes).
 * d_values_out receives n values of the stream's native width (nulls as 0),
 * values_cap_bytes being its size; d_validity_out (optional) receives the
 * ceil(n/8)-byte bitmap when the stream has one.  *wire_out and *n_out get
 * the stream's dtype and value count (also with QUOIN_ERR_BUFFER_TOO_SMALL).
 * `stream` is a cudaStream_t (NULL = the context's stream); the call returns
 * after the decode completed. */
int quoin_b200_decompress_column_device(QuoinCtx *ctx, const uint8_t *d_src, size_t src_len,
                                        void *d_values_out, size_t values_cap_bytes,
                                        uint8_t *d_validity_out, int32_t *wire_out, uint64_t *n_out,
                                        void *stream);

/* Decodes of device-resident streams since the process started: out[0] read
 * by the device reader, out[1] read by the host reader, out[2] why the last
 * one was (1 a header the device reader does not take, 2 a frame table it
 * could not resolve, 3 more frame candidates than its tables held); for the
 * last stream the device reader read, out[3] its frame-header candidates and
 * out[4] how many times it laid out its tables (2 after a capacity retry);
 * out[5] the columns quoin_b200_decompress_queue_device decoded in batches. */
void quoin_b200_reader_stats(uint64_t out[6]);

/* No counterpart in the reference.  Allocation-free device decode for callers
 * that cannot let the library allocate device memory (an engine that owns all
 * device memory through its own pool, or a process that must keep a fixed
 * footprint): decodes the device-resident stream d_src[0 .. src_len) into
 * d_values_out (8-byte aligned, room for out_cap_values values) using only a
 * fixed scratch arena compiled into the library (2,433,088 bytes per device),
 * and writes the value count to *n_out.  Limits: at most 262,144 values and
 * 256 frames, dtype f64/i64/u64, no validity bitmap; other streams, and frames
 * with an entropy-coded part (levels above Fast), are rejected with
 * QUOIN_ERR_NOALLOC_LIMIT.  When n exceeds out_cap_values the call returns
 * QUOIN_ERR_BUFFER_TOO_SMALL with the needed count in *n_out; on every other
 * nonzero return *n_out is 0 and the contents of d_values_out are
 * unspecified (frames before a corrupt one may have been written).  The
 * caller zeroes nothing: each call resets the arena.
 * Calls on one device share the arena, so calls that overlap in time race and
 * must be serialised by the caller.  The first call on each device looks the
 * arena up (and may load the module); make it before any stream capture.
 * `stream` is a cudaStream_t (NULL = the default stream); the call returns
 * after the work on it has completed. */
int quoin_b200_decompress_device_noalloc(const uint8_t *d_src, size_t src_len, void *d_values_out,
                                         size_t out_cap_values, uint64_t *n_out, void *stream);

/* Per-mode win counts of the GPU competition since the last reset, indexed by
 * mode id (src/lib.rs:540-547, src/diag.rs). */
void quoin_b200_mode_win_counts(uint64_t out[64]);
void quoin_b200_reset_mode_win_counts(void);

/* Number of GPU kernels this library has launched in the calling process. */
uint64_t quoin_b200_kernel_launches(void);

/* Per-kernel-class device time, measured with CUDA events recorded on the
 * launching stream around each launch: 0 competition, 1 emission, 2 block
 * decode, 3 final scatter/narrow, 4 lowering, 5 probe+plan, 6 validity,
 * 7 other, 8 the device stream reader.  enable(1) resets and starts recording; read() returns the number
 * of classes written (ms totals and call counts). */
void quoin_b200_timing_enable(int on);
int quoin_b200_timing_read(double *ms_out, uint64_t *calls_out, int n);

/* ---------------- batches of columns ---------------- */

/* No reference counterpart (the batched configuration: many columns of uneven
 * length and mixed dtype).  A batch holds `workers` contexts (1..64) on the
 * current device; a batch call hands its columns, longest first, to one host
 * worker per context, so short columns' launch and synchronisation latencies
 * overlap.  Every column's stream is byte-identical to the single-column
 * call's.  One batch call at a time per batch. */
typedef struct QuoinBatch QuoinBatch;
QuoinBatch *quoin_b200_batch_create(int workers);
void quoin_b200_batch_free(QuoinBatch *batch);

/* One column of quoin_b200_compress_batch_device: the arguments of
 * quoin_b200_compress_column_device (device pointers) and its results. */
typedef struct {
    int32_t wire_dtype;
    int8_t scale;
    uint8_t precision;
    size_t n;
    const void *d_values;
    const uint8_t *d_validity;
    uint8_t *d_dst;
    size_t dst_cap;
    size_t out_len; /* out: stream length (the needed size on BUFFER_TOO_SMALL) */
    int32_t status; /* out: the column's return code */
} QuoinB200CompressJob;

/* One column of quoin_b200_decompress_batch_device: the arguments of
 * quoin_b200_decompress_indexed_device and its return code. */
typedef struct {
    const QuoinDecodeIndex *idx;
    const uint8_t *d_src;
    void *d_values_out;
    uint8_t *d_validity_out;
    int32_t status; /* out */
} QuoinB200DecompressJob;

/* Every job is attempted; returns QUOIN_OK, or the status of the first failing
 * job in job order (each job's own status is in its record). */
int quoin_b200_compress_batch_device(QuoinBatch *batch, QuoinB200CompressJob *jobs, size_t njobs,
                                     const QuoinConfig *cfg);
int quoin_b200_decompress_batch_device(QuoinBatch *batch, QuoinB200DecompressJob *jobs, size_t njobs);

/* One column of quoin_b200_decompress_queue_device: a device-resident stream
 * and the device buffers for its values (values_cap_bytes) and bitmap
 * (optional), as for quoin_b200_decompress_column_device. */
typedef struct {
    const uint8_t *d_src;
    size_t src_len;
    void *d_values_out;
    size_t values_cap_bytes;
    uint8_t *d_validity_out;
    int32_t wire;   /* out: the stream's dtype */
    uint64_t n;     /* out: its value count */
    int32_t status; /* out: the column's return code */
} QuoinB200DeviceDecodeJob;

/* No reference counterpart (the batched configuration).  Decodes every job's
 * device-resident stream with one launch per kernel class for the whole
 * batch (src/decoder.rs:43-190 per column): the headers, validity bitmaps,
 * frame chains and warp-item tables of all columns are read by one set of
 * launches over a device-side table of (column, chunk) and (column,
 * candidate) work, and one launch of each block-decoder kernel decodes every
 * column's frames, each frame writing through its column's output.  Columns
 * this path leaves out (entropy-coded frames, damaged streams, all-null
 * columns) are decoded one by one as by
 * quoin_b200_decompress_column_device, so every column gets its own status.
 * Returns QUOIN_OK or the first failing job's status in job order. */
int quoin_b200_decompress_queue_device(QuoinCtx *ctx, QuoinB200DeviceDecodeJob *jobs, size_t njobs,
                                       void *stream);

/* ---------------- Request server ---------------- */

/* No counterpart in the reference.  A server runs compress and decompress
 * requests on device-resident buffers for many callers: requests are queued
 * in arrival order and admitted when the device memory they hold fits the
 * server's budget beside the running ones and the device's free memory
 * (cudaMemGetInfo, 1 GiB kept free) at that moment (a request above the
 * budget on its own is refused with QUOIN_ERR_OVER_BUDGET), then run on a
 * pool of contexts.  Each request's bytes are those of the single-column
 * call. */
#define QUOIN_ERR_OVER_BUDGET (-23) /* a request needs more device memory than the server's budget */
#define QUOIN_ERR_TIMEOUT     (-24) /* quoin_b200_server_wait: the request has not finished yet */
#define QUOIN_B200_OP_COMPRESS   0
#define QUOIN_B200_OP_DECOMPRESS 1

typedef struct QuoinServer QuoinServer;

typedef struct {
    int32_t op;                       /* QUOIN_B200_OP_COMPRESS or QUOIN_B200_OP_DECOMPRESS */
    /* compress: the arguments of quoin_b200_compress_column_device */
    int32_t wire_dtype;
    int8_t scale;
    uint8_t precision;
    size_t n;
    const void *d_values;
    const uint8_t *d_validity;
    uint8_t *d_dst;
    size_t dst_cap;
    /* decompress: the arguments of quoin_b200_decompress_indexed_device */
    const QuoinDecodeIndex *idx;
    const uint8_t *d_src;
    void *d_values_out;
    uint8_t *d_validity_out;
    /* device memory the request's own buffers hold while it waits and runs */
    uint64_t device_bytes;
    /* out */
    size_t out_len;                   /* compress: stream length */
    int32_t status;                   /* the call's return code */
    int32_t done;                     /* set when the request has finished */
    uint64_t t_submit_ns, t_start_ns, t_end_ns; /* steady clock, ns since the server started */
} QuoinB200Request;

/* workers: 1..64 contexts; budget_bytes: device memory the admitted requests may hold. */
QuoinServer *quoin_b200_server_create(int workers, uint64_t budget_bytes, const QuoinConfig *cfg);
/* Queues `req` (which must stay valid until it is done) and returns at once. */
int quoin_b200_server_submit(QuoinServer *server, QuoinB200Request *req);
/* Waits up to timeout_ms (negative: without limit) for `req`; returns its
 * status, or QUOIN_ERR_TIMEOUT. */
int quoin_b200_server_wait(QuoinServer *server, QuoinB200Request *req, int timeout_ms);
/* Peak device bytes held by admitted requests (budget accounting, including the
 * server's estimate of each request's working memory). */
uint64_t quoin_b200_server_peak_bytes(QuoinServer *server);
/* Finishes the queued requests and frees the server. */
void quoin_b200_server_free(QuoinServer *server);

/* ---------------- Arrow C Data Interface ---------------- */

/* The standard Arrow C Data Interface structs (declared here unless the
 * caller's Arrow headers already did). */
#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE
#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4
struct ArrowSchema {
    const char *format;
    const char *name;
    const char *metadata;
    int64_t flags;
    int64_t n_children;
    struct ArrowSchema **children;
    struct ArrowSchema *dictionary;
    void (*release)(struct ArrowSchema *);
    void *private_data;
};
struct ArrowArray {
    int64_t length;
    int64_t null_count;
    int64_t offset;
    int64_t n_buffers;
    int64_t n_children;
    const void **buffers;
    struct ArrowArray **children;
    struct ArrowArray *dictionary;
    void (*release)(struct ArrowArray *);
    void *private_data;
};
#endif
typedef struct ArrowSchema ArrowSchema;
typedef struct ArrowArray ArrowArray;

/* Replaces compress_array(&dyn Array, Config) (src/arrow.rs:61-123): compresses
 * a primitive Arrow array (Float64 "g", Float32 "f", Int64 "l", UInt64 "L",
 * Int32 "i", UInt32 "I", Decimal128 "d:P,S", Decimal256 "d:P,S,256") with its
 * validity; the array's offset is honoured (a sliced bitmap is re-packed).
 * Other types: QUOIN_ERR_UNSUPPORTED_ARROW_TYPE.  The array is only read. */
int quoin_b200_compress_arrow(QuoinCtx *ctx, const struct ArrowSchema *schema,
                              const struct ArrowArray *array, const QuoinConfig *cfg, uint8_t *dst,
                              size_t dst_cap, size_t *out_len);

/* Replaces decompress_array(&[u8]) (src/arrow.rs:129-160): fills *schema_out and
 * *array_out with a new array of the stream's type (null slots hold 0); the
 * caller owns both and frees them through their release callbacks. */
int quoin_b200_decompress_arrow(QuoinCtx *ctx, const uint8_t *src, size_t src_len,
                                struct ArrowSchema *schema_out, struct ArrowArray *array_out);

/* ---------------- Arrow C Device Data Interface ---------------- */

/* The standard device-array struct (declared here unless the caller's Arrow
 * headers already did). */
#ifndef ARROW_C_DEVICE_DATA_INTERFACE
#define ARROW_C_DEVICE_DATA_INTERFACE
typedef int32_t ArrowDeviceType;
#define ARROW_DEVICE_CPU 1
#define ARROW_DEVICE_CUDA 2
#define ARROW_DEVICE_CUDA_HOST 3
#define ARROW_DEVICE_CUDA_MANAGED 13
struct ArrowDeviceArray {
    struct ArrowArray array;
    int64_t device_id;
    ArrowDeviceType device_type;
    void *sync_event; /* for CUDA: a cudaEvent_t* to wait on before reading, or NULL */
    int64_t reserved[3];
};
#endif
typedef struct ArrowDeviceArray ArrowDeviceArray;

/* Zero-copy compress of a device-resident Arrow array (device_type CUDA or
 * CUDA_MANAGED, on the context's device): the values buffer (and validity
 * bitmap) are read in place on `stream` (a cudaStream_t; NULL = the context's
 * stream) after its sync_event; a bitmap whose offset is not a multiple of 8
 * is re-packed on the device.  d_dst / out_len as in
 * quoin_b200_compress_column_device.  Types and errors as
 * quoin_b200_compress_arrow; QUOIN_ERR_BAD_ARG for a host device_type. */
int quoin_b200_compress_arrow_device(QuoinCtx *ctx, const struct ArrowSchema *schema,
                                     const struct ArrowDeviceArray *array, const QuoinConfig *cfg,
                                     uint8_t *d_dst, size_t dst_cap, size_t *out_len, void *stream);

/* Decodes the indexed stream (device copy d_src) into a new device-resident
 * Arrow array (device_type CUDA, the context's device, sync_event NULL: the
 * data is ready when the call returns); the caller owns *schema_out and
 * *array_out and frees them (and the device buffers) through their release
 * callbacks. */
int quoin_b200_decompress_arrow_device(QuoinCtx *ctx, const QuoinDecodeIndex *idx, const uint8_t *d_src,
                                       struct ArrowSchema *schema_out, struct ArrowDeviceArray *array_out,
                                       void *stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* QUOIN_H */
