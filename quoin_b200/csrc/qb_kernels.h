// Host-side launchers of the quoin B200 kernels (declared here, defined in the
// .cu files).  All take an explicit CUDA stream and only plain device pointers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "qb_layout.h"

struct QuoinCtx;

namespace qb {

// ---- decoder (qb_decode.cu) ----
// Payload bytes of one XORZ warp item (the readers cut XORZ frames into
// items of this many bytes; other modes into items of 512 values).
constexpr uint32_t kXorzItemBytes = 2048;
// The entropy area of a listed frame of n values (128-byte aligned pieces):
// the mode's own layout (24 bytes per value + 1,152), the range coder's
// 256 x 256 model (128 KB), the FCM / DFCM table of PRED, PRED_RC and PRED2
// (8 << predictor_log2 bytes), and the LZ cascade's scratch for an inner LZ
// stream of up to twice the largest residual bound (16n + 1,024) + 64.
__host__ __device__ inline uint64_t ent_rc_off(uint64_t n) { return (24 * n + 1152 + 127) & ~127ull; }
__host__ __device__ inline bool ent_has_table(uint32_t mode) { return mode == 0 || mode == 25 || mode == 29; }
__host__ __device__ inline uint64_t ent_table_off(uint64_t n) { return ent_rc_off(n) + 131072; }
__host__ __device__ inline uint64_t ent_lz_off(uint64_t n, uint32_t mode, uint32_t plog2) {
  return ent_table_off(n) + (ent_has_table(mode) ? (8ull << plog2) : 0);
}
__host__ __device__ inline uint64_t ent_lz_cap(uint64_t n) { return 32 * n + 2112; }
__host__ __device__ inline uint64_t ent_area_bytes(uint64_t n, uint32_t mode, uint32_t plog2) {
  return ent_lz_off(n, mode, plog2) + ((ent_lz_cap(n) + 127) & ~127ull);
}

// Walk (validation + sub-block offsets) and decode of nf frames.  `aux` is
// device scratch of decode_aux_bytes(nf) bytes.
uint64_t decode_aux_bytes(int nf);
// Where decoded values go: the lane (out = u64 per lane value, bm32 null,
// dtype DT_U64) or the typed column (narrowed to dtype's native width and,
// with bm32, scattered through the validity words with nulls as 0; wrank =
// exclusive popcount prefix per 32-bit word, sel from launch_select_table).
struct DecodeOut {
  void* out;
  int dtype;
  const uint32_t* bm32;
  const uint64_t* wrank;
  const uint64_t* sel;
  uint64_t n;       // logical values (positions)
  uint64_t nvalid;  // lane values
  uint32_t plog2 = 16;  // the stream header's predictor_log2 (FCM / DFCM table size)
};
void launch_decode_frames(const uint8_t* stream, const FrameDesc* frames, int nf, int dtype, const DecodeOut& out,
                          uint64_t* scratch, void* aux, unsigned long long* err, cudaStream_t st);
// A batch of columns decoded by one launch per kernel class: frame f belongs
// to column frame_col[f], whose output, lane dtype and decode scratch replace
// the launch's own (payload offsets are then absolute device addresses, with
// a null stream base).
struct BatchCol {
  DecodeOut O;
  int dtype, pad;
  uint64_t* scratch;
};
struct BatchView {
  const uint32_t* frame_col;
  const BatchCol* cols;
};
// Warp-item decode of one lane (every item covers at most 512 values or 512
// XORZ payload bytes).  The host builds the tables from the frame table:
// pre_items / main_items name (frame, item index within the frame);
// frame_pre[f] = (first prepass item of frame f, count); list = frames decoded
// whole by one CTA (DICT, ALP-RD with exceptions, modes outside the items).
// `pre` holds npre records of prepass_rec_bytes().
struct ItemRef {
  uint32_t frame, local;
};
struct ItemPlan {
  const ItemRef* pre_items;
  uint32_t npre;
  const ItemRef* main_items;
  uint32_t nmain;
  const uint2* frame_pre;
  const uint32_t* list;
  uint32_t nlist;
  bool need_scan;
  uint8_t* ent;  // entropy areas of the listed frames (FrameDesc::aux), or null
};
uint64_t prepass_rec_bytes();
void launch_decode_items(const uint8_t* stream, const FrameDesc* frames, int nf, int dtype, const DecodeOut& out,
                         const ItemPlan& plan, void* pre, uint64_t* scratch, void* aux, unsigned long long* err,
                         cudaStream_t st, const BatchView* batch = nullptr);
// ---- device stream reader (qb_dparse.cu) ----
// One lane stream of a column: the stream itself, or a decimal limb's.
struct DpLane {
  uint64_t base, len;   // the lane stream's bytes within the buffer
  uint64_t fstart;      // offset of its first frame header
  uint64_t logical_n;   // the lane header's value count
  uint32_t dtype, plog2, has_validity, pad;
};
// The parsed header.  kind != 0: the device reader does not take this
// stream (an error, or a form the host reader decodes), the host parses it.
struct DpHead {
  uint32_t kind, wire, decimal, has_validity, nl, precision;
  int32_t scale, pad;
  uint64_t n;
  uint64_t vblob_off, vblob_len;  // the validity blob's bytes after its tag
  uint32_t vtag, pad2;            // 0 RAW (ceil(n/8) bitmap bytes), 1 RLE (varint runs)
  uint64_t vmin[4];
  DpLane lanes[4];
};
// A frame-header candidate (pos = header offset; plen < 2^24).
struct DpCand {
  uint64_t pos;
  uint32_t n, plen_mode;  // plen << 8 | mode
};
// A candidate's successor candidate (or ~0); after the chain is resolved, the
// j-th chain frame: its candidate index (in succ) and warp items (flags: 1
// listed, 2 needs the prepass scan, 4 uses the decode scratch).
struct DpNode {
  uint32_t succ, nmain, npre, flags;
  uint64_t ent;  // entropy area bytes when listed with a coded part
};
// The reader's result for one lane (status != 0: the host parses the stream;
// ncand tells the host how many candidates the tables must hold).
struct DpLaneOut {
  uint32_t status, nframes, nmain, npre, nlist, need_scan, any_dict, pad;
  uint64_t ncand, ent_bytes;
};
// Where k_dp_layout and k_dp_expand write a lane's decode tables (capacity = the candidate
// capacity; main_off one entry more).
struct DpTables {
  FrameDesc* frames;
  uint2* frame_pre;
  uint64_t* main_off;
  uint32_t* list;
  ItemRef* main_items;
  ItemRef* pre_items;
};
constexpr uint64_t kDpChainSmem = 200 * 1024;  // successor tables in shared memory up to 25,598 candidates
void launch_dp_head(const uint8_t* s, uint64_t len, DpHead* H, cudaStream_t st);
// The validity bitmap of an n-value stream as 32-bit words (ceil(n/32) + 1
// written, the last zero) and each word's popcount in cnt: from a RAW blob,
// or from an RLE blob (validity.rs:92-119; `ends` holds vblob_len entries).
// An RLE blob the sequential reader would reject sets H->kind, so the host
// reader takes the stream.
void launch_dp_bitmap(const uint8_t* s, const DpHead* H, uint64_t n, uint8_t* bm, uint64_t* cnt, cudaStream_t st);
void launch_dp_bitmap_rle(const uint8_t* s, DpHead* H, uint64_t n, uint64_t* ends, uint64_t* nruns, uint8_t* bm,
                          uint64_t* cnt, cudaStream_t st);
// Candidate chunks of a lane whose frames span `lane_frames_bytes` bytes (cnt
// needs dp_chunks() + 1 entries, slots dp_slot_bytes(); *d_ncand gets the
// count, at most cap written to cand).
uint64_t dp_chunks(uint64_t lane_frames_bytes);
uint64_t dp_slot_bytes(uint64_t lane_frames_bytes);
void launch_dp_candidates(const uint8_t* s, uint64_t buf_len, const DpHead* H, int lane, uint64_t lane_frames_bytes,
                          uint64_t* cnt, DpCand* slots, uint64_t* tile_tmp, uint64_t* d_ncand, DpCand* cand,
                          uint64_t cap, cudaStream_t st);
// Chain resolution + item tables of lane `lane` (nodes: cap entries; gJ: 8 *
// cap bytes of global scratch (successor tables that exceed shared memory,
// then the chain's candidate list); gmarks: cap bytes; d_ctl: two words).
void launch_dp_chain(const uint8_t* s, const DpHead* H, int lane, const uint64_t* d_nvalid, const DpCand* cand,
                     const uint64_t* d_ncand, uint64_t cap, DpNode* nodes, uint32_t* gJ, uint8_t* gmarks,
                     uint64_t* d_ctl, const DpTables& T, DpLaneOut* out, cudaStream_t st);

// ---- batches of device streams (qb_dparse.cu) ----
// One column of a batch read by one launch per kernel class: its stream and
// header facts (host-filled from the parsed headers), and where its bitmap,
// ranks, select table, candidate chunks and decode scratch sit in the
// batch's arrays.
struct DpBLane {
  const uint8_t* s;
  uint64_t buf_len;
  DpLane L;               // the lane (base 0: the column's own stream)
  uint64_t vblob_off;     // the validity blob's bytes after its tag, when has_bm
  uint64_t vblob_len;
  uint32_t vtag, pad;     // 0 RAW, 1 RLE
  uint64_t rle_off;       // an RLE blob's run ends in the batch's run-end array
  uint64_t bm_n;          // the column's value count (its bitmap's bits)
  uint32_t has_bm;        // this lane reads the column's bitmap (a plain column's, or a decimal's first limb)
  uint32_t decimal;       // a limb lane of a decimal container
  int32_t vlane;          // the lane holding the column's bitmap and valid count (itself for a plain column)
  uint32_t pad2;
  uint64_t word0, nw;     // its bitmap words (nw, then one zero word)
  uint64_t sel0;          // its select table entries
  uint64_t chunk0;        // its first candidate chunk (the batch has one more entry: the total)
  uint8_t* valid_out;     // the caller's bitmap, or null
};
// Device-written per column.
struct DpBLaneOut {
  uint64_t nvalid, nmarked, fbase, main_base, pre_base, list_base, ent;
  uint32_t status, nframes, nmain, npre, nlist, need_scan, any_dict, pad;
};
struct DpBTotals {
  uint64_t nframes, nmain, npre, nlist;
  uint32_t need_scan, pad;
};
// The batch reader's arrays (device).  words = sum of (nw + 1); chunks =
// lanes[nlanes - 1].chunk0's total; cap = candidate capacity.
struct DpBatch {
  DpBLane* lanes;
  const uint64_t* chunk0;  // nlanes + 1 chunk offsets (a copy of lanes[].chunk0 plus the total)
  const uint64_t* word0;   // nlanes + 1 word offsets (a copy of lanes[].word0 plus the total)
  DpBLaneOut* out;
  DpBTotals* tot;
  int nlanes;
  uint32_t* bm32;        // words
  uint64_t* ranks;       // words + 1
  uint64_t* rbase;       // nlanes
  uint64_t* sel;         // select tables
  uint64_t* cnt;         // chunks + 1
  DpCand* slots;         // chunks * kDpSlots (dp_batch_slot_bytes)
  DpCand* cand;          // cap
  uint32_t* cand_lane;   // cap
  DpNode* nodes;         // cap
  uint32_t* gJ;          // 2 * cap
  uint8_t* gmarks;       // cap
  uint4* ftmp;           // cap (per chain frame: pre offset, pre count, main offset, main count)
  uint32_t* flist;       // cap (per chain frame: its index in the column's list, or ~0)
  uint64_t cap, words, chunks;
  FrameDesc* frames;     // cap
  uint32_t* frame_col;   // cap
  uint2* frame_pre;      // cap
  ItemRef* main_items;   // item capacity
  ItemRef* pre_items;    // item capacity
  uint32_t* list;        // cap
  uint64_t item_cap;
  uint64_t* rle_ends;         // the RLE columns' run ends (sum of their blob lengths)
  uint64_t* rle_nruns;        // nlanes
  const uint32_t* rle_cols;   // nrle lane indices
  int nrle;
};
uint64_t dp_batch_slot_bytes(uint64_t chunks);
// Headers of n streams (srcs[i], lens[i]) into H[i].
void launch_dp_batch_heads(const uint8_t* const* srcs, const uint64_t* lens, int n, DpHead* H, cudaStream_t st);
// Validity, candidates, chains and item tables of every column of the batch
// (tile_tmp holds scan_tile_count(max(words + 1, chunks + 1)) + 16 entries).
void launch_dp_batch_read(const DpBatch& B, uint64_t* tile_tmp, cudaStream_t st);

// sel[m] = position of the (512*m)-th valid value, m < ceil(nvalid / 512).
void launch_select_table(const uint8_t* bm, uint64_t n, const uint64_t* word_rank, uint64_t nvalid, uint64_t* sel,
                         cudaStream_t st);
void launch_word_popcount(const uint8_t* bm, uint64_t n, uint64_t* cnt, cudaStream_t st);
void launch_finalize(const uint64_t* lane, const uint8_t* bm, const uint64_t* word_rank, uint64_t n, int dtype,
                     void* out, cudaStream_t st);
void launch_decimal_combine(const uint64_t* limbs, uint64_t limb_stride, int nlimbs, const uint64_t* vmin,
                            const uint8_t* bm, const uint64_t* word_rank, uint64_t n, uint8_t* out, cudaStream_t st);

// ---- encoder (qb_encode.cu) ----
// Per-block scratch the competition may use: 32 bytes per lane value.
constexpr uint64_t kEncScratchPerValue = 32;

// Competition part 1: per-sub-block statistics (and, for adaptive blocks, the
// window grow flags and probe bitsets).  Sizes: sub_stats_items(n, bs) records
// of sub_stats_bytes(); FLOAT_MULT records of fm_stats_bytes() for float
// columns; smp16 holds n/16 + 1 values (float columns); grow one byte per
// 32768-value window and winbits kWinWords words per window: the 14-bit probe
// bucket bitsets at stride max(len/4096,1) ([0,512)) and stride 32
// ([512,1024)), then word 1024 = the number of distinct 17-bit dictionary
// hash buckets over the whole window (a lower bound of its cardinality).
constexpr uint64_t kWinWords = 1028;
uint64_t sub_stats_items(uint64_t n, uint64_t fixed_bs);
uint64_t sub_stats_bytes();
uint64_t fm_stats_bytes();
void launch_sub_stats(const uint64_t* lane, uint64_t n, uint64_t fixed_bs, int dtype, int level, void* ss, void* fms,
                      uint64_t* smp16, uint8_t* grow, uint32_t* winbits, cudaStream_t st);
void launch_plan(const uint8_t* grow, uint64_t n, uint64_t fixed_bs, FrameDesc* frames, uint32_t* nb,
                 cudaStream_t st);
// Competition part 2: one CTA per planned block; writes mode / plen / aux.
// With `ent` (max_blocks records of ent_rec_bytes()) the Balanced in-pool
// candidates run too (rANS-coded parts, BYTE_TRANSPOSE) and their choices
// are recorded there for the emission.  `sample`: Selection::Sample (levels
// Fastest and Fast; not with `ent`).
void launch_decide(const uint64_t* lane, FrameDesc* frames, const uint32_t* nb, uint32_t max_blocks, uint64_t fixed_bs,
                   int dtype, int level, const void* ss, const void* fms, const uint64_t* smp16,
                   const uint32_t* winbits, uint8_t* scratch, void* ent, bool sample, cudaStream_t st);
uint64_t ent_rec_bytes();
// `base` (device) holds the byte offset at which the first frame starts.
void launch_frame_offsets(FrameDesc* frames, const uint32_t* nb, uint32_t max_blocks, const uint64_t* base,
                          uint64_t* sizes_tmp, uint64_t* tile_tmp, uint64_t* total, cudaStream_t st);
// Emission: one CTA per frame; FoR / DELTA / FLOAT_MULT / XORZ layouts are read
// from the statistics records of launch_sub_stats.  Frames that would end past
// out_cap bytes are not written.
void launch_emit(const uint64_t* lane, const FrameDesc* frames, const uint32_t* nb, uint32_t max_blocks,
                 uint64_t fixed_bs, int dtype, const void* ss, const void* fms, uint8_t* scratch, uint8_t* out,
                 uint64_t out_cap, const void* ent, cudaStream_t st);

// ---- lowering / validity (qb_lower.cu) ----
// Lower n native values (dtype width) to the u64 lane, keeping only positions
// whose validity bit is set when `word_rank` is given (compaction).
void launch_lower(const void* values, int dtype, const uint8_t* bm, const uint64_t* word_rank, uint64_t n,
                  uint64_t* lane, cudaStream_t st);
// Decimal: compacted limbs of (v - vmin).  `vmin` is computed on device.
void launch_decimal_vmin(const uint8_t* values, int nlimbs, const uint8_t* bm, uint64_t n, uint64_t* vmin_tmp,
                         uint64_t* vmin, cudaStream_t st);
void launch_decimal_split(const uint8_t* values, int nlimbs, const uint8_t* bm, const uint64_t* word_rank,
                          uint64_t n, const uint64_t* vmin, uint64_t* limbs, uint64_t limb_stride, cudaStream_t st);
// Validity run-length blob (reference validity.rs:40-70): the blob is written
// to out (tag + payload) and its length to *blob_len.
void launch_validity_blob(const uint8_t* bm, uint64_t n, uint64_t* tmp, uint64_t* tile_tmp, uint8_t* out,
                          uint64_t* blob_len, cudaStream_t st);
uint64_t validity_tmp_words(uint64_t n);
// Adds the bitmap's bit-transition count to *count (zero it first).
void launch_bitmap_transitions(const uint8_t* bm, uint64_t n, unsigned long long* count, cudaStream_t st);
// Short columns: a bitmap of at most kSmallWords words ranked, counted and its
// transitions counted by one CTA (rank = exclusive word ranks, *total = the
// valid count, *trans = 0/1 transitions); frame offsets of at most
// kSmallWords blocks by one CTA.
constexpr uint32_t kSmallPer = 8, kSmallWords = 1024 * kSmallPer;
void launch_valid_small(const uint8_t* bm, uint64_t n, uint64_t* rank, uint64_t* total, unsigned long long* trans,
                        cudaStream_t st);
// The stream a call on context c runs on: `stream` when given, else the
// context's own (the default context when c is null).
cudaStream_t ctx_stream(struct ::QuoinCtx* c, void* stream);
// Bits [bit_off, bit_off + n) of src re-packed into dst from bit 0 (ceil(n/8) bytes, trailing bits clear).
void launch_bitmap_repack(const uint8_t* src, uint64_t bit_off, uint64_t n, uint8_t* dst, cudaStream_t st);
// Writes varint(len) + the RAW validity blob of an n-bit bitmap at dst and the
// stream offset after it (dst_off + its length) to *d_base.
void launch_put_validity_raw(uint8_t* dst, uint64_t dst_off, const uint8_t* bm, uint64_t n, uint64_t* d_base,
                             cudaStream_t st);
void launch_write_bytes(uint8_t* dst, const uint8_t* src_dev, uint64_t len, cudaStream_t st);

// Mode win counters (reference src/diag.rs).
unsigned long long* device_win_counters();

// Small writers used by the stream assembly.
struct Bytes16 {
  uint8_t b[16];
};
void launch_put_header(uint8_t* dst, Bytes16 hdr, uint64_t* d_base, cudaStream_t st);
// Writes varint(*blob_len) ++ blob at dst and sets *d_base = dst_off + varint + blob.
void launch_put_validity(uint8_t* dst, uint64_t dst_off, const uint8_t* blob, const uint64_t* blob_len,
                         uint64_t* d_base, cudaStream_t st);

// Exclusive prefix sum of n u64 (in may alias out); grand total to *grand.
void launch_scan_sum(const uint64_t* in, uint64_t* out, uint64_t n, uint64_t* tile_tmp, uint64_t* grand,
                     cudaStream_t st);
inline uint64_t scan_tile_count(uint64_t n) {
  uint64_t t = (n + 2047) / 2048;  // kScanTile
  return t ? t : 1;
}

// Number of kernels launched by this library (all launchers add to it).
void count_launches(uint64_t k);
uint64_t launches_total();

}  // namespace qb
