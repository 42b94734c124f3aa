// Allocation-free decode entry point: quoin_b200_decompress_device_noalloc.
//
// Callers that manage every byte of device memory themselves (a column store
// with its own pool, a process that must not grow its footprint mid-query)
// cannot use the context-based device API, whose arenas grow with cudaMalloc.
// This entry point decodes a device-resident stream into a caller-provided
// device buffer using only a fixed scratch arena that lives in this file as a
// static __device__ array, so the call itself allocates nothing.
//
// Limits (the arena is sized for them, larger streams are rejected with
// QUOIN_ERR_NOALLOC_LIMIT before any decode work): at most
// kNoAllocMaxValues values and kNoAllocMaxFrames frames; 8-byte dtypes
// (f64 / i64 / u64) without a validity bitmap.  Frames with an entropy-coded
// part (levels above Fast) need a decode area the arena does not hold: the
// decode reports them with QUOIN_ERR_NOALLOC_LIMIT.
//
// Nothing in the arena has to start at zero: every call's first kernel resets
// the status words and the frame table before the decode kernels read them.
// All calls on one device share the arena, so calls that overlap in time (two
// host threads, or two streams whose work overlaps) race; callers serialise
// them.  The first call on each device looks up the arena's address
// (cudaGetSymbolAddress, which may load the module); make that first call
// before any stream capture.
#include <mutex>

#include "qb_common.cuh"
#include "qb_kernels.h"
#include "qb_layout.h"
#include "../../include/quoin.h"

namespace qb {
namespace {

constexpr uint32_t kNoAllocMaxFrames = 256;
constexpr uint64_t kNoAllocMaxValues = 262144;
constexpr uint64_t kNoAllocAuxBytes = 1280;  // per frame, >= the decoder's per-frame record
constexpr uint64_t kMaxLogicalValuesD = 1ull << 36;
constexpr int kMaxDevices = 64;

struct NoAllocStatus {
  unsigned long long err;  // decode error word: ~0 = none, else (frame << 8) | kind
  uint32_t kind;           // header / frame-table error kind (0 = ok, 0xFF = over the limits)
  uint32_t nf;
  uint64_t n;
  uint64_t pad[5];
};

struct NoAllocArena {
  NoAllocStatus st;
  FrameDesc frames[kNoAllocMaxFrames];
  uint8_t aux[kNoAllocMaxFrames * kNoAllocAuxBytes];
  uint64_t dict[kNoAllocMaxValues];  // decode scratch (large dictionaries, RLE run ends, ALP-RD), one slot per value
};
// The arena's footprint on every device that loads the library (quoted in
// include/quoin.h): 64 + 256 x 32 + 256 x 1,280 + 262,144 x 8 bytes.
static_assert(sizeof(NoAllocArena) == 2433088, "documented arena size");

static __device__ __align__(256) NoAllocArena g_noalloc_arena;

constexpr uint32_t kLimit = 0xFF;

__device__ inline bool mode_known_d(uint32_t id) {  // reference mode.rs:60-84
  switch (id) {
    case 0: case 1: case 2: case 3: case 4: case 5: case 7: case 9: case 11: case 17:
    case 19: case 20: case 25: case 29: case 45: case 50: case 51: case 52: case 53: case 54:
      return true;
    default: return false;
  }
}

// One thread: header + frame table walk with the host parser's checks and
// error kinds (reference format.rs:65-94, decoder.rs:43-94), then the table
// padded with empty frames so the decode kernels can run over the full arena.
__global__ void k_noalloc_parse(const uint8_t* __restrict__ s, uint64_t len, uint64_t cap_values,
                                NoAllocArena* __restrict__ A) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t kind = E_OK, nf = 0;
  uint64_t n = 0;
  A->st.err = ~0ull;
  do {
    if (len < 16) { kind = E_TRUNCATED; break; }
    if (s[0] != 'F' || s[1] != 'C' || s[2] != 'R' || s[3] != '1') { kind = E_BAD_MAGIC; break; }
    if (s[5] & 2) { kind = kLimit; break; }  // decimal container
    if (s[4] != 2) { kind = E_UNSUPPORTED_VERSION; break; }
    if (s[5] & ~1u) { kind = E_CORRUPT; break; }
    if (s[6] < 10 || s[6] > 16) { kind = E_CORRUPT; break; }
    if (s[7] > 7) { kind = E_UNSUPPORTED_DTYPE; break; }
    n = ld_u64(s + 8);
    if (n > kMaxLogicalValuesD) { kind = E_CORRUPT; break; }
    if ((s[5] & 1) || s[7] > DT_U64 || n > kNoAllocMaxValues) { kind = kLimit; break; }
    uint64_t pos = 16, counted = 0;
    while (counted < n) {
      if (len - pos < 9) { kind = E_TRUNCATED; break; }
      uint32_t mode = s[pos];
      if (!mode_known_d(mode)) { kind = E_UNKNOWN_MODE; break; }
      uint64_t fn = ld_u32(s + pos + 1), plen = ld_u32(s + pos + 5);
      pos += 9;
      if (fn > (uint64_t)kMaxBlock) { kind = E_CORRUPT; break; }
      if (len - pos < plen) { kind = E_TRUNCATED; break; }
      if (nf == kNoAllocMaxFrames) { kind = kLimit; break; }
      FrameDesc f;
      f.payload_off = pos;
      f.value_off = counted;
      f.n = (uint32_t)fn;
      f.plen = (uint32_t)plen;
      f.mode = mode;
      f.aux = 0;
      A->frames[nf++] = f;
      pos += plen;
      counted += fn;
      if (counted > n) { kind = E_CORRUPT; break; }
    }
  } while (false);
  if (kind == E_OK && n > cap_values) kind = kLimit + 1;  // caller's buffer too small
  if (kind != E_OK) nf = 0;
  for (uint32_t i = nf; i < kNoAllocMaxFrames; i++) {
    FrameDesc f;
    f.payload_off = 0;
    f.value_off = 0;
    f.n = 0;
    f.plen = 0;
    f.mode = M_RAW;
    f.aux = 0;
    A->frames[i] = f;
  }
  A->st.kind = kind;
  A->st.nf = nf;
  A->st.n = n;
}

std::mutex g_setup_mu;
NoAllocArena* g_arena_ptr[kMaxDevices] = {};

int kind_code(uint32_t kind) {
  switch (kind) {
    case E_BAD_MAGIC: return QUOIN_ERR_BAD_MAGIC;
    case E_UNSUPPORTED_VERSION: return QUOIN_ERR_UNSUPPORTED_VERSION;
    case E_TRUNCATED: return QUOIN_ERR_TRUNCATED;
    case E_UNKNOWN_MODE: return QUOIN_ERR_UNKNOWN_MODE;
    case E_CORRUPT: return QUOIN_ERR_CORRUPT_PAYLOAD;
    case E_LENGTH_MISMATCH: return QUOIN_ERR_LENGTH_MISMATCH;
    case E_UNSUPPORTED_DTYPE: return QUOIN_ERR_UNSUPPORTED_DTYPE;
    case E_DTYPE_MISMATCH: return QUOIN_ERR_DTYPE_MISMATCH;
    case kLimit:
    case E_NO_ENTROPY_AREA: return QUOIN_ERR_NOALLOC_LIMIT;
    case kLimit + 1: return QUOIN_ERR_BUFFER_TOO_SMALL;
    default: return QUOIN_ERR_UNSUPPORTED;
  }
}

// Set-up, once per device, with that device current.
int arena_for_current_device(NoAllocArena** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return QUOIN_ERR_CUDA;
  std::lock_guard<std::mutex> l(g_setup_mu);
  if (!g_arena_ptr[dev]) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_arena);
    if (rc != cudaSuccess || !p) {
      cudaGetLastError();
      return QUOIN_ERR_CUDA;
    }
    if (decode_aux_bytes((int)kNoAllocMaxFrames) > sizeof(((NoAllocArena*)nullptr)->aux)) return QUOIN_ERR_PANIC;
    g_arena_ptr[dev] = static_cast<NoAllocArena*>(p);
  }
  *out = g_arena_ptr[dev];
  return QUOIN_OK;
}

}  // namespace
}  // namespace qb

extern "C" int quoin_b200_decompress_device_noalloc(const uint8_t* d_src, size_t src_len, void* d_values_out,
                                                    size_t out_cap_values, uint64_t* n_out, void* stream) {
  using namespace qb;
  try {
    if (!d_src || !d_values_out || !n_out) return QUOIN_ERR_NULL;
    if (((uintptr_t)d_values_out & 7) != 0) return QUOIN_ERR_BAD_ARG;
    *n_out = 0;
    NoAllocArena* A = nullptr;
    int rc = arena_for_current_device(&A);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_noalloc_parse<<<1, 32, 0, st>>>(d_src, src_len, out_cap_values, A);
    count_launches(1);
    DecodeOut O{d_values_out, DT_U64, nullptr, nullptr, nullptr, 0, 0};
    launch_decode_frames(d_src, A->frames, (int)kNoAllocMaxFrames, DT_U64, O, A->dict, A->aux, &A->st.err, st);
    NoAllocStatus hs;
    if (cudaMemcpyAsync(&hs, &A->st, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      return QUOIN_ERR_CUDA;
    }
    if (cudaGetLastError() != cudaSuccess) return QUOIN_ERR_CUDA;
    if (hs.kind == kLimit + 1) *n_out = hs.n;  // the count the buffer needs
    if (hs.kind) return kind_code(hs.kind);
    if (hs.err != ~0ull) return kind_code((uint32_t)(hs.err & 0xFF));
    *n_out = hs.n;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}
