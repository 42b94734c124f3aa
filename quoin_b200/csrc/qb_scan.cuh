// Device-wide exclusive scans over u64 (three passes: per-tile totals, a
// single-CTA scan of the tile totals, per-tile scan with the tile offset).
// Op is ScanSum (prefix sums: validity ranks, frame and varint offsets) or
// ScanMax (last-seen position scans for the validity run lengths).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qb {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;  // items per thread
constexpr int kScanTile = kScanThreads * kScanItems;

struct ScanSum {
  __device__ static uint64_t id() { return 0; }
  __device__ static uint64_t op(uint64_t a, uint64_t b) { return a + b; }
};
struct ScanMax {
  __device__ static uint64_t id() { return 0; }
  __device__ static uint64_t op(uint64_t a, uint64_t b) { return a > b ? a : b; }
};

template <class Op>
__device__ inline uint64_t block_excl_scan(uint64_t v, uint64_t* s_warp, uint64_t* total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint64_t inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint64_t u = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc = Op::op(u, inc);
  }
  uint64_t exc = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) exc = Op::id();
  if (lane == 31) s_warp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    uint64_t w = lane < nw ? s_warp[lane] : Op::id();
    uint64_t wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      uint64_t u = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi = Op::op(u, wi);
    }
    uint64_t we = __shfl_up_sync(0xffffffffu, wi, 1);
    if (lane == 0) we = Op::id();
    if (lane < nw) s_warp[lane] = we;  // exclusive warp offsets
    if (lane == nw - 1) s_warp[32] = wi;
  }
  __syncthreads();
  uint64_t r = Op::op(s_warp[wid], exc);
  if (total) *total = s_warp[32];
  __syncthreads();
  return r;
}

template <class Op>
__global__ void k_scan_tile_sums(const uint64_t* __restrict__ in, size_t n, uint64_t* __restrict__ sums) {
  __shared__ uint64_t s_warp[33];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint64_t acc = Op::id();
#pragma unroll
  for (int k = 0; k < kScanItems; k++)
    if (base + k < n) acc = Op::op(acc, in[base + k]);
  uint64_t tot;
  block_excl_scan<Op>(acc, s_warp, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Single CTA: exclusive scan of the tile sums in place; writes the grand total.
template <class Op>
__global__ void k_scan_sums(uint64_t* __restrict__ sums, size_t ntiles, uint64_t* __restrict__ grand) {
  __shared__ uint64_t s_warp[33];
  uint64_t carry = Op::id();
  for (size_t b = 0; b < ntiles; b += blockDim.x) {
    size_t i = b + threadIdx.x;
    uint64_t v = i < ntiles ? sums[i] : Op::id(), tot;
    uint64_t ex = block_excl_scan<Op>(v, s_warp, &tot);
    if (i < ntiles) sums[i] = Op::op(carry, ex);
    carry = Op::op(carry, tot);
  }
  if (threadIdx.x == 0 && grand) *grand = carry;
}

template <class Op>
__global__ void k_scan_apply(const uint64_t* in, size_t n, const uint64_t* __restrict__ sums, uint64_t* out) {
  __shared__ uint64_t s_warp[33];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint64_t v[kScanItems], acc = Op::id();
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    v[k] = base + k < n ? in[base + k] : Op::id();
    acc = Op::op(acc, v[k]);
  }
  uint64_t ex = Op::op(sums[blockIdx.x], block_excl_scan<Op>(acc, s_warp, nullptr));
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    if (base + k < n) out[base + k] = ex;
    ex = Op::op(ex, v[k]);
  }
}

inline size_t scan_tiles(size_t n) {
  size_t t = (n + kScanTile - 1) / kScanTile;
  return t ? t : 1;
}

// Exclusive scan of n u64 values (in may alias out).  `tile_tmp` must hold
// scan_tiles(n) entries; the grand total lands in *grand (device) if given.
template <class Op = ScanSum>
inline void scan_exclusive(const uint64_t* in, uint64_t* out, size_t n, uint64_t* tile_tmp, uint64_t* grand,
                           cudaStream_t st) {
  size_t ntiles = scan_tiles(n);
  k_scan_tile_sums<Op><<<(unsigned)ntiles, kScanThreads, 0, st>>>(in, n, tile_tmp);
  k_scan_sums<Op><<<1, 1024, 0, st>>>(tile_tmp, ntiles, grand);
  k_scan_apply<Op><<<(unsigned)ntiles, kScanThreads, 0, st>>>(in, n, tile_tmp, out);
}

inline void scan_exclusive_u64(const uint64_t* in, uint64_t* out, size_t n, uint64_t* tile_tmp, uint64_t* grand,
                               cudaStream_t st) {
  scan_exclusive<ScanSum>(in, out, n, tile_tmp, grand, st);
}

}  // namespace qb
