// Host/device shared layout of the frame index that drives the block decoder
// and the block encoder.  One entry per frame (= one encoded block).
#pragma once
#include <cstdint>

namespace qb {

struct FrameDesc {
  uint64_t payload_off;  // byte offset of the frame payload within the stream buffer
  uint64_t value_off;    // index of the frame's first value in the compacted lane
  uint32_t n;            // values in the frame (<= 131072)
  uint32_t plen;         // payload bytes
  uint32_t mode;         // mode wire id
  uint32_t aux;          // encoder: winner-specific parameter; decoder: unused
};
static_assert(sizeof(FrameDesc) == 32, "FrameDesc layout");

}  // namespace qb
