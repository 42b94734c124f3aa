// Arrow adapter over the Arrow C Data Interface (replaces the reference's
// src/arrow.rs compress_array / decompress_array, which take arrow-rs arrays;
// a C ABI cannot, so the standard ArrowSchema / ArrowArray structs stand in).
//
// Supported types, as in the reference: Float64 "g", Float32 "f", Int64 "l",
// UInt64 "L", Int32 "i", UInt32 "I", Decimal128 "d:P,S[,128]" and Decimal256
// "d:P,S,256"; anything else is QUOIN_ERR_UNSUPPORTED_ARROW_TYPE.  An Arrow
// validity bitmap is quoin's validity format (LSB first, 1 = valid); a sliced
// array's bitmap is re-packed from its first logical bit (arrow.rs:29-52).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/quoin.h"
#include "qb_kernels.h"

namespace {

struct ArrowType {
  int32_t wire = -1;
  uint32_t width = 0;
  int precision = 0, scale = 0;
};

// Format string -> wire dtype (src/arrow.rs:61-123); false when unsupported.
bool arrow_type(const char* f, ArrowType* t) {
  if (!f) return false;
  if (!strcmp(f, "g")) *t = {QUOIN_WIRE_F64, 8};
  else if (!strcmp(f, "f")) *t = {QUOIN_WIRE_F32, 4};
  else if (!strcmp(f, "l")) *t = {QUOIN_WIRE_I64, 8};
  else if (!strcmp(f, "L")) *t = {QUOIN_WIRE_U64, 8};
  else if (!strcmp(f, "i")) *t = {QUOIN_WIRE_I32, 4};
  else if (!strcmp(f, "I")) *t = {QUOIN_WIRE_U32, 4};
  else if (f[0] == 'd' && f[1] == ':') {
    int p = 0, s = 0, bits = 128, used = 0;
    int k = sscanf(f + 2, "%d,%d%n", &p, &s, &used);
    if (k != 2) return false;
    const char* rest = f + 2 + used;
    if (*rest == ',') {
      int u2 = 0;
      if (sscanf(rest + 1, "%d%n", &bits, &u2) != 1 || rest[1 + u2] != 0) return false;
    } else if (*rest != 0) {
      return false;
    }
    if (p < 0 || p > 255 || s < -128 || s > 127) return false;
    if (bits == 128) *t = {QUOIN_WIRE_DECIMAL128, 16, p, s};
    else if (bits == 256) *t = {QUOIN_WIRE_DECIMAL256, 32, p, s};
    else return false;
  } else {
    return false;
  }
  return true;
}

// The array's validity as a bitmap from logical bit 0 (trailing bits clear),
// or empty when the array has no validity buffer.
std::vector<uint8_t> repack_validity(const ArrowArray* a) {
  std::vector<uint8_t> bm;
  const uint8_t* src = a->n_buffers > 0 ? static_cast<const uint8_t*>(a->buffers[0]) : nullptr;
  if (!src || a->null_count == 0) return bm;
  uint64_t n = (uint64_t)a->length, off = (uint64_t)a->offset;
  bm.assign((n + 7) / 8, 0);
  if (off % 8 == 0) {
    if (n) memcpy(bm.data(), src + off / 8, bm.size());
  } else {
    for (uint64_t i = 0; i < n; i++) {
      uint64_t b = off + i;
      if ((src[b >> 3] >> (b & 7)) & 1u) bm[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
  }
  if (n & 7) bm[bm.size() - 1] &= (uint8_t)((1u << (n & 7)) - 1u);
  return bm;
}

struct SchemaPrivate {
  char format[32];
};
struct ArrayPrivate {
  void* values;
  uint8_t* validity;
  const void* buffers[2];
};

void release_schema(ArrowSchema* s) {
  if (!s || !s->release) return;
  delete static_cast<SchemaPrivate*>(s->private_data);
  s->release = nullptr;
}
void release_array(ArrowArray* a) {
  if (!a || !a->release) return;
  ArrayPrivate* p = static_cast<ArrayPrivate*>(a->private_data);
  free(p->values);
  free(p->validity);
  delete p;
  a->release = nullptr;
}

}  // namespace

extern "C" int quoin_b200_compress_arrow(QuoinCtx* ctx, const ArrowSchema* schema, const ArrowArray* array,
                                         const QuoinConfig* cfg, uint8_t* dst, size_t dst_cap, size_t* out_len) {
  if (!schema || !array || !dst || !out_len) return QUOIN_ERR_NULL;
  try {
    ArrowType t;
    if (!arrow_type(schema->format, &t) || schema->n_children != 0 || schema->dictionary) {
      return QUOIN_ERR_UNSUPPORTED_ARROW_TYPE;
    }
    if (array->length < 0 || array->offset < 0 || array->n_buffers < 2) return QUOIN_ERR_BAD_ARG;
    uint64_t n = (uint64_t)array->length;
    const uint8_t* base = static_cast<const uint8_t*>(array->buffers[1]);
    if (!base && n) return QUOIN_ERR_NULL;
    const uint8_t* values = base ? base + (uint64_t)array->offset * t.width : nullptr;
    std::vector<uint8_t> bm = repack_validity(array);
    return quoin_b200_compress_column(ctx, t.wire, n, values, bm.empty() ? nullptr : bm.data(), (int8_t)t.scale,
                                      (uint8_t)t.precision, cfg, dst, dst_cap, out_len);
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

extern "C" int quoin_b200_decompress_arrow(QuoinCtx* ctx, const uint8_t* src, size_t src_len,
                                           ArrowSchema* schema_out, ArrowArray* array_out) {
  if (!src || !schema_out || !array_out) return QUOIN_ERR_NULL;
  try {
    int32_t wire = 0, has_validity = 0;
    uint64_t n = 0;
    int8_t scale = 0;
    uint8_t precision = 0;
    int rc = quoin_b200_stream_info(src, src_len, &wire, &n, &has_validity, &scale, &precision);
    if (rc) return rc;
    ArrowType t;
    const char* fmt = nullptr;
    switch (wire) {
      case QUOIN_WIRE_F64: fmt = "g"; t.width = 8; break;
      case QUOIN_WIRE_F32: fmt = "f"; t.width = 4; break;
      case QUOIN_WIRE_I64: fmt = "l"; t.width = 8; break;
      case QUOIN_WIRE_U64: fmt = "L"; t.width = 8; break;
      case QUOIN_WIRE_I32: fmt = "i"; t.width = 4; break;
      case QUOIN_WIRE_U32: fmt = "I"; t.width = 4; break;
      case QUOIN_WIRE_DECIMAL128: t.width = 16; break;
      case QUOIN_WIRE_DECIMAL256: t.width = 32; break;
      default: return QUOIN_ERR_UNSUPPORTED_DTYPE;
    }
    // 64-byte aligned buffers, as Arrow recommends
    size_t vbytes = ((size_t)n * t.width + 63) & ~(size_t)63;
    void* values = aligned_alloc(64, vbytes ? vbytes : 64);
    uint8_t* validity = nullptr;
    if (!values) return QUOIN_ERR_PANIC;
    if (has_validity) {
      size_t bbytes = (((size_t)n + 7) / 8 + 63) & ~(size_t)63;
      validity = static_cast<uint8_t*>(aligned_alloc(64, bbytes ? bbytes : 64));
      if (!validity) {
        free(values);
        return QUOIN_ERR_PANIC;
      }
      memset(validity, 0, bbytes ? bbytes : 64);
    }
    rc = quoin_b200_decompress_column(ctx, src, src_len, values, validity);
    if (rc) {
      free(values);
      free(validity);
      return rc;
    }
    int64_t nulls = 0;
    if (validity) {
      uint64_t valid = 0;
      for (uint64_t i = 0; i < (n + 7) / 8; i++) valid += (uint64_t)__builtin_popcount(validity[i]);
      nulls = (int64_t)(n - valid);
    }
    SchemaPrivate* sp = new SchemaPrivate();
    if (fmt) snprintf(sp->format, sizeof sp->format, "%s", fmt);
    else if (wire == QUOIN_WIRE_DECIMAL128) snprintf(sp->format, sizeof sp->format, "d:%d,%d", precision, scale);
    else snprintf(sp->format, sizeof sp->format, "d:%d,%d,256", precision, scale);
    ArrayPrivate* ap = new ArrayPrivate();
    ap->values = values;
    ap->validity = validity;
    ap->buffers[0] = validity;
    ap->buffers[1] = values;

    memset(schema_out, 0, sizeof *schema_out);
    schema_out->format = sp->format;
    schema_out->name = "";
    schema_out->flags = ARROW_FLAG_NULLABLE;
    schema_out->release = release_schema;
    schema_out->private_data = sp;

    memset(array_out, 0, sizeof *array_out);
    array_out->length = (int64_t)n;
    array_out->null_count = nulls;
    array_out->n_buffers = 2;
    array_out->buffers = ap->buffers;
    array_out->release = release_array;
    array_out->private_data = ap;
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

// ---------------------------------------------------------------------------
// Arrow C Device Data Interface: device-resident arrays, read and written in
// place (no host copy of the values).
// ---------------------------------------------------------------------------
namespace {

// The Arrow format of a stream's wire dtype (and decimal scale / precision).
bool format_of(int32_t wire, int8_t scale, uint8_t precision, char* out, size_t cap, uint32_t* width) {
  switch (wire) {
    case QUOIN_WIRE_F64: snprintf(out, cap, "g"); *width = 8; return true;
    case QUOIN_WIRE_F32: snprintf(out, cap, "f"); *width = 4; return true;
    case QUOIN_WIRE_I64: snprintf(out, cap, "l"); *width = 8; return true;
    case QUOIN_WIRE_U64: snprintf(out, cap, "L"); *width = 8; return true;
    case QUOIN_WIRE_I32: snprintf(out, cap, "i"); *width = 4; return true;
    case QUOIN_WIRE_U32: snprintf(out, cap, "I"); *width = 4; return true;
    case QUOIN_WIRE_DECIMAL128: snprintf(out, cap, "d:%d,%d", precision, scale); *width = 16; return true;
    case QUOIN_WIRE_DECIMAL256: snprintf(out, cap, "d:%d,%d,256", precision, scale); *width = 32; return true;
    default: return false;
  }
}

struct DeviceArrayPrivate {
  void* values;
  uint8_t* validity;
  const void* buffers[2];
};

void release_device_array(ArrowArray* a) {
  if (!a || !a->release) return;
  DeviceArrayPrivate* p = static_cast<DeviceArrayPrivate*>(a->private_data);
  cudaFree(p->values);
  if (p->validity) cudaFree(p->validity);
  delete p;
  a->release = nullptr;
}

}  // namespace

extern "C" int quoin_b200_compress_arrow_device(QuoinCtx* ctx, const ArrowSchema* schema, const ArrowDeviceArray* darr,
                                                const QuoinConfig* cfg, uint8_t* d_dst, size_t dst_cap,
                                                size_t* out_len, void* stream) {
  if (!schema || !darr || !d_dst || !out_len) return QUOIN_ERR_NULL;
  try {
    ArrowType t;
    if (!arrow_type(schema->format, &t) || schema->n_children != 0 || schema->dictionary) {
      return QUOIN_ERR_UNSUPPORTED_ARROW_TYPE;
    }
    if (darr->device_type != ARROW_DEVICE_CUDA && darr->device_type != ARROW_DEVICE_CUDA_MANAGED) {
      return QUOIN_ERR_BAD_ARG;
    }
    const ArrowArray* a = &darr->array;
    if (a->length < 0 || a->offset < 0 || a->n_buffers < 2) return QUOIN_ERR_BAD_ARG;
    uint64_t n = (uint64_t)a->length, off = (uint64_t)a->offset;
    const uint8_t* base = static_cast<const uint8_t*>(a->buffers[1]);
    if (!base && n) return QUOIN_ERR_NULL;
    cudaStream_t st = qb::ctx_stream(ctx, stream);
    if (darr->sync_event && cudaStreamWaitEvent(st, *static_cast<cudaEvent_t*>(darr->sync_event), 0) != cudaSuccess) {
      cudaGetLastError();
      return QUOIN_ERR_CUDA;
    }
    const uint8_t* values = base ? base + off * t.width : nullptr;
    const uint8_t* src_bm = static_cast<const uint8_t*>(a->buffers[0]);
    uint8_t* bm = nullptr;
    if (src_bm && a->null_count != 0 && n) {  // re-packed from the array's offset, trailing bits clear
      if (cudaMallocAsync(reinterpret_cast<void**>(&bm), (n + 7) / 8, st) != cudaSuccess) {
        cudaGetLastError();
        return QUOIN_ERR_CUDA;
      }
      qb::launch_bitmap_repack(src_bm, off, n, bm, st);
    }
    int rc = quoin_b200_compress_column_device(ctx, t.wire, n, values, bm, (int8_t)t.scale, (uint8_t)t.precision, cfg,
                                               d_dst, dst_cap, out_len, st);
    if (bm) cudaFreeAsync(bm, st);
    return rc;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}

extern "C" int quoin_b200_decompress_arrow_device(QuoinCtx* ctx, const QuoinDecodeIndex* idx, const uint8_t* d_src,
                                                  ArrowSchema* schema_out, ArrowDeviceArray* out, void* stream) {
  if (!idx || !d_src || !schema_out || !out) return QUOIN_ERR_NULL;
  try {
    int32_t wire = 0, hv = 0;
    uint64_t n = 0, n_valid = 0;
    int8_t scale = 0;
    uint8_t precision = 0;
    int rc = quoin_b200_index_info(idx, &wire, &n, &hv);
    if (!rc) rc = quoin_b200_index_decimal(idx, &scale, &precision, &n_valid);
    if (rc) return rc;
    SchemaPrivate* sp = new SchemaPrivate();
    uint32_t width = 0;
    if (!format_of(wire, scale, precision, sp->format, sizeof sp->format, &width)) {
      delete sp;
      return QUOIN_ERR_UNSUPPORTED_DTYPE;
    }
    // 64-byte aligned device buffers, as Arrow recommends (cudaMalloc aligns to 256)
    void* values = nullptr;
    uint8_t* validity = nullptr;
    size_t vbytes = (size_t)n * width;
    if (cudaMalloc(&values, vbytes ? vbytes : 64) != cudaSuccess ||
        (hv && cudaMalloc(reinterpret_cast<void**>(&validity), (n + 7) / 8 ? (n + 7) / 8 : 64) != cudaSuccess)) {
      cudaGetLastError();
      cudaFree(values);
      delete sp;
      return QUOIN_ERR_CUDA;
    }
    rc = quoin_b200_decompress_indexed_device(ctx, idx, d_src, values, validity, stream);
    if (rc) {
      cudaFree(values);
      if (validity) cudaFree(validity);
      delete sp;
      return rc;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    DeviceArrayPrivate* ap = new DeviceArrayPrivate();
    ap->values = values;
    ap->validity = validity;
    ap->buffers[0] = validity;
    ap->buffers[1] = values;

    memset(schema_out, 0, sizeof *schema_out);
    schema_out->format = sp->format;
    schema_out->name = "";
    schema_out->flags = ARROW_FLAG_NULLABLE;
    schema_out->release = release_schema;
    schema_out->private_data = sp;

    memset(out, 0, sizeof *out);
    out->array.length = (int64_t)n;
    out->array.null_count = hv ? (int64_t)(n - n_valid) : 0;
    out->array.n_buffers = 2;
    out->array.buffers = ap->buffers;
    out->array.release = release_device_array;
    out->array.private_data = ap;
    out->device_id = dev;
    out->device_type = ARROW_DEVICE_CUDA;
    out->sync_event = nullptr;  // the call returned after the decode completed
    return QUOIN_OK;
  } catch (...) {
    return QUOIN_ERR_PANIC;
  }
}
