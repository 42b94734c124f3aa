"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a plain-C restatement of the reference compressor's in-path
algorithm (see quoin_oracle.c).  Only the tests, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` import this module, and only as the
checker or the timed reference arm — never as part of the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libquoin_oracle.so")

DT_F64, DT_I64, DT_U64, DT_I32, DT_U32, DT_F32, DT_DEC128, DT_DEC256 = range(8)
NATIVE_WIDTH = {DT_F64: 8, DT_I64: 8, DT_U64: 8, DT_I32: 4, DT_U32: 4, DT_F32: 4,
                DT_DEC128: 16, DT_DEC256: 32}
NP_DTYPE = {DT_F64: np.float64, DT_I64: np.int64, DT_U64: np.uint64, DT_I32: np.int32,
            DT_U32: np.uint32, DT_F32: np.float32}

ERR_NAMES = {1: "BadMagic", 2: "UnsupportedVersion", 3: "Truncated", 4: "UnknownMode",
             5: "CorruptPayload", 6: "LengthMismatch", 7: "UnsupportedDType",
             8: "DTypeMismatch", 9: "Unsupported", 10: "BadArg"}

LEVEL_FASTEST, LEVEL_FAST, LEVEL_BALANCED_INPOOL = 0, 1, 2
SELECT_SAMPLE = 0x100  # added to a level: Selection::Sample (reference src/encoder.rs:470-620)


class OracleError(Exception):
    def __init__(self, code: int):
        super().__init__(ERR_NAMES.get(code, f"code {code}"))
        self.code = code
        self.kind = ERR_NAMES.get(code, str(code))


def build() -> str:
    """Compile the oracle with its Makefile (gcc only, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P, S, U8P = ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint8)
        L.oq_compress_column.argtypes = [ctypes.c_int, S, P, P, ctypes.c_int8, ctypes.c_uint8,
                                         ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                         ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_compress_column_mt.argtypes = [ctypes.c_int, S, P, P, ctypes.c_int8, ctypes.c_uint8,
                                            ctypes.c_int, ctypes.c_long, ctypes.c_int,
                                            ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_decompress_column.argtypes = [P, S, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(S),
                                           ctypes.POINTER(P), ctypes.POINTER(U8P),
                                           ctypes.POINTER(ctypes.c_int8),
                                           ctypes.POINTER(ctypes.c_uint8)]
        L.oq_decompress_column_mt.argtypes = [P, S, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(S), ctypes.POINTER(P),
                                              ctypes.POINTER(U8P), ctypes.POINTER(ctypes.c_int8),
                                              ctypes.POINTER(ctypes.c_uint8)]
        L.oq_free.argtypes = [P]
        L.oq_rans_compress.argtypes = [P, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_rans_decompress.argtypes = [P, S, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_encode_mode.argtypes = [ctypes.c_int, P, S, ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_decode_mode.argtypes = [ctypes.c_int, P, S, S, ctypes.c_int, P]
        L.oq_linear_payload.argtypes = [ctypes.c_int, P, S, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_rc_compress.argtypes = [P, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_linear_select_order.argtypes = [P, S]
        L.oq_pred_payload.argtypes = [ctypes.c_int, P, S, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_tans_compress.argtypes = [P, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_tans_decompress.argtypes = [P, S, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_crc32c_u64.argtypes = [ctypes.c_uint32, ctypes.c_uint64]
        L.oq_crc32c_u64.restype = ctypes.c_uint32
        L.oq_lz_compress.argtypes = [P, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_lz_decompress.argtypes = [P, S, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_rc_decompress.argtypes = [P, S, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_pack32.argtypes = [P, ctypes.c_uint32, P]
        L.oq_unpack32.argtypes = [P, ctypes.c_uint32, P]
        L.oq_pack64.argtypes = [P, ctypes.c_uint32, P]
        L.oq_unpack64.argtypes = [P, ctypes.c_uint32, P]
        L.oq_validity_encode.argtypes = [P, S, ctypes.POINTER(U8P), ctypes.POINTER(S)]
        L.oq_validity_decode.argtypes = [P, S, S, P]
        L.oq_mode_win_counts.argtypes = [P]
        L.oq_probe_windows.argtypes = [P, S, P]
        _lib = L
    return _lib


def _take(ptr, n) -> bytes:
    if not ptr:
        return None
    data = ctypes.string_at(ptr, n)
    lib().oq_free(ptr)
    return data


def _ptr(a):
    return None if a is None else a.ctypes.data


def compress_column(values: np.ndarray, dtype: int, validity=None, level: int = LEVEL_FAST,
                    block_size=None, scale: int = 0, precision: int = 0, predictor_log2: int = 16,
                    threads: int = 1, sample: bool = False) -> bytes:
    values = np.ascontiguousarray(values)
    if sample:
        level |= SELECT_SAMPLE
    n = values.nbytes // NATIVE_WIDTH[dtype]
    vb = None if validity is None else np.ascontiguousarray(validity, dtype=np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    bs = 0 if block_size is None else int(block_size)
    if threads > 1:
        rc = lib().oq_compress_column_mt(dtype, n, _ptr(values), _ptr(vb), scale, precision, level,
                                         bs, threads, ctypes.byref(out), ctypes.byref(olen))
    else:
        rc = lib().oq_compress_column(dtype, n, _ptr(values), _ptr(vb), scale, precision, level, bs,
                                      predictor_log2, ctypes.byref(out), ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value)


def decompress_column(stream: bytes, threads: int = 1):
    """Returns (dtype, values ndarray, validity ndarray|None, scale, precision)."""
    buf = np.frombuffer(stream, dtype=np.uint8) if len(stream) else np.zeros(1, np.uint8)
    dt = ctypes.c_int()
    n = ctypes.c_size_t()
    vals = ctypes.c_void_p()
    bm = ctypes.POINTER(ctypes.c_uint8)()
    sc = ctypes.c_int8()
    pr = ctypes.c_uint8()
    if threads > 1:
        rc = lib().oq_decompress_column_mt(buf.ctypes.data, len(stream), threads, ctypes.byref(dt),
                                           ctypes.byref(n), ctypes.byref(vals), ctypes.byref(bm),
                                           ctypes.byref(sc), ctypes.byref(pr))
    else:
        rc = lib().oq_decompress_column(buf.ctypes.data, len(stream), ctypes.byref(dt),
                                        ctypes.byref(n), ctypes.byref(vals), ctypes.byref(bm),
                                        ctypes.byref(sc), ctypes.byref(pr))
    if rc:
        raise OracleError(rc)
    w = NATIVE_WIDTH[dt.value]
    raw = _take(vals.value, n.value * w) or b""
    if dt.value in NP_DTYPE:
        arr = np.frombuffer(raw, dtype=NP_DTYPE[dt.value]).copy()
    else:
        arr = np.frombuffer(raw, dtype=np.uint8).reshape(n.value, w).copy()
    bmp = ctypes.cast(bm, ctypes.c_void_p).value
    validity = None
    if bmp:
        validity = np.frombuffer(_take(bmp, (n.value + 7) // 8) or b"", dtype=np.uint8).copy()
    return dt.value, arr, validity, sc.value, pr.value


def rans_compress(data: bytes):
    a = np.frombuffer(data, dtype=np.uint8) if data else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    lib().oq_rans_compress(a.ctypes.data, len(data), ctypes.byref(out), ctypes.byref(olen))
    p = ctypes.cast(out, ctypes.c_void_p).value
    return _take(p, olen.value) if p else None


def rans_decompress(payload: bytes, max_len: int) -> bytes:
    a = np.frombuffer(payload, dtype=np.uint8) if payload else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_rans_decompress(a.ctypes.data, len(payload), max_len, ctypes.byref(out),
                                  ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""


def rc_compress(data: bytes) -> bytes:
    """The range coder (entropy/rc.rs): varint(len) ++ coded bytes."""
    a = np.frombuffer(data, dtype=np.uint8) if data else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    lib().oq_rc_compress(a.ctypes.data, len(data), ctypes.byref(out), ctypes.byref(olen))
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""


def rc_decompress(payload: bytes, max_len: int) -> bytes:
    a = np.frombuffer(payload, dtype=np.uint8) if payload else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_rc_decompress(a.ctypes.data, len(payload), max_len, ctypes.byref(out), ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""


TAG_RC, TAG_TANS, TAG_RANS = 0, 1, 2


def tans_compress(data: bytes):
    """tans.rs compress_bytes: the coded bytes (no tag), None where the coder declines."""
    a = np.frombuffer(data, dtype=np.uint8) if data else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_tans_compress(a.ctypes.data, len(data), ctypes.byref(out), ctypes.byref(olen))
    if rc:
        return None
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value)


def tans_decompress(payload: bytes, max_len: int) -> bytes:
    a = np.frombuffer(payload, dtype=np.uint8) if payload else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_tans_decompress(a.ctypes.data, len(payload), max_len, ctypes.byref(out), ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""
M_ORDERED_DELTA, M_DELTA2, M_DELTA_DP = 7, 20, 45


M_PRED, M_PRED2, M_PRED_RC = 0, 25, 29


def pred_payload(mode: int, lane: np.ndarray, plog2: int = 16, tag: int = TAG_RC) -> bytes:
    """A PRED / PRED_RC / PRED2 frame payload (codecs/pred.rs)."""
    lane = np.ascontiguousarray(lane, dtype=np.uint64)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_pred_payload(mode, lane.ctypes.data, lane.size, plog2, tag, ctypes.byref(out), ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""


def lz_compress(data: bytes) -> bytes:
    """The LZ stream of codecs/lz.rs."""
    a = np.frombuffer(data, dtype=np.uint8) if data else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    lib().oq_lz_compress(a.ctypes.data, len(data), ctypes.byref(out), ctypes.byref(olen))
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""


def lz_decompress(stream: bytes, expected: int) -> bytes:
    a = np.frombuffer(stream, dtype=np.uint8) if stream else np.zeros(1, np.uint8)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_lz_decompress(a.ctypes.data, len(stream), expected, ctypes.byref(out), ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    return _take(ctypes.cast(out, ctypes.c_void_p).value, olen.value) or b""


M_LZ, TAG_LZ = 4, 3


def crc32c_u64(crc: int, v: int) -> int:
    return lib().oq_crc32c_u64(crc, v)


def linear_select_order(lane: np.ndarray) -> int:
    lane = np.ascontiguousarray(lane, dtype=np.uint64)
    return lib().oq_linear_select_order(lane.ctypes.data, lane.size)


def linear_payload(mode: int, lane: np.ndarray, order: int = 0, tag: int = TAG_RC):
    """A DELTA2 / DELTA_DP / ORDERED_DELTA frame payload (codecs/linear.rs) whose
    residual bytes are coded by `tag`; None when DELTA_DP does not apply."""
    lane = np.ascontiguousarray(lane, dtype=np.uint64)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_linear_payload(mode, lane.ctypes.data, lane.size, order, tag, ctypes.byref(out),
                                 ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    p = ctypes.cast(out, ctypes.c_void_p).value
    return _take(p, olen.value) if p else None


def encode_mode(mode: int, lane: np.ndarray, dtype: int = DT_U64, level: int = LEVEL_FAST):
    lane = np.ascontiguousarray(lane, dtype=np.uint64)
    out = ctypes.POINTER(ctypes.c_uint8)()
    olen = ctypes.c_size_t()
    rc = lib().oq_encode_mode(mode, lane.ctypes.data, lane.size, dtype, level, ctypes.byref(out),
                              ctypes.byref(olen))
    if rc:
        raise OracleError(rc)
    p = ctypes.cast(out, ctypes.c_void_p).value
    return _take(p, olen.value) if p else None


def decode_mode(mode: int, payload: bytes, n: int, dtype: int = DT_U64) -> np.ndarray:
    a = np.frombuffer(payload, dtype=np.uint8) if payload else np.zeros(1, np.uint8)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    rc = lib().oq_decode_mode(mode, a.ctypes.data, len(payload), n, dtype, out.ctypes.data)
    if rc:
        raise OracleError(rc)
    return out[:n]


def pack32(values: np.ndarray, width: int) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.uint32)
    out = np.zeros(max(32 * width, 1), dtype=np.uint32)
    lib().oq_pack32(v.ctypes.data, width, out.ctypes.data)
    return out[:32 * width]


def unpack32(packed: np.ndarray, width: int) -> np.ndarray:
    p = np.ascontiguousarray(packed, dtype=np.uint32)
    if p.size == 0:
        p = np.zeros(1, np.uint32)
    out = np.zeros(1024, dtype=np.uint32)
    lib().oq_unpack32(p.ctypes.data, width, out.ctypes.data)
    return out


def pack64(values: np.ndarray, width: int) -> np.ndarray:
    v = np.ascontiguousarray(values, dtype=np.uint64)
    out = np.zeros(max(16 * width, 1), dtype=np.uint64)
    lib().oq_pack64(v.ctypes.data, width, out.ctypes.data)
    return out[:16 * width]


def unpack64(packed: np.ndarray, width: int) -> np.ndarray:
    p = np.ascontiguousarray(packed, dtype=np.uint64)
    if p.size == 0:
        p = np.zeros(1, np.uint64)
    out = np.zeros(1024, dtype=np.uint64)
    lib().oq_unpack64(p.ctypes.data, width, out.ctypes.data)
    return out


def probe_windows(lane: np.ndarray) -> np.ndarray:
    """plan_blocks' probe byte for every 32,768-value window of a u64 lane."""
    lane = np.ascontiguousarray(lane, dtype=np.uint64)
    flags = np.zeros(max((lane.size + 32767) // 32768, 1), dtype=np.uint8)
    lib().oq_probe_windows(_ptr(lane), lane.size, _ptr(flags))
    return flags[: (lane.size + 32767) // 32768]


def mode_win_counts() -> np.ndarray:
    out = np.zeros(64, dtype=np.uint64)
    lib().oq_mode_win_counts(out.ctypes.data)
    return out


def reset_mode_win_counts() -> None:
    lib().oq_reset_mode_win_counts()
