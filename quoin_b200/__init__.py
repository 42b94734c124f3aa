"""quoin_b200 — B200-native quoin column compressor.

Python mirror of the reference crate's public API (src/lib.rs): ``Config``,
``Level``, ``compress``/``decompress``, ``compress_column``/
``decompress_column``, ``decompressed_len``, ``mode_win_counts``.  Every call
goes through the C ABI of ``libquoin_b200.so`` (include/quoin.h), whose
competition and block decoder run as sm_100a CUDA kernels.  There is no CPU
fallback: importing the package without the built library raises.
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libquoin_b200.so")

MAX_BLOCK_SIZE = 131072  # reference src/lib.rs:250

# Extended error codes (include/quoin.h) -> reference Error variants (src/error.rs).
_ERRORS = {
    -10: "BadMagic", -11: "UnsupportedVersion", -12: "Truncated", -13: "UnknownMode",
    -14: "CorruptPayload", -15: "LengthMismatch", -16: "UnsupportedDType", -17: "DTypeMismatch",
    -18: "Unsupported", -19: "Cuda", -20: "BadArg", -1: "Null", -2: "BufferTooSmall", -3: "Corrupt",
    -4: "Panic", -21: "NoAllocLimit", -22: "UnsupportedArrowType", -23: "OverBudget", -24: "Timeout",
}


class Error(Exception):
    """A decode/encode failure; ``kind`` names the reference Error variant."""

    def __init__(self, code: int):
        self.code = code
        self.kind = _ERRORS.get(code, f"code {code}")
        super().__init__(self.kind)


class Level(enum.IntEnum):
    """Speed/ratio ladder (reference src/lib.rs:93-119).  BALANCED_INPOOL is
    Balanced's competition without its Lz and Pco candidates (lambda 2, the
    rANS-coded FLOAT_MULT / ALP-RD / DICT parts and BYTE_TRANSPOSE): reference
    streams, equal to Level.BALANCED's wherever neither Lz nor Pco would win."""
    FASTEST = 0
    FAST = 1
    BALANCED = 2
    HIGH = 3
    MAX = 4
    BALANCED_INPOOL = 258


class Selection(enum.Enum):
    """Mode selection (reference src/lib.rs:65-73): FULL sizes every candidate
    on the whole block; SAMPLE sizes them on a stratified sample and encodes
    only the winner in full (Level.FASTEST and Level.FAST)."""
    FULL = "full"
    SAMPLE = "sample"


@dataclass
class Config:
    """Encoder configuration (reference src/lib.rs:195-245).  The GPU covers
    Level.FASTEST, Level.FAST and Level.BALANCED_INPOOL; ``block_size=None``
    selects adaptive blocks."""
    level: Level = Level.FAST
    block_size: Optional[int] = None
    predictor_log2: int = 16
    selection: Selection = Selection.FULL
    threads: Optional[int] = None


class _QuoinConfig(ctypes.Structure):
    _fields_ = [("level", ctypes.c_int32), ("block_size", ctypes.c_int64), ("predictor_log2", ctypes.c_int32),
                ("selection", ctypes.c_int32)]


# Stream dtype wire ids (reference src/dtype.rs:68-78).
F64, I64, U64, I32, U32, F32, DECIMAL128, DECIMAL256 = range(8)
DTYPE_NAMES = {F64: "f64", I64: "i64", U64: "u64", I32: "i32", U32: "u32", F32: "f32",
               DECIMAL128: "decimal128", DECIMAL256: "decimal256"}
NATIVE_WIDTH = {F64: 8, I64: 8, U64: 8, I32: 4, U32: 4, F32: 4, DECIMAL128: 16, DECIMAL256: 32}
_NP = {F64: np.float64, I64: np.int64, U64: np.uint64, I32: np.int32, U32: np.uint32, F32: np.float32}
_FROM_NP = {np.dtype(np.float64): F64, np.dtype(np.int64): I64, np.dtype(np.uint64): U64,
            np.dtype(np.int32): I32, np.dtype(np.uint32): U32, np.dtype(np.float32): F32}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python quoin_b200/build.py` (nvcc, sm_100a)")
    L = ctypes.CDLL(LIB_PATH)
    P, S = ctypes.c_void_p, ctypes.c_size_t
    L.quoin_version.restype = ctypes.c_char_p
    L.quoin_compress_bound.argtypes = [S]
    L.quoin_compress_bound.restype = S
    L.quoin_compress.argtypes = [P, S, P, S, ctypes.POINTER(S)]
    L.quoin_decompress.argtypes = [P, S, P, S, ctypes.POINTER(S)]
    L.quoin_decompressed_value_count.argtypes = [P, S]
    L.quoin_decompressed_value_count.restype = ctypes.c_ssize_t
    L.quoin_ctx_create.argtypes = [S]
    L.quoin_ctx_create.restype = P
    L.quoin_ctx_free.argtypes = [P]
    L.quoin_compress_ctx.argtypes = [P, P, S, P, S, ctypes.POINTER(S)]
    L.quoin_decompress_ctx.argtypes = [P, P, S, P, S, ctypes.POINTER(S)]
    L.quoin_dtype_width.argtypes = [ctypes.c_int32]
    L.quoin_dtype_width.restype = S
    L.quoin_typed_compress_bound.argtypes = [ctypes.c_int32, S]
    L.quoin_typed_compress_bound.restype = S
    L.quoin_typed_compress.argtypes = [ctypes.c_int32, S, P, P, P, S]
    L.quoin_typed_compress.restype = S
    L.quoin_typed_compress_decimal.argtypes = [ctypes.c_int32, S, P, P, ctypes.c_int8, ctypes.c_uint8, P, S]
    L.quoin_typed_compress_decimal.restype = S
    L.quoin_typed_decompress.argtypes = [ctypes.c_int32, S, P, S, P, P]
    L.quoin_b200_compress_column.argtypes = [P, ctypes.c_int32, S, P, P, ctypes.c_int8, ctypes.c_uint8,
                                             ctypes.POINTER(_QuoinConfig), P, S, ctypes.POINTER(S)]
    L.quoin_b200_stream_info.argtypes = [P, S, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64),
                                         ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int8),
                                         ctypes.POINTER(ctypes.c_uint8)]
    L.quoin_b200_decompress_column.argtypes = [P, P, S, P, P]
    L.quoin_b200_parse.argtypes = [P, S, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(ctypes.c_int32)]
    L.quoin_b200_timing_enable.argtypes = [ctypes.c_int]
    L.quoin_b200_timing_read.argtypes = [P, P, ctypes.c_int]
    L.quoin_b200_compress_column_device.argtypes = [P, ctypes.c_int32, S, P, P, ctypes.c_int8, ctypes.c_uint8,
                                                    ctypes.POINTER(_QuoinConfig), P, S, ctypes.POINTER(S), P]
    L.quoin_b200_index_create.argtypes = [P, P, S, ctypes.POINTER(P)]
    L.quoin_b200_index_free.argtypes = [P]
    L.quoin_b200_index_info.argtypes = [P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_uint64),
                                        ctypes.POINTER(ctypes.c_int32)]
    L.quoin_b200_decompress_indexed_device.argtypes = [P, P, P, P, P, P]
    L.quoin_b200_decompress_column_device.argtypes = [P, P, S, P, S, P, ctypes.POINTER(ctypes.c_int32),
                                                      ctypes.POINTER(ctypes.c_uint64), P]
    L.quoin_b200_mode_win_counts.argtypes = [P]
    L.quoin_b200_reader_stats.argtypes = [P]
    L.quoin_b200_decompress_queue_device.argtypes = [P, P, S, P]
    L.quoin_b200_reset_mode_win_counts.argtypes = []
    L.quoin_b200_probe_windows_device.argtypes = [P, ctypes.c_int32, S, P, P, P, S, ctypes.POINTER(ctypes.c_uint64), P]
    L.quoin_b200_stream_prefix_device.argtypes = [P, ctypes.c_int32, S, P, ctypes.POINTER(_QuoinConfig), P, S,
                                                  ctypes.POINTER(S), P]
    L.quoin_b200_kernel_launches.restype = ctypes.c_uint64
    return L


lib = _load()

VERSION = lib.quoin_version().decode()


def _cfg(cfg: Optional[Config]) -> _QuoinConfig:
    cfg = cfg or Config()
    return _QuoinConfig(int(cfg.level), int(cfg.block_size or 0), int(cfg.predictor_log2),
                        1 if cfg.selection == Selection.SAMPLE else 0)


def _check(rc: int) -> None:
    if rc != 0:
        raise Error(rc)


def _bitmap(validity, n: int):
    if validity is None:
        return None
    a = np.frombuffer(bytes(validity), dtype=np.uint8) if not isinstance(validity, np.ndarray) else validity
    a = np.ascontiguousarray(a, dtype=np.uint8)
    need = (n + 7) // 8
    if a.size < need:
        raise ValueError(f"validity bitmap needs {need} bytes, got {a.size}")
    return a


def _stream_bound(wire: int, n: int, has_validity: bool, block_size: Optional[int] = None) -> int:
    """Upper bound of a stream's length: header, validity blob, and per block a
    9-byte frame header plus at most the RAW payload (no winner is longer)."""
    lb = 4 if wire in (I32, U32, F32) else 8
    bs = min(max(int(block_size), 1), MAX_BLOCK_SIZE) if block_size else 32768
    blocks = (n + bs - 1) // bs
    vb = 12 + (n + 7) // 8 if has_validity else 0
    if wire in (DECIMAL128, DECIMAL256):
        nl = 2 if wire == DECIMAL128 else 4
        return 19 + 32 + vb + nl * (10 + 16 + 9 * blocks + 8 * n + 64) + 64
    return 16 + vb + 9 * blocks + lb * n + 64


def compress_column(values, validity=None, cfg: Optional[Config] = None, dtype: Optional[int] = None,
                    scale: int = 0, precision: int = 0, ctx=None) -> bytes:
    """Compress a typed column (reference src/lib.rs:429-455).

    ``values`` is a numpy array of f64/i64/u64/i32/u32/f32, or for decimals
    (``dtype=DECIMAL128/DECIMAL256``) an array of n*16 / n*32 little-endian
    bytes (any shape, e.g. (n, 2) int64 limbs).  ``validity`` is an Arrow
    LSB-first bitmap (1 = valid) of ceil(n/8) bytes, or None.
    """
    arr = np.ascontiguousarray(values)
    if dtype is None:
        dtype = _FROM_NP.get(arr.dtype)
        if dtype is None:
            raise TypeError(f"unsupported column dtype {arr.dtype}")
    n = arr.nbytes // NATIVE_WIDTH[dtype]
    bm = _bitmap(validity, n)
    cap = _stream_bound(dtype, n, bm is not None, (cfg or Config()).block_size)
    out = np.empty(max(cap, 16), dtype=np.uint8)
    olen = ctypes.c_size_t()
    c = _cfg(cfg)
    rc = lib.quoin_b200_compress_column(ctx, dtype, n, arr.ctypes.data if n else None,
                                        None if bm is None else bm.ctypes.data, scale, precision,
                                        ctypes.byref(c), out.ctypes.data, out.size, ctypes.byref(olen))
    _check(rc)
    return out[: olen.value].tobytes()


@dataclass
class DecodedColumn:
    """A decoded column (reference src/lib.rs:413-420): values (null slots 0),
    the validity bitmap or None, the wire dtype and decimal scale/precision."""
    values: np.ndarray
    validity: Optional[bytes]
    dtype: int
    scale: int = 0
    precision: int = 0


def stream_info(stream: bytes):
    buf = np.frombuffer(stream, dtype=np.uint8) if stream else np.zeros(1, np.uint8)
    w = ctypes.c_int32()
    n = ctypes.c_uint64()
    hv = ctypes.c_int32()
    sc = ctypes.c_int8()
    pr = ctypes.c_uint8()
    _check(lib.quoin_b200_stream_info(buf.ctypes.data, len(stream), ctypes.byref(w), ctypes.byref(n),
                                      ctypes.byref(hv), ctypes.byref(sc), ctypes.byref(pr)))
    return w.value, n.value, bool(hv.value), sc.value, pr.value


def decompress_column(stream: bytes, ctx=None) -> DecodedColumn:
    """Decompress a stream from ``compress_column`` (reference src/lib.rs:462-508)."""
    buf = np.frombuffer(stream, dtype=np.uint8) if stream else np.zeros(1, np.uint8)
    pw, pn, phv = ctypes.c_int32(), ctypes.c_uint64(), ctypes.c_int32()
    _check(lib.quoin_b200_parse(buf.ctypes.data, len(stream), ctypes.byref(pw), ctypes.byref(pn), ctypes.byref(phv)))
    wire, n, hv, sc, pr = stream_info(stream)
    w = NATIVE_WIDTH[wire]
    out = np.zeros(max(n * w, 8), dtype=np.uint8)
    bm = np.zeros(max((n + 7) // 8, 1), dtype=np.uint8) if hv else None
    _check(lib.quoin_b200_decompress_column(ctx, buf.ctypes.data, len(stream), out.ctypes.data,
                                            None if bm is None else bm.ctypes.data))
    raw = out[: n * w]
    if wire in _NP:
        vals = raw.view(_NP[wire]).copy()
    else:
        vals = raw.reshape(n, w).copy()
    return DecodedColumn(vals, None if bm is None else bm[: (n + 7) // 8].tobytes(), wire, sc, pr)


def compress(values, cfg: Optional[Config] = None) -> bytes:
    """Compress f64 values (reference src/lib.rs:514-516)."""
    return compress_column(np.ascontiguousarray(values, dtype=np.float64), None, cfg, dtype=F64)


def decompress(stream: bytes) -> np.ndarray:
    """Decompress an f64 stream (reference src/lib.rs:522-527)."""
    wire, _, _, _, _ = stream_info(stream)
    if wire != F64:
        raise Error(-17)
    return decompress_column(stream).values


def decompressed_len(stream: bytes) -> int:
    buf = np.frombuffer(stream, dtype=np.uint8) if stream else np.zeros(1, np.uint8)
    r = lib.quoin_decompressed_value_count(buf.ctypes.data, len(stream))
    if r < 0:
        raise Error(-14)
    return int(r)


def mode_win_counts() -> np.ndarray:
    out = np.zeros(64, dtype=np.uint64)
    lib.quoin_b200_mode_win_counts(out.ctypes.data)
    return out


def reset_mode_win_counts() -> None:
    lib.quoin_b200_reset_mode_win_counts()


def kernel_launches() -> int:
    return int(lib.quoin_b200_kernel_launches())


MODE_NAMES = {0: "PRED", 1: "CONST", 2: "STRIDE", 3: "XORZ", 4: "LZ", 5: "RAW", 7: "ORDERED_DELTA", 9: "ALP",
              11: "BYTE_TRANSPOSE", 17: "FLOAT_MULT", 19: "DICT", 20: "DELTA2", 25: "PRED2", 29: "PRED_RC",
              45: "DELTA_DP", 50: "FOR_BITPACK", 51: "DELTA_BITPACK", 52: "ALP_RD", 53: "RLE", 54: "PCO"}


def mode_name(mode_id: int) -> str:
    return MODE_NAMES.get(mode_id, "?")
