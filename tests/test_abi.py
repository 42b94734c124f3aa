"""CPU checks of the drop-in boundary: libquoin_b200.so loads, exports every
function include/quoin.h declares (the reference capi/include/quoin.h symbols
plus the B200 extensions), and its host-only entry points (bounds, widths,
header parsing) match the reference's rules.  No kernel is launched here."""
import ctypes
import os
import re
import struct

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "quoin.h")

REFERENCE_SYMBOLS = [  # capi/include/quoin.h:36-142
    "quoin_version", "quoin_compress_bound", "quoin_compress", "quoin_decompress",
    "quoin_decompressed_value_count", "quoin_ctx_create", "quoin_ctx_free", "quoin_compress_ctx",
    "quoin_decompress_ctx", "quoin_dtype_width", "quoin_typed_compress_bound", "quoin_typed_compress",
    "quoin_typed_compress_decimal", "quoin_typed_decompress",
]


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(quoin_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_reference_symbols():
    decl = declared_functions()
    for s in REFERENCE_SYMBOLS:
        assert s in decl, s


def test_library_exports_every_declared_symbol(qb):
    lib = ctypes.CDLL(qb.LIB_PATH)
    missing = [s for s in declared_functions() if not hasattr(lib, s)]
    assert not missing, missing


def test_host_only_entry_points(qb):
    L = qb.lib
    assert L.quoin_compress_bound(0) == 1024 and L.quoin_compress_bound(10) == 1114
    widths = {0: 1, 1: 1, 2: 2, 3: 4, 4: 8, 5: 1, 6: 2, 7: 4, 8: 8, 9: 4, 10: 8, 11: 4, 12: 8, 13: 16, 14: 32,
              15: 0, -1: 0}
    for d, w in widths.items():
        assert L.quoin_dtype_width(d) == w
    assert L.quoin_typed_compress_bound(1, 100) == 100 * 9 + 1024     # capi/src/typed.rs:65-69
    assert L.quoin_typed_compress_bound(14, 100) == 100 * 33 + 1024
    assert qb.VERSION.startswith("quoin")


def test_header_parsing_matches_reference_rules(qb):
    good = b"FCR1" + bytes([2, 0, 16, 0]) + struct.pack("<Q", 12345)
    assert qb.decompressed_len(good) == 12345
    assert qb.stream_info(good) == (0, 12345, False, 0, 0)
    bad_cases = {
        b"FCR1\x02": "Truncated",
        b"XCR1" + good[4:]: "BadMagic",
        good[:4] + b"\x03" + good[5:]: "UnsupportedVersion",
        good[:6] + b"\x09" + good[7:]: "CorruptPayload",   # predictor_log2 out of 10..16
        good[:7] + b"\x09" + good[8:]: "UnsupportedDType",
        good[:5] + b"\x04" + good[6:]: "CorruptPayload",   # unknown flag
    }
    for b, kind in bad_cases.items():
        try:
            qb.stream_info(b)
            raise AssertionError(f"accepted {b!r}")
        except qb.Error as e:
            assert e.kind == kind, (b, e.kind)


def test_null_arguments_return_null_code(qb):
    L = qb.lib
    n = ctypes.c_size_t()
    assert L.quoin_compress(None, 0, None, 0, ctypes.byref(n)) == -1
    assert L.quoin_decompress(None, 0, None, 0, ctypes.byref(n)) == -1
    assert L.quoin_decompressed_value_count(None, 0) == -1
    assert L.quoin_typed_compress(3, 4, None, None, None, 0) == 0
    assert L.quoin_typed_decompress(3, 4, None, 0, None, None) == -1
