"""The Arrow adapter (reference src/arrow.rs) through the Arrow C Data Interface:
quoin_b200_compress_arrow must write the same stream as the typed compress of
the array's values and validity (its offset honoured, a sliced bitmap
re-packed), quoin_b200_decompress_arrow must give back an equal Arrow array of
the stream's type, and unsupported types must be refused with
UnsupportedArrowType (arrow.rs tests: primitive_with_nulls_roundtrip,
decimal128/256_roundtrip, sliced_array_roundtrip, unsupported_type_errors).
"""
import ctypes
import decimal

import numpy as np
import pytest

pa = pytest.importorskip("pyarrow")

pytestmark = pytest.mark.gpu

F64, I64, U64, I32, U32, F32, DEC128, DEC256 = range(8)
ERR_UNSUPPORTED_ARROW_TYPE = -22


class ArrowSchema(ctypes.Structure):
    pass


ArrowSchema._fields_ = [("format", ctypes.c_char_p), ("name", ctypes.c_char_p), ("metadata", ctypes.c_char_p),
                        ("flags", ctypes.c_int64), ("n_children", ctypes.c_int64), ("children", ctypes.c_void_p),
                        ("dictionary", ctypes.c_void_p), ("release", ctypes.c_void_p),
                        ("private_data", ctypes.c_void_p)]


class ArrowArray(ctypes.Structure):
    _fields_ = [("length", ctypes.c_int64), ("null_count", ctypes.c_int64), ("offset", ctypes.c_int64),
                ("n_buffers", ctypes.c_int64), ("n_children", ctypes.c_int64),
                ("buffers", ctypes.POINTER(ctypes.c_void_p)), ("children", ctypes.c_void_p),
                ("dictionary", ctypes.c_void_p), ("release", ctypes.c_void_p), ("private_data", ctypes.c_void_p)]


@pytest.fixture(scope="module")
def arrow_api(qb):
    L = qb.lib
    P, S = ctypes.c_void_p, ctypes.c_size_t
    L.quoin_b200_compress_arrow.argtypes = [P, ctypes.POINTER(ArrowSchema), ctypes.POINTER(ArrowArray),
                                            ctypes.POINTER(qb._QuoinConfig), P, S, ctypes.POINTER(S)]
    L.quoin_b200_compress_arrow.restype = ctypes.c_int
    L.quoin_b200_decompress_arrow.argtypes = [P, ctypes.c_char_p, S, ctypes.POINTER(ArrowSchema),
                                              ctypes.POINTER(ArrowArray)]
    L.quoin_b200_decompress_arrow.restype = ctypes.c_int
    return L


def compress_arrow(qb, L, arr, cfg):
    sch, car = ArrowSchema(), ArrowArray()
    arr._export_to_c(ctypes.addressof(car), ctypes.addressof(sch))
    try:
        cap = 32 * len(arr) + 4096
        out = (ctypes.c_uint8 * cap)()
        olen = ctypes.c_size_t()
        c = qb._cfg(cfg)
        rc = L.quoin_b200_compress_arrow(None, ctypes.byref(sch), ctypes.byref(car), ctypes.byref(c), out, cap,
                                         ctypes.byref(olen))
        return rc, bytes(out[: olen.value]) if rc == 0 else b""
    finally:  # hand the exported structs back to pyarrow, which releases them
        pa.Array._import_from_c(ctypes.addressof(car), ctypes.addressof(sch))


def decompress_arrow(L, stream):
    sch, car = ArrowSchema(), ArrowArray()
    rc = L.quoin_b200_decompress_arrow(None, stream, len(stream), ctypes.byref(sch), ctypes.byref(car))
    assert rc == 0
    return pa.Array._import_from_c(ctypes.addressof(car), ctypes.addressof(sch))


def typed_parts(arr, width):
    """(native value bytes of the array's slice, its validity bitmap or None)."""
    buf = arr.buffers()[1]
    if buf is None or len(arr) == 0:
        return np.zeros(0, np.uint8), None
    raw = np.frombuffer(buf, np.uint8)[arr.offset * width:(arr.offset + len(arr)) * width].copy()
    bm = None
    if arr.null_count:
        valid = np.array([v is not None for v in arr.to_pylist()], bool)
        bm = np.packbits(valid, bitorder="little")
    return raw, bm


def cases():
    rng = np.random.default_rng(4)
    n = 30000
    nulls = rng.random(n) < 0.1
    f64 = pa.array(np.floor(rng.random(n) * 1e6 + 0.5) / 100.0, mask=nulls)
    i64 = pa.array((1_700_000_000_000 + np.cumsum(rng.poisson(50, n))).astype(np.int64), mask=nulls)
    dec = [None if m else decimal.Decimal(int(x)).scaleb(-4) for x, m in zip(rng.integers(-10**12, 10**12, 5000),
                                                                              nulls[:5000])]
    d256 = [None if m else decimal.Decimal(int(x) * 10**25 + 7).scaleb(-2)
            for x, m in zip(rng.integers(-10**9, 10**9, 3000), nulls[:3000])]
    return [
        ("f64_nulls", f64, F64, 8, 0, 0),
        ("i64_nulls", i64, I64, 8, 0, 0),
        ("u64", pa.array(rng.integers(0, 2**63, n, dtype=np.uint64)), U64, 8, 0, 0),
        ("i32_nulls", pa.array(rng.integers(-500, 500, n).astype(np.int32), mask=nulls), I32, 4, 0, 0),
        ("u32", pa.array(np.arange(n, dtype=np.uint32) * 3), U32, 4, 0, 0),
        ("f32_nulls", pa.array(rng.normal(0, 1, n).astype(np.float32), mask=nulls), F32, 4, 0, 0),
        ("dec128_nulls", pa.array(dec, type=pa.decimal128(18, 4)), DEC128, 16, 4, 18),
        ("dec256_nulls", pa.array(d256, type=pa.decimal256(40, 2)), DEC256, 32, 2, 40),
        ("i64_sliced_3", i64.slice(3, 20000), I64, 8, 0, 0),
        ("f64_sliced_16", f64.slice(16, 9999), F64, 8, 0, 0),
        ("empty", pa.array(np.zeros(0, np.int64)), I64, 8, 0, 0),
    ]


@pytest.mark.parametrize("case", cases(), ids=lambda c: c[0])
def test_arrow_matches_typed_path_and_roundtrips(qb, arrow_api, case):
    name, arr, dt, w, scale, precision = case
    cfg = qb.Config(level=qb.Level.FAST)
    rc, stream = compress_arrow(qb, arrow_api, arr, cfg)
    assert rc == 0
    raw, bm = typed_parts(arr, w)
    want = qb.compress_column(raw, bm, cfg, dtype=dt, scale=scale, precision=precision)
    assert stream == want
    back = decompress_arrow(arrow_api, stream)
    assert back.type == arr.type
    assert back.equals(arr), name
    back2 = decompress_arrow(arrow_api, stream)  # a second array from the same stream
    assert back2.equals(arr)


@pytest.mark.parametrize("arr", [pa.array([True, False, None]), pa.array(["a", "b"]),
                                 pa.array([1, 2], type=pa.int16()), pa.array([1, 2], type=pa.date32())],
                         ids=["bool", "string", "int16", "date32"])
def test_arrow_unsupported_types_are_refused(qb, arrow_api, arr):
    rc, _ = compress_arrow(qb, arrow_api, arr, qb.Config())
    assert rc == ERR_UNSUPPORTED_ARROW_TYPE
