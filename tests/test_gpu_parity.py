"""GPU parity tests: the CUDA competition/emission must produce the oracle's
exact bytes, and the CUDA block decoder must reproduce the oracle's decode of
every stream (values bit for bit, validity bitmaps, error vs success).

All calls go through the C ABI of libquoin_b200.so (the product); the oracle
(oracle/) is only the checker.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import bitmap_from_bools, lcg1_seq, lcg_seq
from quoin_b200 import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
F64, I64, U64, I32, U32, F32, DEC128, DEC256 = range(8)
NW = {F64: 8, I64: 8, U64: 8, I32: 4, U32: 4, F32: 4, DEC128: 16, DEC256: 32}


def expected_values(vals, dt, bm):
    """Input bytes with null slots zeroed (the decoder's null fill)."""
    raw = np.ascontiguousarray(vals).view(np.uint8).reshape(-1, NW[dt]).copy()
    if bm is not None:
        n = raw.shape[0]
        valid = np.unpackbits(np.asarray(bm, np.uint8), bitorder="little")[:n].astype(bool)
        raw[~valid] = 0
    return raw.tobytes()


def gpu_compress(qb, vals, dt, bm=None, level=1, block_size=None, scale=0, precision=0):
    return qb.compress_column(vals, bm, qb.Config(level=qb.Level(level), block_size=block_size), dtype=dt,
                              scale=scale, precision=precision)


def dec_bytes(d):
    return np.ascontiguousarray(d.values).view(np.uint8).tobytes()


# ---------------------------------------------------------------------------
# Golden fixtures (tests/golden/make_golden.py)
# ---------------------------------------------------------------------------
def golden_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_golden_streams(qb, case):
    dt = case["dtype"]
    raw = np.fromfile(os.path.join(GOLDEN, case["name"] + ".in"), dtype=np.uint8)
    bm = np.fromfile(os.path.join(GOLDEN, case["name"] + ".valid"), dtype=np.uint8) if case["validity"] else None
    for lvl, fn in case["streams"].items():
        want = open(os.path.join(GOLDEN, fn), "rb").read()
        got = gpu_compress(qb, raw, dt, bm, int(lvl), case["block_size"], case["scale"], case["precision"])
        assert got == want, f"{case['name']} L{lvl}: GPU stream differs from golden"
        d = qb.decompress_column(want)
        assert dec_bytes(d) == expected_values(raw, dt, bm)
        if bm is not None:
            assert d.validity == bm.tobytes()[: (case["n"] + 7) // 8]
        if dt in (DEC128, DEC256):
            assert (d.scale, d.precision) == (case["scale"], case["precision"])


# ---------------------------------------------------------------------------
# Live-oracle parity over shapes
# ---------------------------------------------------------------------------
def shape_cases():
    rng = np.random.default_rng(1234)
    c = [
        ("one_i64", np.array([42], np.int64), I64, None),
        ("edges_i64", np.array([-1, 0, 1, -2**63, 2**63 - 1], np.int64), I64, None),
        ("two_f64", np.array([1.0, 2.0]), F64, None),
        ("negramp_i64", np.arange(-5000, 0, dtype=np.int64), I64, None),
        ("wide_u64", lcg_seq(7, 40000), U64, None),
        ("i32_edges", np.array([-2**31, -1, 0, 1, 2**31 - 1], np.int32), I32, None),
        ("u32_ids", (100_000 + np.arange(8000) % 300).astype(np.uint32), U32, None),
        ("runs_i64", np.repeat((1_000_000 + np.arange(500) * 7).astype(np.int64), 200), I64, None),
        ("midcard_u64", (500_000_000 + (lcg1_seq(5, 40000) >> np.uint64(53)) % 2000).astype(np.uint64), U64, None),
        ("highcard_44bit", (lcg_seq(11, 70000) >> np.uint64(20)).astype(np.uint64), U64, None),
        ("dict_grown_200k", (lcg_seq(9, 200000) >> np.uint64(59)).astype(np.int64), I64, None),
        ("pairs_repeat", np.repeat(lcg_seq(21, 40000), 2), U64, None),
        ("ramp_f64", np.arange(10000) * 0.5, F64, None),
        ("sine_f64", np.sin(np.arange(70000) * 1e-4), F64, None),
        ("random_f64", lcg_seq(0x123456789ABCDEF0, 65536).view(np.float64), F64, None),
        ("nan_block", np.full(1000, np.nan), F64, None),
        ("inf_alt", np.where(np.arange(5000) % 2 == 0, np.inf, -np.inf), F64, None),
        ("expbits", (lcg_seq(7, 5000) & np.uint64(0xFFF0000000000000)).view(np.float64), F64, None),
        ("sqrt_f64", np.sqrt(np.arange(70000, dtype=np.float64)), F64, None),
        ("f32_smooth", np.arange(8192, dtype=np.float32) * np.float32(0.01) + np.float32(5.0), F32, None),
        ("f32_special", np.array([0x00000001, 0x80000000, 0x7F800000, 0xFF800000, 0x0DA24260], np.uint32)
         .view(np.float32), F32, None),
        ("allnull_u64", np.full(1000, 9, np.uint64), U64, bitmap_from_bools(np.zeros(1000, bool))),
        ("allvalid_i64", np.full(1000, 5, np.int64), I64, bitmap_from_bools(np.ones(1000, bool))),
        ("odd_nulls_i32", np.array([10, 20, 30, 40, 50, 60, 70], np.int32), I32,
         bitmap_from_bools([1, 0, 1, 1, 0, 1, 1])),
        ("lead_trail_nulls", np.arange(3000, dtype=np.int64), I64,
         bitmap_from_bools([100 <= i < 2900 for i in range(3000)])),
    ]
    # Dictionaries beyond the shared-memory hash (more than 1536 distinct
    # values): the scratch hash, radix sort and rank table.
    pool = lcg_seq(31, 3000) >> np.uint64(8)  # 56-bit: FoR compresses a little, so DICT is tried
    c.append(("dict_scratch_wide_u64", pool[(lcg1_seq(32, 40000) >> np.uint64(40)) % 1800], U64, None))
    pool_max = pool.copy()
    pool_max[17] = np.uint64(2**64 - 1)
    c.append(("dict_scratch_with_max", pool_max[(lcg1_seq(33, 70000) >> np.uint64(40)) % 1800], U64, None))
    c.append(("dict_scratch_i32", (pool[(lcg1_seq(34, 50000) >> np.uint64(40)) % 2500] >> np.uint64(32))
              .astype(np.uint32).view(np.int32), I32, None))
    c.append(("dict_scratch_big", (lcg_seq(35, 17000) >> np.uint64(8))[(lcg1_seq(36, 32768) >> np.uint64(40)) % 17000],
              U64, None))
    p17 = lcg_seq(38, 17500) >> np.uint64(8)  # 17500 distinct > 32768/2+1, bucket lower bound below it
    c.append(("dict_scratch_bail", np.concatenate([p17, p17[:32768 - 17500]])[np.argsort(lcg_seq(39, 32768))],
              U64, None))
    c.append(("dict_scratch_grown", np.repeat(pool[(lcg1_seq(37, 60000) >> np.uint64(40)) % 2800], 3)[:170000],
              U64, None))
    # Nullable columns of every decode shape: values are scattered through the
    # bitmap straight from the block decoder.
    vb2 = rng.random(150000) > 0.2
    cats = (lcg_seq(41, 64) >> np.uint64(33)).astype(np.int64) - (1 << 30)
    c.append(("nullable_i32_rle", np.repeat(cats[rng.integers(0, 64, 10000)], 15)[:150000].astype(np.int32), I32,
              bitmap_from_bools(vb2)))
    c.append(("nullable_u64_xorz", synth.runs_u64(150000, np.random.default_rng(5)), U64, bitmap_from_bools(vb2)))
    c.append(("nullable_f32", (np.round(rng.normal(25, 5, 150000) * 10) / 10).astype(np.float32), F32,
              bitmap_from_bools(vb2)))
    c.append(("nullable_f64_walk", 20.0 + np.cumsum(rng.normal(0, 1e-3, 150000)), F64, bitmap_from_bools(vb2)))
    u12 = rng.random(150000) + 1.0
    u12[rng.integers(0, 150000, 1500)] = rng.random(1500) * 1e6
    c.append(("nullable_f64_alprd", u12, F64, bitmap_from_bools(vb2)))
    c.append(("nullable_f64_alp", np.floor(rng.random(150000) * 1_000_000 + 0.5) / 100.0, F64, bitmap_from_bools(vb2)))
    c.append(("nullable_dict_scratch", pool[(lcg1_seq(43, 150000) >> np.uint64(40)) % 2500], U64,
              bitmap_from_bools(vb2)))
    vb = rng.random(300000) > 0.1
    c.append(("nullable_ts_300k", (np.cumsum(1_000_000 + rng.poisson(5000, 300000)) + 1_700_000_000_000_000_000)
              .astype(np.int64), I64, bitmap_from_bools(vb)))
    return c


@pytest.mark.parametrize("level", [0, 1])
@pytest.mark.parametrize("case", shape_cases(), ids=lambda c: c[0])
def test_shapes_match_oracle(qb, oracle, case, level):
    name, vals, dt, bm = case
    want = oracle.compress_column(vals, dt, bm, level=level)
    got = gpu_compress(qb, vals, dt, bm, level)
    assert got == want
    d = qb.decompress_column(want)
    od = oracle.decompress_column(want)
    assert dec_bytes(d) == np.ascontiguousarray(od[1]).view(np.uint8).tobytes()
    assert (d.validity is None) == (od[2] is None)
    if od[2] is not None:
        assert d.validity == od[2].tobytes()


@pytest.mark.parametrize("bs", [1, 7, 64, 1000, 8192, 1 << 30])
def test_fixed_block_sizes(qb, oracle, bs):
    vals = (1000 + np.arange(40_000) % 777).astype(np.int64)
    assert gpu_compress(qb, vals, I64, block_size=bs) == oracle.compress_column(vals, I64, block_size=bs)


@pytest.mark.parametrize("bs", [1000, 2048, 5000])
def test_fixed_block_sizes_with_nulls(qb, oracle, bs):
    """Block sizes that are and are not multiples of 1024, with a bitmap."""
    rng = np.random.default_rng(bs)
    vals = (1_000_000 + np.cumsum(rng.poisson(40, 30_000))).astype(np.int64)
    bm = bitmap_from_bools(rng.random(30_000) > 0.3)
    want = oracle.compress_column(vals, I64, bm, block_size=bs)
    assert gpu_compress(qb, vals, I64, bm, block_size=bs) == want
    d = qb.decompress_column(want)
    assert dec_bytes(d) == expected_values(vals, I64, bm)
    vals32 = (vals % 1000).astype(np.int32)
    want32 = oracle.compress_column(vals32, I32, bm, block_size=bs)
    assert gpu_compress(qb, vals32, I32, bm, block_size=bs) == want32
    assert dec_bytes(qb.decompress_column(want32)) == expected_values(vals32, I32, bm)


def test_predictor_log2_is_recorded(qb, oracle):
    vals = np.arange(100, dtype=np.int64)
    for p in (3, 10, 13, 16, 40):
        got = qb.compress_column(vals, None, qb.Config(predictor_log2=p))
        assert got == oracle.compress_column(vals, I64, predictor_log2=p)


# ---------------------------------------------------------------------------
# Benchmark-shaped columns (seeded synthetic stand-ins), 1M values
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("kind", ["prices", "integer", "float"])
def test_benchmark_columns_match_oracle(qb, oracle, kind):
    from quoin_b200 import synth
    n = 1 << 20
    for name, dt, vals, bm in synth.benchmark_columns(kind, n):
        sc, pr = (4, 18) if dt == DEC128 else (0, 0)
        want = oracle.compress_column(vals, dt, bm, level=1, scale=sc, precision=pr, threads=8)
        got = gpu_compress(qb, vals, dt, bm, 1, scale=sc, precision=pr)
        assert got == want, name
        assert dec_bytes(qb.decompress_column(got)) == expected_values(vals, dt, bm), name


# ---------------------------------------------------------------------------
# Decode of a stream the GPU encoder never produces: Balanced level, with
# rANS-coded ALP-RD codes (tests/test_entropy_decode.py covers every tag).
# ---------------------------------------------------------------------------
def test_balanced_stream_decodes(qb, oracle):
    vals = np.sin(np.arange(40000) * 0.01)
    s = oracle.compress_column(vals, F64, level=2)
    assert dec_bytes(qb.decompress_column(s)) == vals.view(np.uint8).tobytes()


# ---------------------------------------------------------------------------
# Robustness (tests/robustness.rs): malformed streams never fault the GPU and
# agree with the oracle on success vs error (and on values when successful).
# ---------------------------------------------------------------------------
def test_mutated_streams_agree_with_oracle(qb, oracle):
    rng = np.random.default_rng(0x13579BDF)
    seeds = [oracle.compress_column(d, dt, level=1) for d, dt in (
        (np.arange(4000) * 0.5, F64), (np.sin(np.arange(4000) * 0.01), F64),
        ((np.arange(4000) & 15).astype(np.float64), F64), (lcg_seq(1, 4000).view(np.float64), F64),
        (np.full(4000, 42.0), F64), ((np.arange(4000) % 1000) / 100.0, F64),
        ((1000 + np.arange(4000) % 300).astype(np.int64), I64),
        (np.repeat(np.arange(40, dtype=np.int64), 100), I64))]
    agree = 0
    for it in range(1500):
        b = bytearray(seeds[rng.integers(len(seeds))])
        for _ in range(1 + rng.integers(4)):
            if not b:
                break
            op = rng.integers(3)
            i = int(rng.integers(len(b)))
            if op == 0:
                b[i] = int(rng.integers(256))
            elif op == 1:
                b[i] ^= 1 << int(rng.integers(8))
            else:
                del b[i:]
        b = bytes(b)
        try:
            od = oracle.decompress_column(b)
            ook = True
        except oracle.OracleError:
            ook = False
        try:
            d = qb.decompress_column(b)
            gok = True
        except qb.Error:
            gok = False
        assert gok == ook, f"iteration {it}: gpu ok={gok} oracle ok={ook}"
        if gok:
            assert dec_bytes(d) == np.ascontiguousarray(od[1]).view(np.uint8).tobytes()
        agree += 1
    assert agree == 1500


def test_random_bytes_never_fault(qb):
    rng = np.random.default_rng(0xABCDEF01)
    for _ in range(300):
        b = rng.integers(0, 256, rng.integers(0, 80), dtype=np.uint8).tobytes()
        try:
            qb.decompress_column(b)
        except qb.Error:
            pass
    # the library is still healthy afterwards
    v = np.arange(1000, dtype=np.int64) * 3
    assert dec_bytes(qb.decompress_column(qb.compress_column(v))) == v.view(np.uint8).tobytes()


# ---------------------------------------------------------------------------
# The reference C ABI (behaviours of capi/test/roundtrip.c:102-222)
# ---------------------------------------------------------------------------
def _abi_roundtrip_f64(L, data, ctx=None):
    n = data.size
    cap = L.quoin_compress_bound(n)
    packed = np.zeros(cap, np.uint8)
    clen = ctypes.c_size_t()
    p = data.ctypes.data if n else np.zeros(1).ctypes.data
    rc = (L.quoin_compress_ctx(ctx, p, n, packed.ctypes.data, cap, ctypes.byref(clen)) if ctx
          else L.quoin_compress(p, n, packed.ctypes.data, cap, ctypes.byref(clen)))
    assert rc == 0
    assert L.quoin_decompressed_value_count(packed.ctypes.data, clen.value) == n
    out = np.zeros(n + 1)
    got = ctypes.c_size_t()
    rc = (L.quoin_decompress_ctx(ctx, packed.ctypes.data, clen.value, out.ctypes.data, n, ctypes.byref(got)) if ctx
          else L.quoin_decompress(packed.ctypes.data, clen.value, out.ctypes.data, n, ctypes.byref(got)))
    assert rc == 0 and got.value == n
    assert out[:n].view(np.uint64).tobytes() == data.view(np.uint64).tobytes()
    return clen.value


def test_capi_f64_roundtrips(qb):
    L = qb.lib
    N = 100_000
    ramp = np.arange(N) * 0.5
    cents = (np.arange(N) % 1000) / 100.0
    sine = np.sin(np.arange(N) * 1e-4)
    special = np.array([0.0, -0.0, np.nan, np.inf, -np.inf, 1e308, 1e-308, 3.14159])
    for d in (ramp, cents, sine, special, np.zeros(0)):
        _abi_roundtrip_f64(L, d)
    ctx = L.quoin_ctx_create(4)
    assert ctx
    _abi_roundtrip_f64(L, ramp, ctx)
    _abi_roundtrip_f64(L, cents, ctx)
    L.quoin_ctx_free(ctx)
    L.quoin_ctx_free(None)


def test_capi_errors(qb):
    L = qb.lib
    junk = np.full(32, 0xAB, np.uint8)
    tmp = np.zeros(4)
    got = ctypes.c_size_t()
    assert L.quoin_decompress(junk.ctypes.data, 32, tmp.ctypes.data, 4, ctypes.byref(got)) == -3
    out = np.zeros(4, np.int64)
    assert L.quoin_typed_decompress(4, 4, junk.ctypes.data, 32, out.ctypes.data, None) == -3
    # buffer too small: needed size reported
    data = np.arange(1000) * 0.25
    small = np.zeros(8, np.uint8)
    n = ctypes.c_size_t()
    assert L.quoin_compress(data.ctypes.data, 1000, small.ctypes.data, 8, ctypes.byref(n)) == -2 and n.value > 8
    packed = np.zeros(L.quoin_compress_bound(1000), np.uint8)
    assert L.quoin_compress(data.ctypes.data, 1000, packed.ctypes.data, packed.size, ctypes.byref(n)) == 0
    few = np.zeros(10)
    assert L.quoin_decompress(packed.ctypes.data, n.value, few.ctypes.data, 10, ctypes.byref(got)) == -2
    assert got.value == 1000
    # a non-f64 stream through quoin_decompress -> CORRUPT (DTypeMismatch)
    s = qb.compress_column(np.arange(10, dtype=np.int64))
    sb = np.frombuffer(s, np.uint8)
    assert L.quoin_decompress(sb.ctypes.data, len(s), few.ctypes.data, 10, ctypes.byref(got)) == -3


def _typed_rt(L, dtype, vals, validity=None):
    n = vals.shape[0]
    cap = L.quoin_typed_compress_bound(dtype, n)
    packed = np.zeros(max(cap, 1), np.uint8)
    vb = None if validity is None else validity.ctypes.data
    clen = L.quoin_typed_compress(dtype, n, vals.ctypes.data if n else packed.ctypes.data, vb, packed.ctypes.data, cap)
    assert clen > 0
    w = L.quoin_dtype_width(dtype)
    out = np.zeros(n * w + 8, np.uint8)
    vout = np.zeros((n + 7) // 8 + 1, np.uint8)
    rc = L.quoin_typed_decompress(dtype, n, packed.ctypes.data, clen, out.ctypes.data, vout.ctypes.data)
    assert rc == 0
    return packed[:clen].tobytes(), out[: n * w].tobytes(), vout[: (n + 7) // 8].tobytes()


def test_capi_typed(qb):
    L = qb.lib
    M = 50_000
    i = np.arange(M)
    for dtype, vals in ((4, (1_000_000 + i % 5000).astype(np.int64)), (2, (-100 + i % 200).astype(np.int16)),
                        (5, (i % 7).astype(np.uint8)), (9, (np.sin(i * 1e-4) * 100).astype(np.float32)),
                        (0, (i % 2).astype(np.uint8)), (1, (i % 100 - 50).astype(np.int8)),
                        (6, (i % 60000).astype(np.uint16)), (3, (i % 99999 - 50000).astype(np.int32)),
                        (7, (i * 3).astype(np.uint32)), (8, (i * 7).astype(np.uint64)), (10, i * 0.125)):
        _, out, vout = _typed_rt(L, dtype, vals)
        assert out == vals.tobytes(), dtype
        assert vout == bitmap_from_bools(np.ones(M, bool)).tobytes()
    _, out, _ = _typed_rt(L, 4, np.zeros(0, np.int64))
    # nulls: every 3rd value null, null slots 0 in the input
    NN = 1000
    valid = np.array([k % 3 != 0 for k in range(NN)])
    vals = np.where(valid, 7000 + np.arange(NN) % 50, 0).astype(np.int32)
    bm = bitmap_from_bools(valid)
    _, out, vout = _typed_rt(L, 3, vals, bm)
    assert out == vals.tobytes() and vout == bm.tobytes()


def test_capi_typed_decimals(qb):
    L = qb.lib
    M = 50_000
    i = np.arange(M)
    d64 = (100_000 + i % 5000).astype(np.int64)
    d128 = np.zeros((M, 2), np.int64)
    d128[:, 0] = 100_000_000 + i % 10000
    d256 = np.zeros((M, 4), np.int64)
    d256[:, 0] = 1_000_000 + i % 5000
    d32 = (-500 + i % 1000).astype(np.int32)
    for dtype, vals, sc, pr in ((12, d64, 4, 18), (13, d128, 8, 38), (14, d256, 8, 50), (11, d32, 2, 9)):
        cap = L.quoin_typed_compress_bound(dtype, M)
        packed = np.zeros(cap, np.uint8)
        clen = L.quoin_typed_compress_decimal(dtype, M, vals.ctypes.data, None, sc, pr, packed.ctypes.data, cap)
        assert clen > 0
        out = np.zeros(vals.nbytes + 8, np.uint8)
        assert L.quoin_typed_decompress(dtype, M, packed.ctypes.data, clen, out.ctypes.data, None) == 0
        assert out[: vals.nbytes].tobytes() == vals.tobytes()
        info = qb.stream_info(packed[:clen].tobytes())
        assert info[3:] == (sc, pr)


def test_capi_unaligned_buffers(qb):
    L = qb.lib
    M = 50_000
    ibuf = np.zeros(M * 8 + 1, np.uint8)
    obuf = np.zeros(M * 8 + 1, np.uint8)
    v = (5000 + np.arange(M) % 137).astype(np.int64)
    ibuf[1:] = v.view(np.uint8)
    cap = L.quoin_typed_compress_bound(4, M)
    packed = np.zeros(cap, np.uint8)
    clen = L.quoin_typed_compress(4, M, ibuf.ctypes.data + 1, None, packed.ctypes.data, cap)
    assert clen > 0
    assert L.quoin_typed_decompress(4, M, packed.ctypes.data, clen, obuf.ctypes.data + 1, None) == 0
    assert obuf[1:].tobytes() == ibuf[1:].tobytes()


def test_mode_win_counts(qb):
    qb.reset_mode_win_counts()
    qb.compress_column(np.full(5000, 7, np.int64))
    qb.compress_column(np.arange(5000, dtype=np.int64))
    w = qb.mode_win_counts()
    assert w[1] == 1 and w[2] == 1 and w.sum() == 2


def test_device_api_and_index(qb):
    """Device-resident compress and the reusable decode index."""
    torch = pytest.importorskip("torch")
    L = qb.lib
    P = ctypes.c_void_p
    n = 300_000
    v = (np.cumsum(1000 + np.arange(n) % 17)).astype(np.int64)
    bm = bitmap_from_bools(np.arange(n) % 10 != 3)
    dv = torch.from_numpy(v.view(np.uint8).copy()).cuda()
    db = torch.from_numpy(bm.copy()).cuda()
    cap = qb._stream_bound(I64, n, True)
    dd = torch.empty(cap, dtype=torch.uint8, device="cuda")
    olen = ctypes.c_size_t()
    cfg = qb._QuoinConfig(1, 0, 16)
    rc = L.quoin_b200_compress_column_device(None, I64, n, P(dv.data_ptr()), P(db.data_ptr()), 0, 0,
                                             ctypes.byref(cfg), P(dd.data_ptr()), cap, ctypes.byref(olen), None)
    assert rc == 0
    s = dd[: olen.value].cpu().numpy().tobytes()
    assert s == qb.compress_column(v, bm)
    idx = P()
    assert L.quoin_b200_index_create(None, s, len(s), ctypes.byref(idx)) == 0
    out = torch.empty(n * 8, dtype=torch.uint8, device="cuda")
    vout = torch.empty((n + 7) // 8, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        assert L.quoin_b200_decompress_indexed_device(None, idx, P(dd.data_ptr()), P(out.data_ptr()),
                                                      P(vout.data_ptr()), None) == 0
        assert out.cpu().numpy().tobytes() == expected_values(v, I64, bm)
        assert vout.cpu().numpy().tobytes() == bm.tobytes()
    L.quoin_b200_index_free(idx)
    # too-small device destination reports the needed size
    rc = L.quoin_b200_compress_column_device(None, I64, n, P(dv.data_ptr()), P(db.data_ptr()), 0, 0,
                                             ctypes.byref(cfg), P(dd.data_ptr()), 100, ctypes.byref(olen), None)
    assert rc == -2 and olen.value > 100
