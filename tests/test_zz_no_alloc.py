"""quoin_b200_decompress_device_noalloc: the allocation-free device decode.

Each stream is decoded twice in a row through the C ABI entry point and
compared with the context-based device decode (quoin_b200_decompress_indexed_
device) of the same stream and with the input values.  The file name sorts
last so the tests also run after every other GPU test in one process.
"""
import ctypes

import numpy as np
import pytest

from conftest import bitmap_from_bools, lcg1_seq, lcg_seq

pytestmark = pytest.mark.gpu

F64, I64, U64, I32 = 0, 1, 2, 3
ERR_BUFFER_TOO_SMALL, ERR_BAD_MAGIC, ERR_TRUNCATED, ERR_NOALLOC_LIMIT = -2, -10, -12, -21
MAX_VALUES = 262144


@pytest.fixture(scope="module")
def api(qb):
    import torch
    L = qb.lib
    P = ctypes.c_void_p
    L.quoin_b200_decompress_device_noalloc.argtypes = [P, ctypes.c_size_t, P, ctypes.c_size_t,
                                                       ctypes.POINTER(ctypes.c_uint64), P]
    L.quoin_b200_decompress_device_noalloc.restype = ctypes.c_int
    torch.cuda.set_device(0)
    return L, torch


def noalloc(api, d_src, n_src, d_out, cap):
    L, torch = api
    n = ctypes.c_uint64(123)
    rc = L.quoin_b200_decompress_device_noalloc(ctypes.c_void_p(d_src.data_ptr()), n_src,
                                                ctypes.c_void_p(d_out.data_ptr()), cap, ctypes.byref(n),
                                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, n.value


def indexed(qb, api, stream, d_src, n):
    L, torch = api
    ctx = ctypes.c_void_p(L.quoin_ctx_create(0))
    idx = ctypes.c_void_p()
    assert L.quoin_b200_index_create(ctx, stream, len(stream), ctypes.byref(idx)) == 0
    d_out = torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")
    rc = L.quoin_b200_decompress_indexed_device(ctx, idx, ctypes.c_void_p(d_src.data_ptr()),
                                                ctypes.c_void_p(d_out.data_ptr()), None,
                                                ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    L.quoin_b200_index_free(idx)
    L.quoin_ctx_free(ctx)
    assert rc == 0
    return d_out[:n].cpu().numpy().tobytes()


def cases():
    rng = np.random.default_rng(99)
    pool = lcg_seq(31, 17000) >> np.uint64(8)
    return [
        ("timestamps_delta", (1_700_000_000_000 + np.cumsum(1000 + rng.poisson(50, 100_000))).astype(np.int64),
         I64, None),
        ("runs_for_xorz", (1 << 40) + (lcg1_seq(3, 200_000) & np.repeat((np.uint64(1) << (np.arange(196) % 38
                                                                                           + 3).astype(np.uint64))
                                                                          - np.uint64(1), 1024)[:200_000]),
         U64, None),
        ("two_big_dicts", pool[(lcg1_seq(36, 65536) >> np.uint64(40)) % 14000], U64, None),
        ("categories_rle", np.repeat(lcg_seq(5, 900) >> np.uint64(50), 200).astype(np.int64)[:150_000], I64, None),
        ("prices_alp", np.floor(rng.random(MAX_VALUES) * 1_000_000 + 0.5) / 100.0, F64, None),
        ("small_blocks", (np.arange(50_000) % 977).astype(np.int64), I64, 256),
        ("empty", np.zeros(0, np.int64), I64, None),
    ]


@pytest.mark.parametrize("case", cases(), ids=lambda c: c[0])
def test_noalloc_matches_device_decode(qb, api, case):
    _, torch = api
    name, vals, dt, bs = case
    stream = qb.compress_column(vals, None, qb.Config(level=qb.Level.FAST, block_size=bs), dtype=dt)
    src = np.frombuffer(stream, np.uint8).copy()
    d_src = torch.from_numpy(src).cuda()
    n = len(vals)
    want = np.ascontiguousarray(vals).view(np.uint8).tobytes()
    ref = indexed(qb, api, stream, d_src, n) if n else b""
    assert ref == want
    outs = []
    for _ in range(2):  # two calls in a row
        d_out = torch.full((max(n, 1),), -1, dtype=torch.int64, device="cuda")
        rc, got_n = noalloc(api, d_src, len(stream), d_out, n)
        assert rc == 0 and got_n == n
        outs.append(d_out[:n].cpu().numpy().tobytes())
    assert outs[0] == want and outs[1] == want


def test_noalloc_rejects_streams_outside_its_limits(qb, api):
    _, torch = api
    d_out = torch.zeros(MAX_VALUES + 8, dtype=torch.int64, device="cuda")

    def run(stream, cap):
        d_src = torch.from_numpy(np.frombuffer(stream, np.uint8).copy()).cuda()
        return noalloc(api, d_src, len(stream), d_out, cap)[0]

    big = qb.compress_column(np.arange(MAX_VALUES + 1, dtype=np.int64), None, qb.Config(), dtype=I64)
    assert run(big, MAX_VALUES + 8) == ERR_NOALLOC_LIMIT
    nullable = qb.compress_column(np.arange(100, dtype=np.int64), bitmap_from_bools(np.arange(100) % 3 > 0),
                                  qb.Config(), dtype=I64)
    assert run(nullable, 100) == ERR_NOALLOC_LIMIT
    narrow = qb.compress_column(np.arange(100, dtype=np.int32), None, qb.Config(), dtype=I32)
    assert run(narrow, 100) == ERR_NOALLOC_LIMIT
    many_frames = qb.compress_column(np.arange(300, dtype=np.int64), None, qb.Config(block_size=1), dtype=I64)
    assert run(many_frames, 300) == ERR_NOALLOC_LIMIT
    ok = qb.compress_column(np.arange(1000, dtype=np.int64) * 3, None, qb.Config(), dtype=I64)
    assert run(ok, 999) == ERR_BUFFER_TOO_SMALL
    d_ok = torch.from_numpy(np.frombuffer(ok, np.uint8).copy()).cuda()
    assert noalloc(api, d_ok, len(ok), d_out, 999) == (ERR_BUFFER_TOO_SMALL, 1000)  # the count it needs
    assert run(b"XCR1" + ok[4:], 1000) == ERR_BAD_MAGIC
    # not a stream, with the decimal-container bit set: the magic is checked first
    assert run(b"ABCD\x02\x02" + ok[6:], 1000) == ERR_BAD_MAGIC
    assert run(ok[:20], 1000) == ERR_TRUNCATED
    # the arena is reset by every call: a good stream decodes after the errors
    d_src = torch.from_numpy(np.frombuffer(ok, np.uint8).copy()).cuda()
    rc, n = noalloc(api, d_src, len(ok), d_out, 1000)
    assert rc == 0 and n == 1000
    assert np.array_equal(d_out[:1000].cpu().numpy(), np.arange(1000, dtype=np.int64) * 3)


def test_noalloc_rejects_entropy_coded_frames_while_decoding(qb, api):
    """A stream inside the size limits whose frames carry an entropy-coded part
    (Balanced: byte-transposed rANS planes) passes the frame-table check and
    is refused by the decode kernels, which have no area for the coded part in
    the fixed arena; the next call still decodes a good stream."""
    _, torch = api
    rng = np.random.default_rng(20240611)
    b = np.minimum(rng.geometric(0.3, (60000, 6)) - 1, 255).astype(np.uint64)
    vals = (b << (np.arange(6, dtype=np.uint64) * np.uint64(8))).sum(axis=1, dtype=np.uint64)
    coded = qb.compress_column(vals, None, qb.Config(level=qb.Level.BALANCED_INPOOL), dtype=U64)
    assert coded[16] == 11  # the first frame is BYTE_TRANSPOSE
    d_out = torch.zeros(60000, dtype=torch.int64, device="cuda")
    d_src = torch.from_numpy(np.frombuffer(coded, np.uint8).copy()).cuda()
    assert noalloc(api, d_src, len(coded), d_out, 60000) == (ERR_NOALLOC_LIMIT, 0)
    ok = qb.compress_column(vals, None, qb.Config(level=qb.Level.FAST), dtype=U64)
    d_src = torch.from_numpy(np.frombuffer(ok, np.uint8).copy()).cuda()
    rc, n = noalloc(api, d_src, len(ok), d_out, 60000)
    assert rc == 0 and n == 60000
    assert d_out.cpu().numpy().view(np.uint64).tobytes() == vals.tobytes()
