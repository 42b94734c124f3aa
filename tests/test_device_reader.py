"""The device-side stream reader (quoin_b200_decompress_column_device).

A stream already in device memory is read on the GPU: header, validity
bitmap and frame table (reference src/decoder.rs:43-118, src/format.rs:65-94,
src/decimal.rs:100-168), then decoded by the block decoder.  Every case here
compares it with the host-parsed decode of the same stream
(quoin_b200_decompress_column, whose values the parity tests pin to the
oracle): the same values, bitmap, dtype and count, and on damaged streams the
same error code.  The cases reach each branch of the reader: plain and
nullable lanes, decimal containers (two and four limb lanes), RLE validity
blobs, tables larger than the first capacity guess
and than shared memory, payloads full of bytes that look like frame headers,
streams at unaligned device addresses, and mutated streams.
"""
import ctypes

import numpy as np
import pytest

from conftest import bitmap_from_bools, lcg1_seq, lcg_seq

pytestmark = pytest.mark.gpu

F64, I64, U64, I32, U32, F32, DEC128, DEC256 = range(8)
NW = {F64: 8, I64: 8, U64: 8, I32: 4, U32: 4, F32: 4, DEC128: 16, DEC256: 32}
ERR_BUFFER_TOO_SMALL = -2


def host_parse(qb, stream):
    """(rc, wire, n) of the host reader's full parse."""
    buf = np.frombuffer(stream, np.uint8) if stream else np.zeros(1, np.uint8)
    w, n, hv = ctypes.c_int32(), ctypes.c_uint64(), ctypes.c_int32()
    rc = qb.lib.quoin_b200_parse(buf.ctypes.data, len(stream), ctypes.byref(w), ctypes.byref(n), ctypes.byref(hv))
    return rc, w.value, n.value


def host_decode(qb, stream, wire, n):
    """(rc, values bytes, bitmap bytes or None) through the host-buffer decode."""
    buf = np.frombuffer(stream, np.uint8)
    out = np.zeros(max(n * NW[wire], 8), np.uint8)
    bm = np.zeros(max((n + 7) // 8, 1), np.uint8)
    rc = qb.lib.quoin_b200_decompress_column(None, buf.ctypes.data, len(stream), out.ctypes.data, bm.ctypes.data)
    return rc, out[: n * NW[wire]].tobytes(), bm[: (n + 7) // 8].tobytes()


def device_decode(qb, stream, cap_bytes, offset=0, ctx=None):
    """(rc, wire, n, values bytes, bitmap bytes) through the device reader; the
    stream sits `offset` bytes into its device buffer."""
    import torch
    src = np.zeros(len(stream) + offset + 1, np.uint8)
    src[offset: offset + len(stream)] = np.frombuffer(stream, np.uint8)
    d_src = torch.from_numpy(src).cuda()
    d_out = torch.full((max(cap_bytes, 8),), 0xA5, dtype=torch.uint8, device="cuda")
    d_bm = torch.full((max(cap_bytes // 4, 8),), 0xA5, dtype=torch.uint8, device="cuda")
    w, n = ctypes.c_int32(), ctypes.c_uint64()
    rc = qb.lib.quoin_b200_decompress_column_device(
        ctx, ctypes.c_void_p(d_src.data_ptr() + offset), len(stream), ctypes.c_void_p(d_out.data_ptr()), cap_bytes,
        ctypes.c_void_p(d_bm.data_ptr()), ctypes.byref(w), ctypes.byref(n),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    nb = n.value * NW.get(w.value, 8)
    vals = d_out[:nb].cpu().numpy().tobytes() if rc == 0 else b""
    bm = d_bm[: (n.value + 7) // 8].cpu().numpy().tobytes() if rc == 0 else b""
    return rc, w.value, n.value, vals, bm


def reader_stats(qb):
    out = (ctypes.c_uint64 * 6)()
    qb.lib.quoin_b200_reader_stats(out)
    return out[0], out[1]


def check_same(qb, stream, offset=0, device_read=True):
    """The device path equals the host path; with device_read the device
    reader (not the host reader) read the stream."""
    before = reader_stats(qb)
    rc, wire, n = host_parse(qb, stream)
    assert rc == 0
    hrc, hv, hb = host_decode(qb, stream, wire, n)
    assert hrc == 0
    drc, dw, dn, dv, db = device_decode(qb, stream, n * NW[wire], offset)
    assert (drc, dw, dn) == (0, wire, n)
    assert dv == hv
    if stream[5] & 1:
        assert db == hb
    after = reader_stats(qb)
    if device_read:
        assert after == (before[0] + 1, before[1]), "the host reader took the stream"
    return hv


def decimal_bytes(v, width=16):
    v = np.asarray(v, np.int64)
    out = np.zeros((v.size, width), np.uint8)
    out[:, :8] = v.view(np.uint8).reshape(-1, 8)
    out[:, 8:] = np.where(v < 0, 255, 0)[:, None]
    return out


def prices_with_exceptions(rng, n, frac=0.03):
    v = np.floor(rng.random(n) * 1_000_000 + 0.5) / 100.0
    bits = rng.integers(0, 1 << 62, n, dtype=np.int64).view(np.uint64) | (rng.integers(0, 2, n).astype(np.uint64) << np.uint64(63))
    bits = bits & ~(np.uint64(0x7FF) << np.uint64(52)) | (rng.integers(0, 0x7FF, n).astype(np.uint64) << np.uint64(52))
    pick = rng.random(n) < frac
    v[pick] = bits[pick].view(np.float64)
    return v


def reader_cases():
    rng = np.random.default_rng(4321)
    vb = rng.random(300_000) > 0.1
    clustered = np.ones(200_000, bool)
    for s in range(0, 200_000, 20_000):
        clustered[s: s + 3000] = False
    cats = (lcg_seq(41, 64) >> np.uint64(33)).astype(np.int64) - (1 << 30)
    # runs of 1..250 positions: an RLE blob of 1-2 bytes a run over several
    # 16 KB reading rounds, one- and two-byte varints
    lens = rng.integers(1, 250, 20_000)
    many = np.repeat(np.arange(lens.size) % 2 == 1, lens)[:2_000_000]
    return [
        ("empty_i64", np.zeros(0, np.int64), I64, None, {}),
        ("one_f64", np.array([3.5]), F64, None, {}),
        ("timestamps_nullable", (np.cumsum(1_000_000 + rng.poisson(5000, 300_000)) + 1_700_000_000_000_000_000)
         .astype(np.int64), I64, bitmap_from_bools(vb), {}),
        ("runs_u64_nullable", (np.uint64(1 << 40) + (lcg1_seq(3, 300_000) & np.repeat(
            (np.uint64(1) << (np.arange(293) % 38 + 3).astype(np.uint64)) - np.uint64(1), 1024)[:300_000])),
         U64, bitmap_from_bools(vb), {}),
        ("categories_i32_nullable", np.repeat(cats[rng.integers(0, 64, 20000)], 15)[:300_000].astype(np.int32), I32,
         bitmap_from_bools(vb), {}),
        ("all_null", np.arange(5000, dtype=np.int64), I64, bitmap_from_bools(np.zeros(5000, bool)), {}),
        ("clustered_nulls_rle_blob", np.arange(200_000, dtype=np.uint64) * 7, U64, bitmap_from_bools(clustered), {}),
        ("rle_blob_many_runs", np.arange(many.size, dtype=np.int64) * 3, I64, bitmap_from_bools(many), {}),
        ("rle_blob_leading_valid", np.arange(5000, dtype=np.int64), I64,
         bitmap_from_bools(np.arange(5000) < 4000), {}),
        ("prices_alp", np.floor(rng.random(200_000) * 1_000_000 + 0.5) / 100.0, F64, None, {}),
        # two-decimal prices with 3 % random-bit values: ALP-RD frames with
        # about a thousand exceptions each, whose lists the reader walks
        ("prices_alprd_exceptions", prices_with_exceptions(rng, 200_000), F64, None, {}),
        ("walk_f64", 20.0 + np.cumsum(rng.normal(0, 1e-3, 200_000)), F64, None, {}),
        ("sensor_f32", (np.round(rng.normal(25, 5, 200_000) * 10) / 10).astype(np.float32), F32, None, {}),
        ("xorz_f64", np.sin(np.arange(100_000) * 1e-4), F64, None, {}),
        ("wide_u64_raw", lcg_seq(7, 100_000), U64, None, {}),
        ("decimal128_nullable", decimal_bytes(rng.integers(-10**14, 10**14, 150_000)), DEC128,
         bitmap_from_bools(vb[:150_000]), {"scale": 4, "precision": 18}),
        ("decimal256", decimal_bytes(rng.integers(0, 40, 70_000) * 1_000_000_007, 32), DEC256, None,
         {"scale": 2, "precision": 60}),
        # 40,000 frames of one value: more candidates than the first capacity
        # guess and than the shared-memory tables
        ("block_size_1", (1000 + np.arange(40_000) % 777).astype(np.int64), I64, None, {"block_size": 1}),
        ("block_size_7_nullable", np.arange(30_000, dtype=np.int64) * 5, I64, bitmap_from_bools(vb[:30_000]),
         {"block_size": 7}),
        ("balanced_entropy", np.sin(np.arange(60_000) * 0.01), F64, None, {"level": 258}),
    ]


@pytest.mark.parametrize("case", reader_cases(), ids=lambda c: c[0])
def test_device_reader_matches_host_reader(qb, case):
    name, vals, dt, bm, kw = case
    level = kw.get("level", 1)
    stream = qb.compress_column(vals, bm, qb.Config(level=qb.Level(level), block_size=kw.get("block_size")),
                                dtype=dt, scale=kw.get("scale", 0), precision=kw.get("precision", 0))
    got = check_same(qb, stream)
    want = np.ascontiguousarray(vals).view(np.uint8).reshape(-1, NW[dt]).copy() if len(vals) else np.zeros(0)
    if bm is not None and len(vals):
        want[~np.unpackbits(bm, bitorder="little")[: len(vals)].astype(bool)] = 0
    assert got == want.tobytes()


@pytest.mark.parametrize("offset", [1, 3, 6, 13])
def test_device_reader_unaligned_stream(qb, offset):
    rng = np.random.default_rng(offset)
    vals = (np.cumsum(1000 + rng.poisson(50, 100_000)) + 10**15).astype(np.int64)
    bm = bitmap_from_bools(rng.random(100_000) > 0.2)
    check_same(qb, qb.compress_column(vals, bm, qb.Config(level=qb.Level.FAST)), offset)


def test_header_like_payload_bytes(qb):
    """RAW payloads where every other value reads as a frame header (mode 5,
    1 <= n <= 100,000, plen = 7, the next value's low byte 0): each points 16
    bytes on, to the next such value, and the last of a frame to the next
    frame's header, so long chains of false candidates merge into the true
    chain."""
    k = np.arange(100_000, dtype=np.uint64)
    fake = np.uint64(5) | ((np.uint64(1) + k) << np.uint64(8)) | (np.uint64(7) << np.uint64(40))
    for seed, first in ((99, 0), (98, 1)):
        vals = lcg_seq(seed, 200_000) & ~np.uint64(0xFF)
        vals[first::2] = fake
        stream = qb.compress_column(vals, None, qb.Config(level=qb.Level.FAST), dtype=U64)
        assert stream[16] == 5  # RAW frames
        assert check_same(qb, stream) == vals.tobytes()


def test_buffer_too_small_reports_count(qb):
    vals = np.arange(10_000, dtype=np.int64)
    stream = qb.compress_column(vals)
    rc, w, n, _, _ = device_decode(qb, stream, 10_000 * 8 - 1)
    assert (rc, w, n) == (ERR_BUFFER_TOO_SMALL, I64, 10_000)


def test_mutated_streams_agree_with_host_reader(qb):
    rng = np.random.default_rng(0x2468ACE)
    vb = rng.random(6000) > 0.15
    seeds = [qb.compress_column(v, b, qb.Config(level=qb.Level.FAST, block_size=bs), dtype=dt) for v, b, dt, bs in (
        ((1000 + np.arange(6000) % 300).astype(np.int64), None, I64, 1000),
        (np.cumsum(rng.poisson(9, 6000)).astype(np.int64), bitmap_from_bools(vb), I64, 1500),
        (np.sin(np.arange(6000) * 0.01), None, F64, None),
        (np.repeat(np.arange(60, dtype=np.int32), 100), bitmap_from_bools(vb), I32, 2000),
        (lcg_seq(5, 6000), None, U64, 700),
        (decimal_bytes(rng.integers(-999, 999, 6000)), None, DEC128, 1024),
        (np.arange(6000, dtype=np.int64), bitmap_from_bools(np.repeat(np.arange(40) % 3 > 0, 150)), I64, 2000))]
    assert any(sd[5] & 1 and sd[17] == 1 for sd in seeds)  # an RLE validity blob among the seeds
    for it in range(600):
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
        prc, wire, n = host_parse(qb, b)
        if prc != 0:
            drc = device_decode(qb, b, 1 << 16)[0]
            assert drc == prc or drc == ERR_BUFFER_TOO_SMALL, f"iteration {it}: device {drc} host {prc}"
            continue
        hrc, hv, hb = host_decode(qb, b, wire, n)
        drc, dw, dn, dv, db = device_decode(qb, b, n * NW[wire])
        assert drc == hrc, f"iteration {it}: device {drc} host {hrc}"
        if hrc == 0:
            assert (dw, dn) == (wire, n) and dv == hv
            if b[5] & 1:
                assert db == hb
    # still healthy
    check_same(qb, seeds[1])


def _stream(frames, dtype, plog2=16):
    """A stream around raw frame payloads [(mode, n, payload)]."""
    n = sum(f[1] for f in frames)
    out = bytearray(b"FCR1" + bytes([2, 0, plog2, dtype]) + n.to_bytes(8, "little"))
    for mode, k, p in frames:
        out += bytes([mode]) + k.to_bytes(4, "little") + len(p).to_bytes(4, "little") + p
    return bytes(out)


def test_high_max_modes(qb, oracle):
    """Frames of the High/Max residual modes (linear recurrences and
    predictors, range-coded or rANS-coded): the device reader reads them,
    except PRED (0), whose untagged LEB128 payload it leaves to the host
    reader; the values agree either way."""
    v = (np.sin(np.arange(20_000) * 0.002) * 100.0 + np.arange(20_000) * 0.01).view(np.uint64)
    cuts = ((0, 1), (1, 4097), (4097, 20_000))
    for mode, tag in ((7, 0), (20, 2), (45, 0)):
        frames = [(mode, hi - lo, oracle.linear_payload(mode, v[lo:hi], 2, tag)) for lo, hi in cuts]
        assert check_same(qb, _stream(frames, U64)) == v.tobytes()
    for mode, tag, read_on_device in ((29, 0, True), (25, 2, True), (0, 0, False)):
        frames = [(mode, hi - lo, oracle.pred_payload(mode, v[lo:hi], 16, tag)) for lo, hi in cuts]
        assert check_same(qb, _stream(frames, U64), device_read=read_on_device) == v.tobytes()
