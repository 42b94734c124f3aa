"""Batched decode of device streams (quoin_b200_decompress_queue_device): one
launch per kernel class reads and decodes every column of the batch.  Each
column's values, bitmap, dtype and count equal the single-column device
decode's (quoin_b200_decompress_column_device), whichever path takes it:
the batch for plain and nullable columns of every dtype and mode mix (RAW
and RLE validity blobs) and for decimal containers (a lane per limb), the
single-column path for entropy-coded frames, all-null and damaged streams,
and short buffers.
"""
import ctypes

import numpy as np
import pytest

from conftest import bitmap_from_bools, lcg_seq
from quoin_b200 import synth

pytestmark = pytest.mark.gpu

NW = {0: 8, 1: 8, 2: 8, 3: 4, 4: 4, 5: 4, 6: 16, 7: 32}


class Job(ctypes.Structure):
    _fields_ = [("d_src", ctypes.c_void_p), ("src_len", ctypes.c_size_t), ("d_values_out", ctypes.c_void_p),
                ("values_cap_bytes", ctypes.c_size_t), ("d_validity_out", ctypes.c_void_p),
                ("wire", ctypes.c_int32), ("n", ctypes.c_uint64), ("status", ctypes.c_int32)]


def stats(qb):
    out = (ctypes.c_uint64 * 6)()
    qb.lib.quoin_b200_reader_stats(out)
    return list(out)


def single(qb, torch, stream, cap):
    d_src = torch.from_numpy(np.frombuffer(stream, np.uint8).copy() if stream else np.zeros(1, np.uint8)).cuda()
    d_out = torch.zeros(max(cap, 8), dtype=torch.uint8, device="cuda")
    d_bm = torch.zeros(max(cap // 4, 8), dtype=torch.uint8, device="cuda")
    w, n = ctypes.c_int32(), ctypes.c_uint64()
    rc = qb.lib.quoin_b200_decompress_column_device(None, ctypes.c_void_p(d_src.data_ptr()), len(stream),
                                                    ctypes.c_void_p(d_out.data_ptr()), cap,
                                                    ctypes.c_void_p(d_bm.data_ptr()), ctypes.byref(w),
                                                    ctypes.byref(n), None)
    nb = n.value * NW.get(w.value, 8)
    return rc, w.value, n.value, d_out[:nb].cpu().numpy().tobytes() if rc == 0 else b"", \
        d_bm[:(n.value + 7) // 8].cpu().numpy().tobytes() if rc == 0 else b""


def run_queue(qb, torch, streams, caps):
    srcs = [torch.from_numpy(np.frombuffer(s, np.uint8).copy() if s else np.zeros(1, np.uint8)).cuda()
            for s in streams]
    outs = [torch.zeros(max(c, 8), dtype=torch.uint8, device="cuda") for c in caps]
    bms = [torch.zeros(max(c // 4, 8), dtype=torch.uint8, device="cuda") for c in caps]
    jobs = (Job * len(streams))()
    for i, s in enumerate(streams):
        jobs[i] = Job(srcs[i].data_ptr(), len(s), outs[i].data_ptr(), caps[i], bms[i].data_ptr(), 0, 0, 0)
    rc = qb.lib.quoin_b200_decompress_queue_device(None, jobs, len(streams), None)
    res = []
    for i in range(len(streams)):
        j = jobs[i]
        nb = j.n * NW.get(j.wire, 8)
        res.append((j.status, j.wire, j.n, outs[i][:nb].cpu().numpy().tobytes() if j.status == 0 else b"",
                    bms[i][:(j.n + 7) // 8].cpu().numpy().tobytes() if j.status == 0 else b""))
    return rc, res


def check_batch(qb, streams, caps, has_bitmap):
    import torch
    want = [single(qb, torch, s, c) for s, c in zip(streams, caps)]
    before = stats(qb)[5]
    rc, got = run_queue(qb, torch, streams, caps)
    batched = stats(qb)[5] - before
    for i, (g, w) in enumerate(zip(got, want)):
        assert g[:3] == w[:3], (i, g[:3], w[:3])
        assert g[3] == w[3], i
        if has_bitmap[i] and g[0] == 0:
            assert g[4] == w[4], i
    first = next((w[0] for w in want if w[0] != 0), 0)
    assert rc == first
    return batched


def test_queue_mixed_columns(qb):
    cols = synth.mixed_columns(48, 1 << 17)
    streams, caps, hb = [], [], []
    for name, dt, v, bm in cols:
        sc, pr = (4, 18) if dt == 6 else (0, 0)
        s = qb.compress_column(v, bm, qb.Config(level=qb.Level.FAST), dtype=dt, scale=sc, precision=pr)
        streams.append(s)
        caps.append(len(v) * NW[dt])
        hb.append(bm is not None)
    batched = check_batch(qb, streams, caps, hb)
    assert batched == len(cols)  # every column of the mix, decimal containers included


def test_queue_special_columns(qb):
    rng = np.random.default_rng(77)
    vb = rng.random(50_000) > 0.1
    clustered = np.ones(50_000, bool)
    clustered[1000:9000] = False
    cases = [
        (np.cumsum(1000 + rng.poisson(50, 50_000)).astype(np.int64), 1, bitmap_from_bools(vb), {}),
        (np.arange(50_000, dtype=np.int64), 1, bitmap_from_bools(clustered), {}),                 # RLE blob
        (np.arange(5000, dtype=np.int64), 1, bitmap_from_bools(np.zeros(5000, bool)), {}),        # all null
        (np.sin(np.arange(40_000) * 0.01), 0, None, {"level": 258}),                            # entropy-coded
        ((1000 + np.arange(20_000) % 777).astype(np.int64), 1, None, {"block_size": 7}),        # many frames
        (lcg_seq(3, 30_000), 2, None, {}),                                                      # RAW / XORZ
        (np.repeat(np.arange(300, dtype=np.int32), 100), 3, bitmap_from_bools(vb[:30_000]), {}),  # RLE / DICT
        ((np.round(rng.normal(25, 5, 40_000) * 10) / 10).astype(np.float32), 5, None, {}),      # f32 DICT
        (np.zeros(0, np.int64), 1, None, {}),                                                   # empty
    ]
    dec = np.zeros((30_000, 16), np.uint8)
    dec[:, :8] = (rng.integers(-10**12, 10**12, 30_000)).view(np.uint8).reshape(-1, 8)
    dec[:, 8:] = np.where(dec[:, 7:8] >= 128, 255, 0)
    streams, caps, hb = [], [], []
    for v, dt, bm, kw in cases:
        s = qb.compress_column(v, bm, qb.Config(level=qb.Level(kw.get("level", 1)), block_size=kw.get("block_size")),
                               dtype=dt)
        streams.append(s)
        caps.append(len(v) * NW[dt])
        hb.append(bm is not None)
    for bm in (None, bitmap_from_bools(vb[:30_000]), bitmap_from_bools(clustered[:30_000])):  # decimal containers
        streams.append(qb.compress_column(dec, bm, qb.Config(level=qb.Level.FAST), dtype=6, scale=3, precision=20))
        caps.append(30_000 * 16)
        hb.append(bm is not None)
    # a damaged stream, a short output buffer and a stream that is not one
    streams.append(streams[0][:len(streams[0]) // 2])
    caps.append(caps[0])
    hb.append(True)
    streams.append(streams[5])
    caps.append(caps[5] - 8)
    hb.append(False)
    streams.append(b"XCR1" + streams[5][4:])
    caps.append(caps[5])
    hb.append(False)
    batched = check_batch(qb, streams, caps, hb)
    assert batched >= 9
