"""Batches of columns (quoin_b200_compress_batch_device /
quoin_b200_decompress_batch_device): columns of the batched configuration
(uneven lengths, mixed dtypes, nulls) spread over a pool of contexts must give
each column the single-column call's stream and values, and a column that
fails (a too-small output buffer) must report its own status without
disturbing the others.
"""
import ctypes

import numpy as np
import pytest

from quoin_b200 import synth

pytestmark = pytest.mark.gpu

P, S = ctypes.c_void_p, ctypes.c_size_t
ERR_BUFFER_TOO_SMALL = -2


class CompressJob(ctypes.Structure):
    _fields_ = [("wire_dtype", ctypes.c_int32), ("scale", ctypes.c_int8), ("precision", ctypes.c_uint8),
                ("n", S), ("d_values", P), ("d_validity", P), ("d_dst", P), ("dst_cap", S), ("out_len", S),
                ("status", ctypes.c_int32)]


class DecompressJob(ctypes.Structure):
    _fields_ = [("idx", P), ("d_src", P), ("d_values_out", P), ("d_validity_out", P), ("status", ctypes.c_int32)]


@pytest.fixture(scope="module")
def batch_api(qb):
    L = qb.lib
    L.quoin_b200_batch_create.restype = P
    L.quoin_b200_batch_create.argtypes = [ctypes.c_int]
    L.quoin_b200_batch_free.argtypes = [P]
    L.quoin_b200_compress_batch_device.argtypes = [P, ctypes.POINTER(CompressJob), S, ctypes.POINTER(qb._QuoinConfig)]
    L.quoin_b200_compress_batch_device.restype = ctypes.c_int
    L.quoin_b200_decompress_batch_device.argtypes = [P, ctypes.POINTER(DecompressJob), S]
    L.quoin_b200_decompress_batch_device.restype = ctypes.c_int
    return L


def expected(v, dt, bm):
    raw = np.ascontiguousarray(v).view(np.uint8).reshape(len(v), -1).copy()
    if bm is not None:
        valid = np.unpackbits(bm, bitorder="little")[:len(v)].astype(bool)
        raw[~valid] = 0
    return raw.tobytes()


def test_batch_matches_single_column_calls(qb, batch_api):
    import torch
    L = batch_api
    torch.cuda.set_device(0)
    cols = synth.mixed_columns(48, 1 << 17)
    cfg = qb._cfg(qb.Config(level=qb.Level.FAST))
    dev = []
    jobs = (CompressJob * len(cols))()
    for j, (name, dt, v, bm) in enumerate(cols):
        n = len(v)
        dv = torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).cuda()
        db = torch.from_numpy(bm.copy()).cuda() if bm is not None else None
        cap = qb._stream_bound(dt, n, bm is not None)
        if j == 5:
            cap = 16  # too small: this column alone reports BUFFER_TOO_SMALL
        dd = torch.zeros(max(cap, 16), dtype=torch.uint8, device="cuda")
        dev.append((dv, db, dd))
        sc, pr = (4, 18) if dt == qb.DECIMAL128 else (0, 0)
        jobs[j] = CompressJob(dt, sc, pr, n, dv.data_ptr(), db.data_ptr() if db is not None else None,
                              dd.data_ptr(), cap, 0, 99)
    b = P(L.quoin_b200_batch_create(4))
    assert b.value
    try:
        rc = L.quoin_b200_compress_batch_device(b, jobs, len(cols), ctypes.byref(cfg))
        assert rc == ERR_BUFFER_TOO_SMALL
        streams = []
        for j, (name, dt, v, bm) in enumerate(cols):
            sc, pr = (4, 18) if dt == qb.DECIMAL128 else (0, 0)
            want = qb.compress_column(v, bm, qb.Config(level=qb.Level.FAST), dtype=dt, scale=sc, precision=pr)
            if j == 5:
                assert jobs[j].status == ERR_BUFFER_TOO_SMALL and jobs[j].out_len >= len(want)  # a size that fits
                streams.append(None)
                continue
            assert jobs[j].status == 0, name
            got = dev[j][2][: jobs[j].out_len].cpu().numpy().tobytes()
            assert got == want, name
            streams.append(got)
        # decode the good columns as one batch
        keep = [j for j in range(len(cols)) if streams[j] is not None]
        djobs = (DecompressJob * len(keep))()
        outs = []
        for k, j in enumerate(keep):
            name, dt, v, bm = cols[j]
            idx = P()
            assert L.quoin_b200_index_create(None, streams[j], len(streams[j]), ctypes.byref(idx)) == 0
            dsrc = torch.from_numpy(np.frombuffer(streams[j], np.uint8).copy()).cuda()
            dout = torch.zeros(max(np.ascontiguousarray(v).nbytes, 8), dtype=torch.uint8, device="cuda")
            dvb = torch.zeros(max((len(v) + 7) // 8, 1), dtype=torch.uint8, device="cuda")
            outs.append((idx, dsrc, dout, dvb))
            djobs[k] = DecompressJob(idx, dsrc.data_ptr(), dout.data_ptr(), dvb.data_ptr(), 99)
        try:
            assert L.quoin_b200_decompress_batch_device(b, djobs, len(keep)) == 0
            for k, j in enumerate(keep):
                name, dt, v, bm = cols[j]
                assert djobs[k].status == 0
                nb = np.ascontiguousarray(v).nbytes
                assert outs[k][2][:nb].cpu().numpy().tobytes() == expected(v, dt, bm), name
                if bm is not None:
                    assert outs[k][3][: (len(v) + 7) // 8].cpu().numpy().tobytes() == bm.tobytes(), name
        finally:
            for idx, *_ in outs:
                L.quoin_b200_index_free(idx)
    finally:
        L.quoin_b200_batch_free(b)


def test_batch_create_rejects_bad_worker_counts(batch_api):
    assert not batch_api.quoin_b200_batch_create(0)
    assert not batch_api.quoin_b200_batch_create(65)


def test_batch_edges(qb, batch_api):
    L = batch_api
    b = P(L.quoin_b200_batch_create(2))
    try:
        assert L.quoin_b200_compress_batch_device(b, None, 0, None) == 0  # no columns
        assert L.quoin_b200_decompress_batch_device(b, None, 0) == 0
        djobs = (DecompressJob * 1)()
        djobs[0] = DecompressJob(None, None, None, None, 99)  # no index: this job alone fails
        assert L.quoin_b200_decompress_batch_device(b, djobs, 1) == -1 and djobs[0].status == -1
        assert L.quoin_b200_compress_batch_device(None, None, 0, None) == -1
    finally:
        L.quoin_b200_batch_free(b)
    L.quoin_b200_batch_free(None)
