"""The request server (quoin_b200_server_*): compress and decompress requests
on device buffers, submitted together from one thread, must each give the
single-column call's stream and values; a request above the budget is
refused with OverBudget; with a budget that admits one or two requests at a
time the requests still all finish, and the admitted bytes never exceed it.
"""
import ctypes

import numpy as np
import pytest

from quoin_b200 import synth

pytestmark = pytest.mark.gpu

P, S, U64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64
OP_COMPRESS, OP_DECOMPRESS = 0, 1
ERR_OVER_BUDGET = -23


class Request(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("wire_dtype", ctypes.c_int32), ("scale", ctypes.c_int8),
                ("precision", ctypes.c_uint8), ("n", S), ("d_values", P), ("d_validity", P), ("d_dst", P),
                ("dst_cap", S), ("idx", P), ("d_src", P), ("d_values_out", P), ("d_validity_out", P),
                ("device_bytes", U64), ("out_len", S), ("status", ctypes.c_int32), ("done", ctypes.c_int32),
                ("t_submit_ns", U64), ("t_start_ns", U64), ("t_end_ns", U64)]


@pytest.fixture(scope="module")
def server_api(qb):
    L = qb.lib
    L.quoin_b200_server_create.restype = P
    L.quoin_b200_server_create.argtypes = [ctypes.c_int, U64, ctypes.POINTER(qb._QuoinConfig)]
    L.quoin_b200_server_submit.argtypes = [P, ctypes.POINTER(Request)]
    L.quoin_b200_server_submit.restype = ctypes.c_int
    L.quoin_b200_server_wait.argtypes = [P, ctypes.POINTER(Request), ctypes.c_int]
    L.quoin_b200_server_wait.restype = ctypes.c_int
    L.quoin_b200_server_peak_bytes.argtypes = [P]
    L.quoin_b200_server_peak_bytes.restype = U64
    L.quoin_b200_server_free.argtypes = [P]
    return L


def _expected(v, bm):
    raw = np.ascontiguousarray(v).view(np.uint8).reshape(len(v), -1).copy()
    if bm is not None:
        raw[~np.unpackbits(bm, bitorder="little")[:len(v)].astype(bool)] = 0
    return raw.tobytes()


def _run(qb, L, cols, workers, budget):
    import torch
    torch.cuda.set_device(0)
    cfg = qb._cfg(qb.Config(level=qb.Level.FAST))
    srv = P(L.quoin_b200_server_create(workers, budget, ctypes.byref(cfg)))
    assert srv.value
    keep, reqs = [], []
    try:
        for name, dt, v, bm in cols:
            n = len(v)
            dv = torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).reshape(-1).copy()).cuda()
            db = torch.from_numpy(bm.copy()).cuda() if bm is not None else None
            cap = qb._stream_bound(dt, n, bm is not None)
            dd = torch.zeros(cap, dtype=torch.uint8, device="cuda")
            sc, pr = (4, 18) if dt == qb.DECIMAL128 else (0, 0)
            r = Request(op=OP_COMPRESS, wire_dtype=dt, scale=sc, precision=pr, n=n, d_values=dv.data_ptr(),
                        d_validity=db.data_ptr() if db is not None else None, d_dst=dd.data_ptr(), dst_cap=cap,
                        device_bytes=dv.numel() + cap)
            keep.append((dv, db, dd))
            reqs.append(r)
        for r in reqs:
            assert L.quoin_b200_server_submit(srv, ctypes.byref(r)) == 0
        streams = []
        for (name, dt, v, bm), r, (dv, db, dd) in zip(cols, reqs, keep):
            assert L.quoin_b200_server_wait(srv, ctypes.byref(r), -1) == 0, name
            assert r.done == 1 and r.t_submit_ns <= r.t_start_ns <= r.t_end_ns
            sc, pr = (4, 18) if dt == qb.DECIMAL128 else (0, 0)
            want = qb.compress_column(v, bm, qb.Config(level=qb.Level.FAST), dtype=dt, scale=sc, precision=pr)
            got = dd[: r.out_len].cpu().numpy().tobytes()
            assert got == want, name
            streams.append(got)
        # the streams back through decompress requests
        idxs, dreqs, outs = [], [], []
        for (name, dt, v, bm), st in zip(cols, streams):
            idx = P()
            assert L.quoin_b200_index_create(None, st, len(st), ctypes.byref(idx)) == 0
            idxs.append(idx)
            ds = torch.from_numpy(np.frombuffer(st, np.uint8).copy()).cuda()
            do = torch.zeros(max(np.ascontiguousarray(v).nbytes, 8), dtype=torch.uint8, device="cuda")
            dvb = torch.zeros(max((len(v) + 7) // 8, 1), dtype=torch.uint8, device="cuda")
            outs.append((ds, do, dvb))
            dreqs.append(Request(op=OP_DECOMPRESS, idx=idx, d_src=ds.data_ptr(), d_values_out=do.data_ptr(),
                                 d_validity_out=dvb.data_ptr(), device_bytes=len(st) + do.numel()))
        try:
            for r in dreqs:
                assert L.quoin_b200_server_submit(srv, ctypes.byref(r)) == 0
            for (name, dt, v, bm), r, (ds, do, dvb) in zip(cols, dreqs, outs):
                assert L.quoin_b200_server_wait(srv, ctypes.byref(r), -1) == 0, name
                nb = np.ascontiguousarray(v).nbytes
                assert do[:nb].cpu().numpy().tobytes() == _expected(v, bm), name
        finally:
            for idx in idxs:
                L.quoin_b200_index_free(idx)
        return L.quoin_b200_server_peak_bytes(srv)
    finally:
        L.quoin_b200_server_free(srv)


def test_server_requests_match_single_calls(qb, server_api):
    cols = synth.mixed_columns(40, 1 << 17)
    peak = _run(qb, server_api, cols, 6, 120 << 30)
    assert peak > 0


def test_server_small_budget(qb, server_api):
    cols = synth.mixed_columns(12, 1 << 15, min_len=1 << 14)
    budget = 6 << 20  # one or two of these requests at a time (48 B/value of working memory + buffers)
    peak = _run(qb, server_api, cols, 4, budget)
    assert 0 < peak <= budget


def test_server_refuses_requests_above_budget(qb, server_api):
    L = server_api
    cfg = qb._cfg(qb.Config(level=qb.Level.FAST))
    srv = P(L.quoin_b200_server_create(2, 1 << 20, ctypes.byref(cfg)))
    try:
        r = Request(op=OP_COMPRESS, wire_dtype=qb.I64, n=1 << 20, d_values=1, d_dst=1, dst_cap=1 << 24,
                    device_bytes=1 << 24)
        assert L.quoin_b200_server_submit(srv, ctypes.byref(r)) == ERR_OVER_BUDGET
        bad = Request(op=7)
        assert L.quoin_b200_server_submit(srv, ctypes.byref(bad)) == -20
    finally:
        L.quoin_b200_server_free(srv)
    assert not L.quoin_b200_server_create(0, 1 << 20, None)
    assert not L.quoin_b200_server_create(4, 0, None)


def test_server_empty_column_and_free_with_queued_requests(qb, server_api):
    import torch
    L = server_api
    cfg = qb._cfg(qb.Config(level=qb.Level.FAST))
    srv = P(L.quoin_b200_server_create(2, 1 << 30, ctypes.byref(cfg)))
    cap = qb._stream_bound(qb.I64, 0, False)
    dd = torch.zeros(max(cap, 64), dtype=torch.uint8, device="cuda")
    dv = torch.zeros(8, dtype=torch.uint8, device="cuda")
    empty = Request(op=OP_COMPRESS, wire_dtype=qb.I64, n=0, d_values=dv.data_ptr(), d_dst=dd.data_ptr(),
                    dst_cap=cap, device_bytes=64)
    assert L.quoin_b200_server_submit(srv, ctypes.byref(empty)) == 0
    assert L.quoin_b200_server_wait(srv, ctypes.byref(empty), -1) == 0
    assert dd[: empty.out_len].cpu().numpy().tobytes() == qb.compress_column(np.zeros(0, np.int64))
    # requests still queued when the server is freed are finished first
    v = np.arange(1 << 16, dtype=np.int64)
    dv2 = torch.from_numpy(v.view(np.uint8).copy()).cuda()
    cap2 = qb._stream_bound(qb.I64, len(v), False)
    outs = [torch.zeros(cap2, dtype=torch.uint8, device="cuda") for _ in range(8)]
    reqs = [Request(op=OP_COMPRESS, wire_dtype=qb.I64, n=len(v), d_values=dv2.data_ptr(), d_dst=o.data_ptr(),
                    dst_cap=cap2, device_bytes=v.nbytes + cap2) for o in outs]
    for r in reqs:
        assert L.quoin_b200_server_submit(srv, ctypes.byref(r)) == 0
    L.quoin_b200_server_free(srv)
    want = qb.compress_column(v)
    for r, o in zip(reqs, outs):
        assert r.done == 1 and r.status == 0
        assert o[: r.out_len].cpu().numpy().tobytes() == want
