"""One column split across ranks (quoin_b200.shard).

CPU: the plan from gathered probe bytes equals plan_blocks' (the oracle's
frames), and the whole sharded compress / decompress — probe, all-gather of
probe bytes, plan, per-rank part streams, all-gather of the parts, frame walk
and per-rank decode — run as two and three gloo ranks (torch.distributed) with
the oracle as each rank's engine, giving the oracle's single-call stream and
values.  GPU: the same with the CUDA engine, the ranks as host threads on one
device exchanging through a host barrier (no kernel waits on another rank)."""
import os
import socket
import sys
import threading

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import quoin_b200 as Q  # noqa: E402
from quoin_b200 import shard  # noqa: E402
from oracle import oracle as O  # noqa: E402

W = 32768


def _lane(values, dtype):
    """The u64 lane of a column's valid values (reference src/lib.rs:389-403)."""
    v = np.ascontiguousarray(values)
    if dtype in (Q.I32,):
        return v.astype(np.int64).view(np.uint64)
    if dtype in (Q.U32,):
        return v.astype(np.uint64)
    if dtype == Q.F32:
        return v.astype(np.float64).view(np.uint64)
    return v.view(np.uint64)


class OracleEngine:
    """Each rank's compute by the oracle (test infrastructure)."""

    def probe_windows(self, values, dtype):
        return O.probe_windows(_lane(values, dtype))

    def prefix(self, n, dtype, bm, cfg):
        s = O.compress_column(np.zeros(n, dtype=Q._NP[dtype]), dtype, bm)
        if not s[5] & 1:
            return s[:16]
        vlen, pos = shard._varint(s, 16)
        return s[:pos + vlen]

    def compress_lane(self, values, dtype, cfg):
        return O.compress_column(np.ascontiguousarray(values), dtype, None)

    def decompress(self, stream):
        dt, vals, bm, sc, pr = O.decompress_column(stream)
        return Q.DecodedColumn(vals, None if bm is None else bytes(bm), dt)


def _columns():
    rng = np.random.default_rng(7)
    out = []
    # u64: random windows, then low-cardinality windows that grow to four
    # windows, so grown blocks cross the ranks' window ranges
    n = 9 * W + 123
    v = rng.integers(0, 2**63, n, dtype=np.uint64)
    v[2 * W:6 * W] = rng.integers(0, 5, 4 * W).astype(np.uint64)
    v[7 * W + 500:] = 42
    out.append(("u64_grown", Q.U64, v, None))
    bm = np.packbits(rng.random(n) < 0.9, bitorder="little")
    out.append(("u64_grown_nulls", Q.U64, v, bm))
    # clustered nulls (an RLE validity blob)
    bits = np.ones(n, dtype=bool)
    bits[1000:90000] = False
    bits[200000:200100] = False
    out.append(("i64_rle_nulls", Q.I64, (np.arange(n, dtype=np.int64) * 3 + 1000), np.packbits(bits,
                                                                                             bitorder="little")))
    m = 5 * W + 7
    out.append(("f64_walk", Q.F64, np.cumsum(rng.normal(0, 1e-3, m)) + 20.0, None))
    out.append(("i32_small", Q.I32, rng.integers(-50, 50, 1000).astype(np.int32), None))
    out.append(("f32_nulls", Q.F32, (rng.integers(0, 400, 3 * W) / 10).astype(np.float32),
                np.packbits(rng.random(3 * W) < 0.7, bitorder="little")))
    out.append(("all_null", Q.U32, np.zeros(70000, dtype=np.uint32), np.zeros((70000 + 7) // 8, dtype=np.uint8)))
    out.append(("empty", Q.I64, np.zeros(0, dtype=np.int64), None))
    return out


# ---------------------------------------------------------------------------
# Host logic alone
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name,dtype,values,bm", _columns(), ids=[c[0] for c in _columns()])
def test_plan_from_probe_bytes_is_plan_blocks(name, dtype, values, bm):
    n = len(values)
    bits = None if bm is None else np.unpackbits(bm, bitorder="little")[:n].astype(bool)
    lane_vals = values if bits is None else values[bits]
    flags = O.probe_windows(_lane(lane_vals, dtype))
    blocks = shard.plan_from_flags(flags, len(lane_vals))
    stream = O.compress_column(values, dtype, bm)
    L = shard.StreamLayout(stream)
    assert [fn for _, fn in L.frames] == [e - s for s, e in blocks]


def test_partition_helpers():
    assert shard.window_split(5, 2) == [(0, 2), (2, 5)]
    assert shard.window_split(1, 3) == [(0, 0), (0, 0), (0, 1)]
    blocks = [(0, W), (W, 5 * W), (5 * W, 6 * W), (6 * W, 6 * W + 9)]
    assert shard.rank_blocks(blocks, 0, 3) == (0, 2)  # the grown block starts in window 1
    assert shard.rank_blocks(blocks, 3, 7) == (2, 4)
    assert shard.frame_split([10, 10, 10, 10], 2) == [(0, 2), (2, 4)]
    assert shard.frame_split([], 2) == [(0, 0), (0, 0)]
    bits = np.array([0, 1, 1, 0, 0, 1], dtype=bool)
    V = shard.ValidPositions(bits, 6)
    assert [V.pos(k) for k in range(4)] == [1, 2, 5, 6]
    assert list(V.take(np.arange(6), 1, 3)) == [2, 5]


# ---------------------------------------------------------------------------
# Ranks as gloo processes (CPU)
# ---------------------------------------------------------------------------
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        eng = OracleEngine()
        res = {}
        for name, dtype, values, bm in _columns():
            s = shard.compress_column_sharded(values, bm, dtype=dtype, engine=eng)
            d = shard.decompress_column_sharded(s, engine=eng)
            res[name] = (s, d.values.tobytes(), d.validity)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    q.put((rank, res))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_gloo_ranks_match_single_call(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for name, dtype, values, bm in _columns():
        ref = O.compress_column(values, dtype, bm)
        _, rv, rbm, _, _ = O.decompress_column(ref)
        for r in range(world):
            s, vals, validity = got[r][name]
            assert s == ref, (name, r)
            assert vals == np.ascontiguousarray(rv).tobytes(), (name, r)
            assert (validity is None) == (rbm is None)
            if rbm is not None:
                assert validity == bytes(rbm), (name, r)


def test_decimal_columns_are_not_sharded():
    with pytest.raises(Q.Error):
        shard.compress_column_sharded(np.zeros((4, 2), np.int64), dtype=Q.DECIMAL128, engine=OracleEngine())


# ---------------------------------------------------------------------------
# Ranks as host threads (the exchange through a host barrier)
# ---------------------------------------------------------------------------
class ThreadGroup:
    def __init__(self, world):
        self.world = world
        self.barrier = threading.Barrier(world)
        self.slots = [None] * world
        self.local = threading.local()


def _run_threads(world, fn, monkeypatch):
    G = ThreadGroup(world)

    def info(group):
        return (G.local.rank, world) if group is G else (0, 1)

    def gather(data, group=None):
        if group is not G:
            return [bytes(data)]
        G.barrier.wait()
        G.slots[G.local.rank] = bytes(data)
        G.barrier.wait()
        out = list(G.slots)
        G.barrier.wait()
        return out

    monkeypatch.setattr(shard, "_group_info", info)
    monkeypatch.setattr(shard, "all_gather_bytes", gather)
    res, errs = [None] * world, []

    def body(r):
        G.local.rank = r
        try:
            res[r] = fn(G)
        except BaseException as e:  # noqa: BLE001
            errs.append(e)
            G.barrier.abort()

    ts = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout=600)
    if errs:
        raise errs[0]
    return res


def test_sharded_thread_ranks_oracle_engine(monkeypatch):
    eng = OracleEngine()
    for name, dtype, values, bm in _columns():
        ref = O.compress_column(values, dtype, bm)
        outs = _run_threads(4, lambda g: shard.compress_column_sharded(values, bm, dtype=dtype, group=g, engine=eng),
                            monkeypatch)
        assert all(s == ref for s in outs), name
        dec = _run_threads(4, lambda g: shard.decompress_column_sharded(ref, group=g, engine=eng), monkeypatch)
        _, rv, rbm, _, _ = O.decompress_column(ref)
        assert all(d.values.tobytes() == np.ascontiguousarray(rv).tobytes() for d in dec), name


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_cuda_engine_matches_single_call(world, monkeypatch):
    eng = shard.CudaEngine()
    for name, dtype, values, bm in _columns():
        ref = Q.compress_column(values, bm, dtype=dtype)
        assert ref == O.compress_column(values, dtype, bm), name
        outs = _run_threads(world, lambda g: shard.compress_column_sharded(values, bm, dtype=dtype, group=g,
                                                                           engine=eng), monkeypatch)
        assert all(s == ref for s in outs), name
        dec = _run_threads(world, lambda g: shard.decompress_column_sharded(ref, group=g, engine=eng), monkeypatch)
        want = Q.decompress_column(ref)
        for d in dec:
            assert d.values.tobytes() == want.values.tobytes(), name
            assert d.validity == want.validity, name


@pytest.mark.gpu
def test_probe_windows_device_parts_concatenate():
    """Probing a column in window-aligned parts gives the whole column's bytes."""
    rng = np.random.default_rng(3)
    v = rng.integers(0, 2**40, 7 * W + 5, dtype=np.uint64)
    v[W:4 * W] = rng.integers(0, 3, 3 * W).astype(np.uint64)
    eng = shard.CudaEngine()
    whole = eng.probe_windows(v, Q.U64)
    assert list(whole) == list(O.probe_windows(v))
    parts = np.concatenate([eng.probe_windows(v[:3 * W], Q.U64), eng.probe_windows(v[3 * W:], Q.U64)])
    assert list(parts) == list(whole)
