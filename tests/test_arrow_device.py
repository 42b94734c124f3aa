"""The Arrow C Device Data Interface entry points: a device-resident Arrow
array (values and bitmap in GPU memory, any offset) compresses in place to
the same stream as the typed path (src/arrow.rs compress_array semantics,
a sliced bitmap re-packed on the device), honouring the producer's sync
event; an indexed stream decodes into a new device array of the stream's
type whose buffers hold the values, the bitmap and the null count.
"""
import ctypes

import numpy as np
import pytest

from test_arrow import ArrowArray, ArrowSchema

pytestmark = pytest.mark.gpu

P, S = ctypes.c_void_p, ctypes.c_size_t
F64, I64, U64, I32, U32, F32, DEC128 = range(7)
ARROW_DEVICE_CPU, ARROW_DEVICE_CUDA = 1, 2


class ArrowDeviceArray(ctypes.Structure):
    _fields_ = [("array", ArrowArray), ("device_id", ctypes.c_int64), ("device_type", ctypes.c_int32),
                ("sync_event", P), ("reserved", ctypes.c_int64 * 3)]


class _DevBytes:
    """A device range seen through __cuda_array_interface__ (torch wraps it without a copy)."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def _read(torch, ptr, nbytes):
    if nbytes == 0:
        return b""
    return torch.as_tensor(_DevBytes(ptr, nbytes), device="cuda").cpu().numpy().tobytes()


@pytest.fixture(scope="module")
def api(qb):
    L = qb.lib
    L.quoin_b200_compress_arrow_device.argtypes = [P, ctypes.POINTER(ArrowSchema), ctypes.POINTER(ArrowDeviceArray),
                                                   ctypes.POINTER(qb._QuoinConfig), P, S, ctypes.POINTER(S), P]
    L.quoin_b200_compress_arrow_device.restype = ctypes.c_int
    L.quoin_b200_decompress_arrow_device.argtypes = [P, P, P, ctypes.POINTER(ArrowSchema),
                                                     ctypes.POINTER(ArrowDeviceArray), P]
    L.quoin_b200_decompress_arrow_device.restype = ctypes.c_int
    return L


def _arrow_bitmap(valid, offset):
    """Arrow validity bits for `valid` placed from bit `offset`."""
    bits = np.zeros(offset + len(valid), bool)
    bits[offset:] = valid
    return np.packbits(bits, bitorder="little")


def cases():
    rng = np.random.default_rng(9)
    n = 40000
    nulls = rng.random(n + 40) < 0.15
    ts = (1_700_000_000_000 + np.cumsum(rng.poisson(50, n + 40))).astype(np.int64)
    prices = np.floor(rng.random(n + 40) * 1e6 + 0.5) / 100.0
    dec = np.zeros((n + 40, 2), np.int64)
    dec[:, 0] = rng.integers(-10**12, 10**12, n + 40)
    dec[:, 1] = np.where(dec[:, 0] < 0, -1, 0)
    return [
        ("i64_offset3_nulls", "l", I64, ts, 8, 3, nulls, 0, 0),
        ("f64_no_nulls", "g", F64, prices, 8, 0, None, 0, 0),
        ("f32_offset16_nulls", "f", F32, prices.astype(np.float32), 4, 16, nulls, 0, 0),
        ("dec128_offset5_nulls", "d:18,4", DEC128, dec, 16, 5, nulls, 4, 18),
        ("u32_offset7", "I", U32, (np.arange(n + 40) * 7).astype(np.uint32), 4, 7, None, 0, 0),
    ]


@pytest.mark.parametrize("case", cases(), ids=lambda c: c[0])
def test_device_arrow_round_trip(qb, api, case):
    import torch
    torch.cuda.set_device(0)
    name, fmt, dt, vals, w, off, nulls, scale, precision = case
    L = api
    n = 40000
    dv = torch.from_numpy(np.ascontiguousarray(vals).view(np.uint8).reshape(-1).copy()).cuda()
    valid = None if nulls is None else ~nulls[off:off + n]
    db = None if valid is None else torch.from_numpy(_arrow_bitmap(valid, off).copy()).cuda()
    bufs = (P * 2)(db.data_ptr() if db is not None else None, dv.data_ptr())
    side = torch.cuda.Stream()
    ev = torch.cuda.Event()
    ev.record(side)
    handle = P(getattr(ev, "cuda_event", 0) or 0)
    arr = ArrowDeviceArray()
    arr.array.length = n
    arr.array.null_count = 0 if valid is None else int((~valid).sum())
    arr.array.offset = off
    arr.array.n_buffers = 2
    arr.array.buffers = ctypes.cast(bufs, ctypes.POINTER(P))
    arr.device_id = 0
    arr.device_type = ARROW_DEVICE_CUDA
    arr.sync_event = ctypes.addressof(handle) if handle.value else None
    sch = ArrowSchema()
    sch.format = fmt.encode()
    cfg = qb._cfg(qb.Config(level=qb.Level.FAST))
    raw = np.ascontiguousarray(vals).view(np.uint8).reshape(len(vals), -1)[off:off + n].copy()
    bm = None if valid is None else np.packbits(valid, bitorder="little")
    want = qb.compress_column(raw.reshape(-1), bm, qb.Config(level=qb.Level.FAST), dtype=dt, scale=scale,
                              precision=precision)
    cap = qb._stream_bound(dt, n, bm is not None)
    dd = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    olen = S()
    rc = L.quoin_b200_compress_arrow_device(None, ctypes.byref(sch), ctypes.byref(arr), ctypes.byref(cfg),
                                            dd.data_ptr(), cap, ctypes.byref(olen), None)
    assert rc == 0
    got = dd[: olen.value].cpu().numpy().tobytes()
    assert got == want, name

    idx = P()
    assert L.quoin_b200_index_create(None, got, len(got), ctypes.byref(idx)) == 0
    try:
        osch, oarr = ArrowSchema(), ArrowDeviceArray()
        assert L.quoin_b200_decompress_arrow_device(None, idx, dd.data_ptr(), ctypes.byref(osch),
                                                    ctypes.byref(oarr), None) == 0
        assert osch.format.decode() == fmt and oarr.device_type == ARROW_DEVICE_CUDA and not oarr.sync_event
        assert oarr.array.length == n and oarr.array.offset == 0
        assert oarr.array.null_count == (0 if valid is None else int((~valid).sum()))
        b = oarr.array.buffers
        exp = raw.copy()
        if valid is not None:
            exp[~valid] = 0
        assert _read(torch, b[1], n * w) == exp.tobytes(), name
        if valid is not None:
            assert _read(torch, b[0], (n + 7) // 8) == bm.tobytes()
        else:
            assert not b[0]
        release_a = ctypes.CFUNCTYPE(None, ctypes.POINTER(ArrowArray))(oarr.array.release)
        release_s = ctypes.CFUNCTYPE(None, ctypes.POINTER(ArrowSchema))(osch.release)
        release_a(ctypes.byref(oarr.array))
        release_s(ctypes.byref(osch))
        assert not oarr.array.release and not osch.release
    finally:
        L.quoin_b200_index_free(idx)


def test_device_arrow_refusals(qb, api):
    import torch
    L = api
    dv = torch.zeros(64, dtype=torch.uint8, device="cuda")
    bufs = (P * 2)(None, dv.data_ptr())
    arr = ArrowDeviceArray()
    arr.array.length = 8
    arr.array.n_buffers = 2
    arr.array.buffers = ctypes.cast(bufs, ctypes.POINTER(P))
    arr.device_type = ARROW_DEVICE_CPU
    sch = ArrowSchema()
    sch.format = b"l"
    cfg = qb._cfg(qb.Config())
    olen = S()
    dd = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    assert L.quoin_b200_compress_arrow_device(None, ctypes.byref(sch), ctypes.byref(arr), ctypes.byref(cfg),
                                              dd.data_ptr(), 4096, ctypes.byref(olen), None) == -20
    arr.device_type = ARROW_DEVICE_CUDA
    sch.format = b"s"  # int16
    assert L.quoin_b200_compress_arrow_device(None, ctypes.byref(sch), ctypes.byref(arr), ctypes.byref(cfg),
                                              dd.data_ptr(), 4096, ctypes.byref(olen), None) == -22
