"""One column split across GPUs: one process per GPU, ``torch.distributed``
for the exchanges.

Blocks are independent (reference src/encoder.rs:7-8, src/decoder.rs:1-4), so
a column shards at block boundaries:

Encode (``compress_column_sharded``)
  1. The column's valid values are cut into 32,768-value windows and each rank
     takes a contiguous range of windows.  It probes them on its GPU
     (``quoin_b200_probe_windows_device``: the probe of plan_blocks,
     src/encoder.rs:154-178 and 705-750).
  2. One all-gather of the probe bytes (one byte per window); every rank then
     runs plan_blocks as a scan over them on the host (``plan_from_flags``).
  3. A block belongs to the rank whose windows hold its first window.  Each
     rank compresses the valid values of its blocks as one lane with no
     validity: that stream without its 16-byte header is exactly those blocks'
     frames, since a block's frame depends only on its values and the level.
  4. One all-gather of the ranks' frame byte counts gives each rank its offset;
     the frames are gathered in rank order behind the prefix (header and
     validity blob, ``quoin_b200_stream_prefix_device``).

Decode (``decompress_column_sharded``)
  Every rank walks the header, validity blob and frame table on the host
  (src/decoder.rs:43-118), cuts the frames into contiguous ranges of about
  equal value count, and decodes its range as a stream of its own: the header
  for its output positions, the validity bits of those positions, its frames.
  Rank r's output positions start at the position of its first frame's first
  valid value (the valid-count prefix of the walk); the ranks' ranges are
  disjoint and are gathered in rank order.

The exchanges are all-gathers of byte tensors (NCCL over NVLink when the
process group is NCCL, gloo on CPU).  Decimal columns (a container of limb
streams) are not sharded: ``Error(QUOIN_ERR_UNSUPPORTED)``.

The per-rank compute goes through an engine: ``CudaEngine`` (the default)
runs it on this process's GPU through the C ABI.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import (DECIMAL128, DECIMAL256, Config, DecodedColumn, Error, _FROM_NP, _NP, _bitmap, _cfg,
               _check, compress_column, decompress_column, lib)

BASE_QUANTUM = 32768   # reference src/encoder.rs: BASE_QUANTUM
MAX_QUANTUM = 131072   # reference src/encoder.rs: MAX_QUANTUM
ERR_UNSUPPORTED = -18
ERR_CORRUPT = -3
ERR_TRUNCATED = -12
ERR_BAD_MAGIC = -10


# ---------------------------------------------------------------------------
# Host-side plan and partition
# ---------------------------------------------------------------------------
def window_split(n_windows: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous window ranges, one per rank, sizes differing by at most one."""
    return [(n_windows * r // world, n_windows * (r + 1) // world) for r in range(world)]


def plan_from_flags(flags: Sequence[int], n_lane: int) -> List[Tuple[int, int]]:
    """plan_blocks (reference src/encoder.rs:154-178) from the probe bytes of
    every 32,768-value window: a block starts at a window and covers it, or
    four windows when the window's probe byte is set (clipped at the lane's
    end).  Probe bytes of windows inside a grown block are not read, as
    plan_blocks never probes them."""
    blocks = []
    start = 0
    while start < n_lane:
        w = start // BASE_QUANTUM
        end = min(start + (MAX_QUANTUM if flags[w] else BASE_QUANTUM), n_lane)
        blocks.append((start, end))
        start = end
    return blocks


def rank_blocks(blocks: Sequence[Tuple[int, int]], wa: int, wb: int) -> Tuple[int, int]:
    """The blocks [ba, bb) whose first window lies in windows [wa, wb)."""
    firsts = np.fromiter((s // BASE_QUANTUM for s, _ in blocks), dtype=np.int64, count=len(blocks))
    return int(np.searchsorted(firsts, wa, "left")), int(np.searchsorted(firsts, wb, "left"))


def frame_split(frame_ns: Sequence[int], world: int) -> List[Tuple[int, int]]:
    """Contiguous frame ranges of about equal value count, one per rank: rank
    r starts at the first frame whose values begin at or after r/world of the
    total."""
    ends = np.cumsum(np.asarray(frame_ns, dtype=np.int64))
    starts = ends - np.asarray(frame_ns, dtype=np.int64)
    total = int(ends[-1]) if len(ends) else 0
    cuts = [0] + [int(np.searchsorted(starts, (total * r + world - 1) // world, "left")) for r in range(1, world)]
    cuts.append(len(frame_ns))
    for r in range(1, world + 1):  # monotone
        cuts[r] = max(cuts[r], cuts[r - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


class ValidPositions:
    """Lane index <-> position over an LSB-first bitmap of n bits."""

    def __init__(self, bits: Optional[np.ndarray], n: int):
        self.n = n
        self.bits = bits  # bool per position, or None (all valid)
        if bits is not None:
            self.cum = np.cumsum(bits, dtype=np.int64)
            self.nv = int(self.cum[-1]) if n else 0
        else:
            self.nv = n

    def pos(self, k: int) -> int:
        """Position of the k-th valid value (0-based); n when k == valid count."""
        if k >= self.nv:
            return self.n
        if self.bits is None:
            return k
        return int(np.searchsorted(self.cum, k + 1, "left"))

    def take(self, arr: np.ndarray, la: int, lb: int) -> np.ndarray:
        """The valid values with lane indices [la, lb)."""
        if self.bits is None:
            return arr[la:lb]
        pa, pb = self.pos(la), self.pos(lb)
        return arr[pa:pb][self.bits[pa:pb]]


def _bits(bm: Optional[np.ndarray], n: int) -> Optional[np.ndarray]:
    if bm is None:
        return None
    return np.unpackbits(bm[: (n + 7) // 8], bitorder="little")[:n].astype(bool)


# ---------------------------------------------------------------------------
# Host stream walk (reference src/format.rs:65-94, src/decoder.rs:43-118)
# ---------------------------------------------------------------------------
def _varint(s: bytes, pos: int) -> Tuple[int, int]:
    v = 0
    for k in range(10):
        if pos + k >= len(s):
            raise Error(ERR_TRUNCATED)
        b = s[pos + k]
        v |= (b & 0x7F) << (7 * k)
        if not b & 0x80:
            return v, pos + k + 1
    raise Error(ERR_CORRUPT)


def _put_varint(v: int) -> bytes:
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        if v:
            out.append(b | 0x80)
        else:
            out.append(b)
            return bytes(out)


class StreamLayout:
    """Header fields, validity bits and frame table of a non-decimal stream."""

    def __init__(self, s: bytes):
        if len(s) < 16:
            raise Error(ERR_TRUNCATED)
        if s[:4] != b"FCR1":
            raise Error(ERR_BAD_MAGIC)
        if s[5] & 2:
            raise Error(ERR_UNSUPPORTED)  # decimal container
        self.head = bytes(s[:16])
        self.dtype = s[7]
        self.n = int.from_bytes(s[8:16], "little")
        self.bits = None
        pos = 16
        if s[5] & 1:
            vlen, pos = _varint(s, pos)
            if vlen == 0 or pos + vlen > len(s):
                raise Error(ERR_TRUNCATED)
            self.bits = _decode_validity(s[pos:pos + vlen], self.n)
            pos += vlen
        self.positions = ValidPositions(self.bits, self.n)
        # frames: [mode u8][n u32][plen u32][payload], until the lane's count
        self.frames = []  # (offset, n)
        total = 0
        while total < self.positions.nv:
            if pos + 9 > len(s):
                raise Error(ERR_TRUNCATED)
            fn = int.from_bytes(s[pos + 1:pos + 5], "little")
            plen = int.from_bytes(s[pos + 5:pos + 9], "little")
            if fn == 0 or pos + 9 + plen > len(s):
                raise Error(ERR_CORRUPT)
            self.frames.append((pos, fn))
            total += fn
            pos += 9 + plen
        if total != self.positions.nv:
            raise Error(ERR_CORRUPT)
        self.end = pos


def _decode_validity(blob: bytes, n: int) -> np.ndarray:
    """Validity blob -> bool per position (reference src/validity.rs:73-119)."""
    tag = blob[0]
    if tag == 0:
        raw = (n + 7) // 8
        if len(blob) - 1 < raw:
            raise Error(ERR_TRUNCATED)
        return np.unpackbits(np.frombuffer(blob[1:1 + raw], np.uint8), bitorder="little")[:n].astype(bool)
    if tag != 1:
        raise Error(ERR_CORRUPT)
    bits = np.zeros(n, dtype=bool)
    i, cur, pos = 0, 0, 1
    while i < n:
        run, pos = _varint(blob, pos)
        if i + run > n:
            raise Error(ERR_CORRUPT)
        if cur:
            bits[i:i + run] = True
        i += run
        cur ^= 1
    return bits


def sub_stream(L: StreamLayout, s: bytes, fa: int, fb: int, pa: int, pb: int) -> bytes:
    """A stream of its own for frames [fa, fb) decoding positions [pa, pb)."""
    n = pb - pa
    head = bytearray(L.head)
    head[8:16] = n.to_bytes(8, "little")
    out = [bytes(head)]
    if L.bits is not None:
        raw = np.packbits(L.bits[pa:pb], bitorder="little").tobytes()
        blob = b"\x00" + raw
        out.append(_put_varint(len(blob)) + blob)
    if fb > fa:
        a = L.frames[fa][0]
        b = L.frames[fb][0] if fb < len(L.frames) else L.end
        out.append(bytes(s[a:b]))
    return b"".join(out)


# ---------------------------------------------------------------------------
# Engines: the per-rank compute
# ---------------------------------------------------------------------------
class CudaEngine:
    """Probe, prefix, compress and decode on this process's GPU (C ABI)."""

    def __init__(self, device: Optional[int] = None, ctx=None):
        import torch
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self.ctx = ctx

    def _dev(self, a: np.ndarray):
        t = self.torch
        return t.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).to(self.device)

    def probe_windows(self, values: np.ndarray, dtype: int) -> np.ndarray:
        n = len(values)
        nwin = (n + BASE_QUANTUM - 1) // BASE_QUANTUM
        flags = np.zeros(max(nwin, 1), dtype=np.uint8)
        if n == 0:
            return flags[:0]
        dv = self._dev(values)
        got = ctypes.c_uint64()
        with self.torch.cuda.device(self.device):
            _check(lib.quoin_b200_probe_windows_device(self.ctx, dtype, n, dv.data_ptr(), None, flags.ctypes.data,
                                                        flags.size, ctypes.byref(got), None))
        return flags[: got.value]

    def prefix(self, n: int, dtype: int, validity: Optional[np.ndarray], cfg: Optional[Config]) -> bytes:
        cap = 16 + 16 + (n + 7) // 8 + 64
        dst = self.torch.empty(cap, dtype=self.torch.uint8, device=self.device)
        db = self._dev(validity) if validity is not None and n else None
        olen = ctypes.c_size_t()
        c = _cfg(cfg)
        with self.torch.cuda.device(self.device):
            _check(lib.quoin_b200_stream_prefix_device(self.ctx, dtype, n, None if db is None else db.data_ptr(),
                                                        ctypes.byref(c), dst.data_ptr(), cap, ctypes.byref(olen),
                                                        None))
        return dst[: olen.value].cpu().numpy().tobytes()

    def compress_lane(self, values: np.ndarray, dtype: int, cfg: Optional[Config]) -> bytes:
        with self.torch.cuda.device(self.device):
            return compress_column(values, None, cfg, dtype=dtype, ctx=self.ctx)

    def decompress(self, stream: bytes) -> DecodedColumn:
        with self.torch.cuda.device(self.device):
            return decompress_column(stream, ctx=self.ctx)


# ---------------------------------------------------------------------------
# Exchanges
# ---------------------------------------------------------------------------
def _group_info(group):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def _comm_device(group):
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def all_gather_bytes(data: bytes, group=None) -> List[bytes]:
    """Every rank's bytes, in rank order: an all-gather of the lengths, then
    one of the buffers padded to the longest."""
    import torch
    import torch.distributed as dist
    rank, world = _group_info(group)
    if world == 1:
        return [bytes(data)]
    dev = _comm_device(group)
    ln = torch.tensor([len(data)], dtype=torch.int64, device=dev)
    lens = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(lens, ln, group=group)
    sizes = [int(x.item()) for x in lens]
    cap = max(max(sizes), 1)
    buf = torch.zeros(cap, dtype=torch.uint8, device=dev)
    if data:
        buf[: len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8).to(dev)
    outs = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    return [o[:sz].cpu().numpy().tobytes() for o, sz in zip(outs, sizes)]


# ---------------------------------------------------------------------------
# Entry points
# ---------------------------------------------------------------------------
def _frames_n(stream: bytes) -> List[int]:
    L = StreamLayout(stream)
    return [fn for _, fn in L.frames]


def compress_column_sharded(values, validity=None, cfg: Optional[Config] = None, dtype: Optional[int] = None,
                            group=None, engine=None) -> bytes:
    """compress_column over every rank of ``group`` (each rank passes the same
    column); returns the whole stream, equal to compress_column's, on every
    rank."""
    arr = np.ascontiguousarray(values)
    if dtype is None:
        dtype = _FROM_NP.get(arr.dtype)
        if dtype is None:
            raise TypeError(f"unsupported column dtype {arr.dtype}")
    if dtype in (DECIMAL128, DECIMAL256):
        raise Error(ERR_UNSUPPORTED)
    arr = arr.view(_NP[dtype]).reshape(-1)
    n = arr.size
    bm = _bitmap(validity, n)
    eng = engine or CudaEngine()
    rank, world = _group_info(group)
    bits = _bits(bm, n)
    V = ValidPositions(bits, n)
    nwin = (V.nv + BASE_QUANTUM - 1) // BASE_QUANTUM
    wa, wb = window_split(nwin, world)[rank]
    mine = V.take(arr, wa * BASE_QUANTUM, min(wb * BASE_QUANTUM, V.nv))
    flags = eng.probe_windows(mine, dtype) if len(mine) else np.zeros(0, np.uint8)
    if len(flags) != wb - wa:
        raise Error(-4)
    all_flags = np.frombuffer(b"".join(all_gather_bytes(flags.tobytes(), group)), dtype=np.uint8)
    blocks = plan_from_flags(all_flags, V.nv)
    ba, bb = rank_blocks(blocks, wa, wb)
    frames = b""
    if bb > ba:
        la, lb = blocks[ba][0], blocks[bb - 1][1]
        part = eng.compress_lane(V.take(arr, la, lb), dtype, cfg)
        if _frames_n(part) != [e - s for s, e in blocks[ba:bb]]:
            raise Error(-4)  # the part's plan must be the column's
        frames = part[16:]
    prefix = eng.prefix(n, dtype, bm, cfg) if rank == 0 else b""
    parts = all_gather_bytes(prefix + frames, group)
    return b"".join(parts)


def decompress_column_sharded(stream: bytes, group=None, engine=None) -> DecodedColumn:
    """decompress_column over every rank of ``group`` (each rank passes the
    same stream); returns the whole column on every rank."""
    eng = engine or CudaEngine()
    rank, world = _group_info(group)
    L = StreamLayout(stream)
    split = frame_split([fn for _, fn in L.frames], world)
    fa, fb = split[rank]
    lane_start = np.concatenate([[0], np.cumsum([fn for _, fn in L.frames], dtype=np.int64)])
    # output positions: from the first valid value of the rank's first frame
    # (rank 0 from 0) to the next rank's start
    starts = [0] + [L.positions.pos(int(lane_start[split[r][0]])) for r in range(1, world)] + [L.n]
    pa, pb = starts[rank], starts[rank + 1]
    part = eng.decompress(sub_stream(L, stream, fa, fb, pa, pb))
    if len(part.values) != pb - pa:
        raise Error(ERR_CORRUPT)
    parts = all_gather_bytes(np.ascontiguousarray(part.values).view(np.uint8).tobytes(), group)
    vals = np.frombuffer(b"".join(parts), dtype=np.uint8).view(_NP[L.dtype]).copy()
    if len(vals) != L.n:
        raise Error(ERR_CORRUPT)
    validity = None if L.bits is None else np.packbits(L.bits, bitorder="little").tobytes()
    return DecodedColumn(vals, validity, L.dtype)
