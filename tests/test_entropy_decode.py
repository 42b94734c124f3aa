"""Decode of streams with entropy-coded parts (Level::Balanced).

Streams written at Balanced carry rANS-coded parts (reference
src/entropy/mod.rs:152-178, src/entropy/rans.rs:110-175) inside
BYTE_TRANSPOSE frames, FLOAT_MULT frames of tag 1, ALP-RD frames whose codes
or rights carry tag 1, and DICT frames whose values carry tag 2 (transposed
byte planes) or whose codes carry tag 1 (byte planes).  The oracle writes
such streams (its Balanced in-pool encoder, oracle/quoin_oracle.c
encode_block); the GPU decoder must return the oracle's values, and the
oracle's error kinds on damaged copies.

The first test (CPU only) pins the cases: every tag combination above occurs
in at least one of them, so the GPU tests below cover each decode branch.
"""
import ctypes

import numpy as np
import pytest

from conftest import bitmap_from_bools, lcg1_seq, lcg_seq

F64, I64, U64, I32, U32, F32, DEC128 = 0, 1, 2, 3, 4, 5, 6
LEVEL_BALANCED = 2


def _varint(b, pos):
    r, sh = 0, 0
    while True:
        x = b[pos]
        pos += 1
        r |= (x & 0x7F) << sh
        if not x & 0x80:
            return r, pos
        sh += 7


def _frames(s, pos=16):
    """(mode, n, payload) of a plain stream's frames (format.rs:65-94)."""
    if s[5] & 1:
        vl, pos = _varint(s, pos)
        pos += vl
    out = []
    while pos < len(s):
        m = s[pos]
        fn = int.from_bytes(s[pos + 1:pos + 5], "little")
        pl = int.from_bytes(s[pos + 5:pos + 9], "little")
        out.append((m, fn, s[pos + 9:pos + 9 + pl], pos + 9))
        pos += 9 + pl
    return out


def _lane_streams(s):
    """The lane streams of a stream: itself, or a decimal container's lanes (decimal.rs:100-168)."""
    if not s[5] & 2:
        return [(s, 0)]
    nl = s[18]
    pos = 19 + 8 * nl
    if s[5] & 1:
        vl, pos = _varint(s, pos)
        pos += vl
    lanes = []
    for _ in range(nl):
        sl, pos = _varint(s, pos)
        lanes.append((s[pos:pos + sl], pos))
        pos += sl
    return lanes


def frame_tags(s):
    """Entropy-relevant tags of every frame, e.g. ("DICT", values tag, codes tag)."""
    tags = []
    for lane, _ in _lane_streams(s):
        for m, _, p, _ in _frames(lane):
            if m == 11:
                tags.append(("BT",))
            elif m == 17:
                tags.append(("FM", p[0]))
            elif m == 52:
                pos = 2 + 8 * p[1]
                nexc, pos = _varint(p, pos)
                for _ in range(nexc):
                    _, pos = _varint(p, pos)
                    pos += 8
                ct = p[pos]
                cl, pos = _varint(p, pos + 1)
                tags.append(("RD", ct, p[pos + cl], nexc > 0))
            elif m == 19:
                _, pos = _varint(p, 0)
                vt = p[pos]
                vl, pos = _varint(p, pos + 1)
                ct = p[pos + vl]
                nb = p[pos + vl + 1] if ct == 1 else 0
                tags.append(("DICT", vt, ct, nb))
    return tags


def _geobytes(rng, prob, n, nb=8):
    """u64 values whose bytes are independently geometric: byte planes of low entropy."""
    b = np.minimum(rng.geometric(prob, (n, nb)) - 1, 255).astype(np.uint64)
    return (b << (np.arange(nb, dtype=np.uint64) * np.uint64(8))).sum(axis=1, dtype=np.uint64)


def _dec128(v):
    v = np.asarray(v, np.int64)
    out = np.zeros((v.size, 16), np.uint8)
    out[:, :8] = v.view(np.uint8).reshape(-1, 8)
    out[:, 8:] = np.where(v < 0, 255, 0)[:, None]
    return out


def entropy_cases():
    """(name, values, wire dtype, bitmap, scale, precision)."""
    rng = np.random.default_rng(20240611)
    n = 60000
    pool = lcg_seq(31, 3000) >> np.uint64(8)
    dict16 = np.unique(_geobytes(rng, 0.6, 400))[:16]
    u12 = rng.random(150000) + 1.0
    u12[rng.integers(0, 150000, 1500)] = rng.random(1500) * 1e6
    vb = rng.random(150000) > 0.2
    c = [
        ("bt_geo03", _geobytes(rng, 0.3, n, 6), U64, None),
        ("bt_geo02_i64", _geobytes(rng, 0.2, 200000, 6).astype(np.int64), I64, None),
        ("fm_ramp", np.arange(10000) * 0.5, F64, None),
        ("fm_walk", np.round(np.cumsum(rng.standard_normal(n)), 3), F64, None),
        ("rd_codes_ent_exc", np.sin(np.arange(40000) * 0.01), F64, None),
        ("rd_both_ent_exc", rng.random(n), F64, None),
        ("rd_rights_ent_f32", np.arange(8192, dtype=np.float32) * np.float32(0.01) + np.float32(5.0), F32, None),
        ("rd_nullable", u12, F64, bitmap_from_bools(vb)),
        ("dict_raw_vals_code_planes", rng.integers(0, 16, n).astype(np.int64) * 1000003, I64, None),
        ("dict_delta_vals_two_planes", pool[(lcg1_seq(32, 40000) >> np.uint64(40)) % 1800], U64, None),
        ("dict_big_two_planes", (lcg_seq(35, 17000) >> np.uint64(8))[(lcg1_seq(36, 32768) >> np.uint64(40)) % 17000],
         U64, None),
        ("dict_bt_vals_one_plane", np.unique(_geobytes(rng, 0.6, 400))[:64][lcg1_seq(6, n) >> np.uint64(58)], U64,
         None),
        ("dict_bt_vals_two_planes", _geobytes(rng, 0.6, 4096)[lcg1_seq(6, n) >> np.uint64(52)], U64, None),
        ("dict_bt_vals_packed_codes", dict16[lcg1_seq(6, 3000) >> np.uint64(60)], U64, None),
        ("dict_nullable_f32", (np.round(rng.normal(25, 5, 150000) * 10) / 10).astype(np.float32), F32,
         bitmap_from_bools(vb)),
        ("dict_i32", (pool[(lcg1_seq(34, 50000) >> np.uint64(40)) % 2500] >> np.uint64(32)).astype(np.uint32)
         .view(np.int32), I32, None),
    ]
    cases = [(name, v, dt, bm, 0, 0) for name, v, dt, bm in c]
    cases.append(("dec128_lanes", _dec128(rng.integers(0, 40, n) * 1_000_000_007 - 20_000_000_000), DEC128, None,
                  4, 30))
    return cases


REQUIRED_TAGS = {
    ("BT",), ("FM", 1),
    ("RD", 1, 0, True), ("RD", 1, 1, True), ("RD", 0, 1, False),
    ("DICT", 0, 1, 1), ("DICT", 1, 1, 2), ("DICT", 2, 1, 1), ("DICT", 2, 1, 2), ("DICT", 2, 0, 0),
}


def test_entropy_cases_cover_every_tag(oracle):
    seen = set()
    for name, v, dt, bm, sc, pr in entropy_cases():
        seen.update(frame_tags(oracle.compress_column(v, dt, bm, level=LEVEL_BALANCED, scale=sc, precision=pr)))
    assert REQUIRED_TAGS <= seen, sorted(REQUIRED_TAGS - seen)


def _expected(v, dt, bm):
    w = {F64: 8, I64: 8, U64: 8, I32: 4, U32: 4, F32: 4, DEC128: 16}[dt]
    raw = np.ascontiguousarray(v).view(np.uint8).reshape(-1, w).copy()
    if bm is not None:
        valid = np.unpackbits(np.asarray(bm, np.uint8), bitorder="little")[:raw.shape[0]].astype(bool)
        raw[~valid] = 0
    return raw.tobytes()


def _dec_bytes(d):
    return np.ascontiguousarray(d.values).view(np.uint8).tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("case", entropy_cases(), ids=lambda c: c[0])
def test_entropy_streams_decode(qb, oracle, case):
    name, v, dt, bm, sc, pr = case
    s = oracle.compress_column(v, dt, bm, level=LEVEL_BALANCED, scale=sc, precision=pr)
    d = qb.decompress_column(s)
    assert _dec_bytes(d) == _expected(v, dt, bm)
    od = oracle.decompress_column(s)
    assert _dec_bytes(d) == np.ascontiguousarray(od[1]).view(np.uint8).tobytes()
    # twice through one context: the entropy areas are reused
    assert _dec_bytes(qb.decompress_column(s)) == _expected(v, dt, bm)


def _outcome(fn, err):
    try:
        return "ok", fn()
    except err as e:
        return e.kind, None


def _agree(qb, oracle, b):
    ok, od = _outcome(lambda: oracle.decompress_column(b), oracle.OracleError)
    gk, gd = _outcome(lambda: qb.decompress_column(b), qb.Error)
    assert gk == ok
    if gk == "ok":
        assert _dec_bytes(gd) == np.ascontiguousarray(od[1]).view(np.uint8).tobytes()
    return gk


@pytest.mark.gpu
def test_rans_part_errors_match_oracle(qb, oracle):
    """Targeted damage to the first rANS part of a BYTE_TRANSPOSE frame."""
    rng = np.random.default_rng(3)
    s = oracle.compress_column(_geobytes(rng, 0.3, 5000, 6), U64, level=LEVEL_BALANCED)
    (m, fn, p, off), = _frames(s)
    assert m == 11 and p[0] == 2
    kinds = []
    # tag 0 re-reads the rANS bytes as range-coder input, which only fails on
    # its declared length (here the same n, so both decoders give the same
    # garbage values); tag 1 reads them as a tANS header, whose weights do not
    # sum to 1024; tag 3 reads them as an LZ cascade, whose inner stream fails;
    # others -> CorruptPayload
    for tag in (0, 1, 3, 4, 255):
        b = bytearray(s)
        b[off] = tag
        kinds.append(_agree(qb, oracle, bytes(b)))
    assert kinds == ["ok"] + ["CorruptPayload"] * 4
    _, n_end = _varint(p, 1)  # payload offset of varint(number of symbols)
    b = bytearray(s)
    b[off + n_end] = 0  # zero symbols
    assert _agree(qb, oracle, bytes(b)) == "CorruptPayload"
    for k in range(1, 6):  # the frequency table: symbols and frequencies
        b = bytearray(s)
        b[off + n_end + k] ^= 0x05
        _agree(qb, oracle, bytes(b))
    for cut in (off + 1, off + n_end + 1, off + len(p) - 1, off + len(p) // 2):
        assert _agree(qb, oracle, s[:cut]) != "ok"  # truncated stream
    # truncated payload inside a well-formed frame: shrink plen by one
    b = bytearray(s)
    b[off - 4:off] = (len(p) - 1).to_bytes(4, "little")
    _agree(qb, oracle, bytes(b[:-1]))


@pytest.mark.gpu
def test_entropy_mutations_agree_with_oracle(qb, oracle):
    rng = np.random.default_rng(0x2468ACE0)
    g = np.random.default_rng(8)
    seeds = [oracle.compress_column(v, dt, level=LEVEL_BALANCED) for v, dt in (
        (_geobytes(g, 0.3, 3000, 6), U64),
        (np.arange(4000) * 0.5, F64),
        (np.sin(np.arange(4000) * 0.01), F64),
        (g.random(3000), F64),
        (np.arange(3000, dtype=np.float32) * np.float32(0.01) + np.float32(5.0), F32),
        (g.integers(0, 16, 4000).astype(np.int64) * 1000003, I64),
        ((lcg_seq(31, 900) >> np.uint64(8))[(lcg1_seq(32, 4000) >> np.uint64(40)) % 700], U64),
        (np.unique(_geobytes(g, 0.6, 400))[:16][lcg1_seq(6, 3000) >> np.uint64(60)], U64),
        (_geobytes(g, 0.6, 600)[(lcg1_seq(6, 4000) >> np.uint64(40)) % 600], U64))]
    covered = set()
    for s in seeds:
        covered.update(frame_tags(s))
    assert {("BT",), ("FM", 1), ("DICT", 2, 0, 0)} <= covered, covered
    kinds = {}
    for it in range(1200):
        b = bytearray(seeds[rng.integers(len(seeds))])
        for _ in range(1 + rng.integers(3)):
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
        k = _agree(qb, oracle, bytes(b))
        kinds[k] = kinds.get(k, 0) + 1
    assert len(kinds) >= 3, kinds


@pytest.mark.gpu
def test_noalloc_rejects_entropy_frames(qb, oracle):
    import torch
    L = qb.lib
    P = ctypes.c_void_p
    L.quoin_b200_decompress_device_noalloc.argtypes = [P, ctypes.c_size_t, P, ctypes.c_size_t,
                                                       ctypes.POINTER(ctypes.c_uint64), P]
    L.quoin_b200_decompress_device_noalloc.restype = ctypes.c_int
    torch.cuda.set_device(0)
    rng = np.random.default_rng(4)
    s = oracle.compress_column(_geobytes(rng, 0.3, 5000, 6), U64, level=LEVEL_BALANCED)
    d_src = torch.from_numpy(np.frombuffer(s, np.uint8).copy()).cuda()
    d_out = torch.zeros(5000, dtype=torch.int64, device="cuda")
    n = ctypes.c_uint64(0)
    rc = L.quoin_b200_decompress_device_noalloc(P(d_src.data_ptr()), len(s), P(d_out.data_ptr()), 5000,
                                                ctypes.byref(n), P(torch.cuda.current_stream().cuda_stream))
    assert rc == -21  # QUOIN_ERR_NOALLOC_LIMIT
