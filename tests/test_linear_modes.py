"""High / Max residual modes: ORDERED_DELTA (7), DELTA2 (20) and DELTA_DP (45)
from src/codecs/linear.rs, PRED (0), PRED_RC (29) and PRED2 (25) from
src/codecs/pred.rs with the CRC32C predictor hash (src/hash.rs), with residual
bytes coded by the range coder (src/entropy/rc.rs, tag 0) or rANS (tag 2), and
the range coder inside other entropy-coded parts; LZ (4) and the Max LZ cascade
(entropy tag 3) from src/codecs/lz.rs.  The oracle restates the encoders and decoders (its CPU
checks port the reference's tests: rc.rs roundtrip_random_bytes /
roundtrip_skewed_bytes / empty, linear.rs float_delta_roundtrips_all_orders /
idelta2_roundtrips / select_order_prefers_high_on_smooth_low_on_noise); the
GPU decode must give the oracle's values, and the oracle's error kinds on
damaged payloads.
"""
import numpy as np
import pytest

from conftest import lcg_seq

F64, I64, U64 = 0, 1, 2
M_OD, M_D2, M_DP, M_BT = 7, 20, 45, 11
TAG_RC, TAG_RANS = 0, 2


def stream(frames, dtype=F64):
    """A stream around raw frame payloads: [(mode, n, payload)]."""
    n = sum(f[1] for f in frames)
    out = bytearray(b"FCR1" + bytes([2, 0, 16, dtype]) + n.to_bytes(8, "little"))
    for mode, k, p in frames:
        out += bytes([mode]) + k.to_bytes(4, "little") + len(p).to_bytes(4, "little") + p
    return bytes(out)


def lanes():
    rng = np.random.default_rng(31)
    i = np.arange(20000, dtype=np.float64)
    walk = np.cumsum(rng.normal(0, 1e-3, 20000)) + 20.0
    special = (i * 0.25).copy()
    special[[5, 6, 700, 701, 702, 9000]] = [np.nan, np.inf, -np.inf, np.nan, -0.0, 1e308]
    return {
        "ramp_half": (i * 0.5).view(np.uint64),
        "parabola": (0.5 * i * i).view(np.uint64),
        "sine": (np.sin(i * 0.002) * 100.0 + i * 0.01).view(np.uint64),
        "walk": walk.view(np.uint64),
        "specials": special.view(np.uint64),
        "int_wrap": (np.arange(20000, dtype=np.uint64) * np.uint64(3) - np.uint64(7)),
        "random": lcg_seq(5, 20000),
    }


def test_oracle_range_coder_and_linear_round_trips(oracle):
    data = bytes((lcg_seq(1, 50000) >> np.uint64(33)).astype(np.uint8))
    assert oracle.rc_decompress(oracle.rc_compress(data), len(data)) == data
    s = lcg_seq(7, 50000)
    skew = np.where(s % np.uint64(16) == 0, (s >> np.uint64(40)).astype(np.uint8), 0).astype(np.uint8).tobytes()
    packed = oracle.rc_compress(skew)
    assert len(packed) < len(skew) and oracle.rc_decompress(packed, len(skew)) == skew
    assert oracle.rc_decompress(oracle.rc_compress(b""), 0) == b""
    lv = lanes()
    for name, v in lv.items():
        for mode in (M_OD, M_D2, M_DP):
            for order in (0, 1, 2, 3, 4):
                for tag in (TAG_RC, TAG_RANS):
                    p = oracle.linear_payload(mode, v, order, tag)
                    if p is None:
                        assert mode == M_DP
                        continue
                    assert np.array_equal(oracle.decode_mode(mode, p, len(v)), v), (name, mode, order, tag)
    assert oracle.linear_select_order(lv["sine"]) >= 3
    assert oracle.linear_select_order(lv["random"]) <= 2


def _agree(qb, oracle, s):
    try:
        want = ("ok", oracle.decompress_column(s))
    except oracle.OracleError as e:
        want = (e.kind, None)
    try:
        got = ("ok", qb.decompress_column(s))
    except qb.Error as e:
        got = (e.kind, None)
    assert got[0] == want[0]
    if got[0] == "ok":
        assert np.ascontiguousarray(got[1].values).view(np.uint8).tobytes() == \
            np.ascontiguousarray(want[1][1]).view(np.uint8).tobytes()
    return got[0]


@pytest.mark.gpu
def test_linear_modes_decode_like_the_oracle(qb, oracle):
    cases = 0
    for name, v in lanes().items():
        for mode in (M_OD, M_D2, M_DP):
            for order, tag in ((0, TAG_RC), (1, TAG_RANS), (2, TAG_RC), (3, TAG_RANS), (4, TAG_RC)):
                frames = []
                for lo, hi in ((0, 1), (1, 4097), (4097, 20000)):  # warm-up edge, a mid frame, a long one
                    p = oracle.linear_payload(mode, v[lo:hi], order, tag)
                    if p is None:
                        break
                    frames.append((mode, hi - lo, p))
                if len(frames) < 3:
                    continue
                dt = U64 if mode == M_OD else F64
                s = stream(frames, dt)
                assert _agree(qb, oracle, s) == "ok", (name, mode, order, tag)
                d = qb.decompress_column(s)
                assert np.ascontiguousarray(d.values).view(np.uint64).tobytes() == v.tobytes(), (name, mode)
                cases += 1
    assert cases >= 60


@pytest.mark.gpu
def test_range_coded_parts_of_other_modes(qb, oracle):
    v = lanes()["walk"][:5000]
    soa = np.ascontiguousarray(v).view(np.uint8).reshape(-1, 8).T.copy().tobytes()  # byte planes
    p = bytes([TAG_RC]) + oracle.rc_compress(soa)
    s = stream([(M_BT, len(v), p)])
    assert _agree(qb, oracle, s) == "ok"
    assert np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64).tobytes() == v.tobytes()


@pytest.mark.gpu
def test_damaged_linear_payloads_match_oracle(qb, oracle):
    v = lanes()["sine"][:3000]
    kinds = {}
    for mode in (M_D2, M_DP, M_OD):
        for tag in (TAG_RC, TAG_RANS):
            good = oracle.linear_payload(mode, v, 2, tag)
            res = (oracle.rc_decompress(good[1:], 10 * len(v) + 16) if tag == TAG_RC
                   else oracle.rans_decompress(good[1:], 10 * len(v) + 16))
            variants = {
                "empty": b"",
                "tag1": b"\x01" + good[1:],
                "tag3": b"\x03" + good[1:],
                "tag9": b"\x09" + good[1:],
                "cut": good[: len(good) // 2],
                "trailing": bytes([tag]) + (oracle.rc_compress(res + b"\x00") if tag == TAG_RC
                                            else oracle.rans_compress(res + b"\x00")),
                "short": bytes([tag]) + (oracle.rc_compress(res[:-3]) if tag == TAG_RC
                                         else oracle.rans_compress(res[:-3])),
            }
            if mode != M_OD:
                for o in (0, 5):
                    r2 = bytes([o]) + res[1:]
                    variants[f"order{o}"] = bytes([tag]) + (oracle.rc_compress(r2) if tag == TAG_RC
                                                            else oracle.rans_compress(r2))
            for k, p in variants.items():
                kinds[(mode, tag, k)] = _agree(qb, oracle, stream([(mode, len(v), p)]))
    assert kinds[(M_D2, TAG_RC, "order0")] == "CorruptPayload"
    assert kinds[(M_D2, TAG_RC, "trailing")] == "CorruptPayload"
    assert kinds[(M_DP, TAG_RANS, "tag1")] == "CorruptPayload"  # rANS bytes read as a tANS header
    assert kinds[(M_OD, TAG_RC, "empty")] == "Truncated"


M_PRED, M_PRED2, M_PRED_RC = 0, 25, 29


def _crc32c_u64(crc, v):
    for _ in range(8):
        crc ^= v & 0xFF
        v >>= 8
        for _ in range(8):
            crc = (crc >> 1) ^ (0x82F63B78 if crc & 1 else 0)
    return crc


def test_oracle_predictor_hash_and_round_trips(oracle):
    for v in [0, 1, 42, 255, 256, 2**64 - 1, 0x0102030405060708] + [int(x) for x in lcg_seq(3, 50)]:
        assert oracle.crc32c_u64(0x9E3779B9, v) == _crc32c_u64(0x9E3779B9, v)
    for name, v in lanes().items():
        for mode in (M_PRED, M_PRED_RC, M_PRED2):
            for plog2 in (10, 16):
                for tag in (TAG_RC, TAG_RANS):
                    p = oracle.pred_payload(mode, v, plog2, tag)
                    s = stream([(mode, len(v), p)], U64)
                    s = s[:6] + bytes([plog2]) + s[7:]
                    got = oracle.decompress_column(s)[1]
                    assert np.ascontiguousarray(got).view(np.uint64).tobytes() == v.tobytes(), (name, mode)


@pytest.mark.gpu
def test_predictor_modes_decode_like_the_oracle(qb, oracle):
    cases = 0
    lv = lanes()
    lv["repeats"] = np.tile(lcg_seq(9, 37), 600)[:20000]
    for name, v in lv.items():
        for mode, plog2, tag in ((M_PRED, 16, TAG_RC), (M_PRED, 10, TAG_RC), (M_PRED_RC, 16, TAG_RC),
                                 (M_PRED_RC, 12, TAG_RANS), (M_PRED2, 16, TAG_RANS), (M_PRED2, 10, TAG_RC)):
            frames = [(mode, hi - lo, oracle.pred_payload(mode, v[lo:hi], plog2, tag))
                      for lo, hi in ((0, 1), (1, 4097), (4097, 20000))]
            s = stream(frames, U64)
            s = s[:6] + bytes([plog2]) + s[7:]
            assert _agree(qb, oracle, s) == "ok", (name, mode, plog2, tag)
            assert np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64).tobytes() == v.tobytes()
            cases += 1
    assert cases == 6 * len(lv)
    # damage: trailing byte, cut residuals, bad tags
    v = lv["sine"][:3000]
    kinds = []
    for mode in (M_PRED, M_PRED_RC, M_PRED2):
        good = oracle.pred_payload(mode, v, 16, TAG_RC)
        for bad in (good + b"\x00", good[:-5], b"\x05" + good[1:], b""):
            kinds.append(_agree(qb, oracle, stream([(mode, len(v), bad)], U64)))
    assert "CorruptPayload" in kinds and "Truncated" in kinds


M_LZ, TAG_LZ = 4, 3


def _varint_bytes(v):
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        if v:
            out.append(b | 0x80)
        else:
            out.append(b)
            return bytes(out)


def _coded(oracle, data, tag):
    return bytes([tag]) + (oracle.rc_compress(data) if tag == TAG_RC else oracle.rans_compress(data))


def _cascade(oracle, res, tag):
    """entropy/mod.rs:124-146: the Max LZ cascade around residual bytes."""
    return bytes([TAG_LZ]) + _varint_bytes(len(res)) + _coded(oracle, oracle.lz_compress(res), tag)


def test_oracle_lz_round_trips(oracle):
    # lz.rs tests roundtrip_repetitive / roundtrip_random_and_edges
    rep = np.array([float(i & 15) for i in range(50000)]).view(np.uint64)
    enc = oracle.lz_compress(rep.tobytes())
    assert len(enc) < rep.nbytes // 4 and oracle.lz_decompress(enc, rep.nbytes) == rep.tobytes()
    rnd = lcg_seq(1, 5000).tobytes()
    assert oracle.lz_decompress(oracle.lz_compress(rnd), len(rnd)) == rnd
    assert oracle.lz_decompress(oracle.lz_compress(b""), 0) == b""
    one = np.array([42], np.uint64).tobytes()
    assert oracle.lz_decompress(oracle.lz_compress(one), 8) == one


@pytest.mark.gpu
def test_lz_mode_and_cascade_decode_like_the_oracle(qb, oracle):
    lv = lanes()
    lv["dict16"] = np.array([float(i & 15) for i in range(20000)]).view(np.uint64)
    lv["repeats"] = np.tile(lcg_seq(9, 37), 600)[:20000]
    for name, v in lv.items():
        for tag in (TAG_RC, TAG_RANS):
            frames = [(M_LZ, hi - lo, _coded(oracle, oracle.lz_compress(v[lo:hi].tobytes()), tag))
                      for lo, hi in ((0, 1), (1, 4097), (4097, 20000))]
            s = stream(frames, U64)
            assert _agree(qb, oracle, s) == "ok", (name, tag)
            assert np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64).tobytes() == v.tobytes()
    # the cascade around DELTA2, PRED2 and BYTE_TRANSPOSE residuals
    v = lv["repeats"][:8000]
    for mode, tag in ((M_D2, TAG_RC), (M_PRED2, TAG_RANS), (M_BT, TAG_RC)):
        if mode == M_D2:
            res = oracle.rc_decompress(oracle.linear_payload(M_D2, v, 2, TAG_RC)[1:], 10 * len(v) + 16)
        elif mode == M_PRED2:
            res = oracle.rc_decompress(oracle.pred_payload(M_PRED2, v, 16, TAG_RC)[1:], 10 * len(v) + 16)
        else:
            res = np.ascontiguousarray(v).view(np.uint8).reshape(-1, 8).T.copy().tobytes()
        s = stream([(mode, len(v), _cascade(oracle, res, tag))], U64)
        assert _agree(qb, oracle, s) == "ok", mode
        assert np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64).tobytes() == v.tobytes()
    # damage inside the LZ stream: bad offset, overrun, wrong length, cuts; cascade length above the bound
    good = oracle.lz_compress(lv["dict16"][:4096].tobytes())
    kinds = []
    variants = [good[:len(good) // 2], good[:-1], _varint_bytes(4096 * 8 + 8) + good[len(_varint_bytes(4096 * 8)):]]
    b = bytearray(good)
    b[len(_varint_bytes(4096 * 8)) + 9:len(_varint_bytes(4096 * 8)) + 10] = b"\x7f"  # an offset byte of the first match
    variants.append(bytes(b))
    for bad in variants:
        kinds.append(_agree(qb, oracle, stream([(M_LZ, 4096, _coded(oracle, bad, TAG_RANS))], U64)))
    huge = bytes([TAG_LZ]) + _varint_bytes(10 ** 9) + _coded(oracle, good, TAG_RC)
    kinds.append(_agree(qb, oracle, stream([(M_D2, 4096, huge)], U64)))
    assert kinds[-1] == "CorruptPayload" and "Truncated" in kinds and "CorruptPayload" in kinds[:-1]
