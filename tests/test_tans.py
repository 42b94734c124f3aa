"""The legacy tANS entropy tag (1) of src/entropy/tans.rs: the reference's
decoder still accepts it wherever residual bytes are entropy coded
(entropy/mod.rs:152-163) although its encoder no longer writes it.  The
oracle restates the coder (its CPU checks port tans.rs roundtrip_skewed and
roundtrip_uniform_and_single); the GPU decode of tANS-coded High / Max
payloads, byte-transposed planes and LZ streams must give the oracle's
values, and the oracle's error kinds on damaged headers.
"""
import numpy as np
import pytest

from test_linear_modes import F64, M_BT, M_D2, M_DP, M_OD, U64, _agree, lanes, stream

TAG_TANS = 1
M_PRED2, M_PRED_RC, M_LZ, TAG_LZ = 25, 29, 4, 3


def _lcg(s):
    s[0] = (s[0] * 6364136223846793005 + 1442695040888963407) & (2**64 - 1)
    return s[0]


def _varint(v):
    out = bytearray()
    while True:
        b, v = v & 0x7F, v >> 7
        out.append(b | (0x80 if v else 0))
        if not v:
            return bytes(out)


def _header(t):
    """(end of varint(len), number of symbols, offset of the state) of tANS bytes."""
    pos = 0
    while t[pos] & 0x80:
        pos += 1
    pos += 1
    num = t[pos] + 1
    return pos, num, pos + 1 + 3 * num


def test_oracle_tans_round_trips(oracle):
    s = [1]
    skewed = bytes(((_lcg(s) >> 50) & 0xFF) if _lcg(s) % 8 == 0 else 0 for _ in range(40000))
    p = oracle.tans_compress(skewed)
    assert p is not None and len(p) < len(skewed)
    assert oracle.tans_decompress(p, len(skewed)) == skewed
    s = [99]
    uniform = bytes((_lcg(s) >> 40) & 0xFF for _ in range(40000))
    for data in (uniform, bytes([7]) * 5000, bytes([42])):
        p = oracle.tans_compress(data)
        if p is not None:
            assert oracle.tans_decompress(p, len(data)) == data
    assert oracle.tans_compress(b"") is None


def test_oracle_tans_header_checks(oracle):
    data = bytes(range(50)) * 40
    t = oracle.tans_compress(data)
    vend, num, st = _header(t)
    kinds = {}

    def kind(b, max_len=len(data)):
        try:
            oracle.tans_decompress(bytes(b), max_len)
            return "ok"
        except oracle.OracleError as e:
            return e.kind

    kinds["good"] = kind(t)
    kinds["over_max_len"] = kind(t, len(data) - 1)
    kinds["no_count"] = kind(t[:vend])
    kinds["short_symbols"] = kind(t[:vend + 1 + num // 2])
    kinds["short_weights"] = kind(t[:st - 1])
    kinds["short_state"] = kind(t[:st + 3])
    for name, val in (("state_low", 0x3FF), ("state_high", 0x800)):
        b = bytearray(t)
        b[st:st + 4] = val.to_bytes(4, "little")
        kinds[name] = kind(b)
    b = bytearray(t)
    b[vend + 1 + num:vend + 3 + num] = b"\x00\x00"
    kinds["zero_weight"] = kind(b)
    b = bytearray(t)
    b[vend + 2] = b[vend + 1]
    kinds["duplicate_symbol"] = kind(b)
    b = bytearray(t)
    b[vend + 1 + num] += 1
    kinds["weight_sum"] = kind(b)
    assert kinds == {"good": "ok", "over_max_len": "CorruptPayload", "no_count": "Truncated",
                     "short_symbols": "Truncated", "short_weights": "Truncated", "short_state": "Truncated",
                     "state_low": "CorruptPayload", "state_high": "CorruptPayload", "zero_weight": "CorruptPayload",
                     "duplicate_symbol": "CorruptPayload", "weight_sum": "CorruptPayload"}


@pytest.mark.gpu
def test_tans_coded_payloads_decode_like_the_oracle(qb, oracle):
    cases = 0
    for name, v in lanes().items():
        for mode, order in ((M_OD, 0), (M_D2, 0), (M_D2, 3), (M_DP, 2)):
            frames = []
            for lo, hi in ((0, 1), (1, 4097), (4097, 20000)):
                p = oracle.linear_payload(mode, v[lo:hi], order, TAG_TANS)
                if p is None:
                    break
                assert p[0] == TAG_TANS
                frames.append((mode, hi - lo, p))
            if len(frames) < 3:
                continue
            s = stream(frames, U64 if mode == M_OD else F64)
            assert _agree(qb, oracle, s) == "ok", (name, mode)
            got = np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64)
            assert got.tobytes() == v.tobytes(), (name, mode)
            cases += 1
        for mode, plog2 in ((M_PRED_RC, 16), (M_PRED2, 12)):
            p = oracle.pred_payload(mode, v[:8000], plog2, TAG_TANS)
            s = bytearray(stream([(mode, 8000, p)], U64))
            s[6] = plog2
            assert _agree(qb, oracle, bytes(s)) == "ok", (name, mode)
            cases += 1
    assert cases >= 30
    # byte-transposed planes and an LZ frame coded by tANS; the LZ cascade with a tANS inner stream
    v = lanes()["walk"][:5000]
    soa = np.ascontiguousarray(v).view(np.uint8).reshape(-1, 8).T.copy().tobytes()
    s = stream([(M_BT, len(v), bytes([TAG_TANS]) + oracle.tans_compress(soa))])
    assert _agree(qb, oracle, s) == "ok"
    assert np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64).tobytes() == v.tobytes()
    rep = np.tile(lanes()["random"][:512], 8)
    lz = oracle.lz_compress(rep.tobytes())
    s = stream([(M_LZ, len(rep), bytes([TAG_TANS]) + oracle.tans_compress(lz))], U64)
    assert _agree(qb, oracle, s) == "ok"
    res = oracle.rc_decompress(oracle.linear_payload(M_D2, v, 2, 0)[1:], 10 * len(v) + 16)
    casc = bytes([TAG_LZ]) + _varint(len(res)) + bytes([TAG_TANS]) + oracle.tans_compress(oracle.lz_compress(res))
    s = stream([(M_D2, len(v), casc)])
    assert _agree(qb, oracle, s) == "ok"
    assert np.ascontiguousarray(qb.decompress_column(s).values).view(np.uint64).tobytes() == v.tobytes()


@pytest.mark.gpu
def test_damaged_tans_payloads_match_oracle(qb, oracle):
    v = lanes()["sine"][:3000]
    good = oracle.linear_payload(M_D2, v, 2, TAG_TANS)
    t = good[1:]
    vend, num, st = _header(t)
    variants = {
        "huge_len": _varint(10**9) + t[vend:],
        "no_count": t[:vend],
        "short_symbols": t[:vend + 2],
        "short_state": t[:st + 2],
        "cut_bits": t[:(st + 4 + len(t)) // 2],
    }
    for name, val in (("state_low", 0x3FF), ("state_high", 0x800)):
        b = bytearray(t)
        b[st:st + 4] = val.to_bytes(4, "little")
        variants[name] = bytes(b)
    b = bytearray(t)
    b[vend + 1 + num:vend + 3 + num] = b"\x00\x00"
    variants["zero_weight"] = bytes(b)
    b = bytearray(t)
    b[vend + 2] = b[vend + 1]
    variants["duplicate_symbol"] = bytes(b)
    b = bytearray(t)
    b[vend + 1 + num] ^= 1
    variants["weight_sum"] = bytes(b)
    kinds = {k: _agree(qb, oracle, stream([(M_D2, len(v), bytes([TAG_TANS]) + p)])) for k, p in variants.items()}
    for k in ("huge_len", "state_low", "state_high", "zero_weight", "duplicate_symbol", "weight_sum"):
        assert kinds[k] == "CorruptPayload", (k, kinds)
    for k in ("no_count", "short_symbols", "short_state"):
        assert kinds[k] == "Truncated", (k, kinds)
