"""ALP-RD exception lists (reference alp_rd.rs:281-283): vals[p] = (left << rbw) |
rights[p] for each (varint p, u64 left) record, in list order.  The frame
decoder applies a list in chunks of 4096 records, in parallel when a chunk's
positions strictly increase and in order otherwise.  These frames are built
with the oracle's ALP-RD encoder directly (a single-frame stream around its
payload), so the lists are long: 4,304 and 17,139 records, i.e. one and five
chunks; a copy with a repeated position checks that the later record wins.
"""
import numpy as np
import pytest

from conftest import lcg_seq
from test_entropy_decode import _varint

pytestmark = pytest.mark.gpu

M_ALP_RD, F64 = 52, 0


def one_frame_stream(payload, n, mode=M_ALP_RD):
    head = b"FCR1" + bytes([2, 0, 16, F64]) + n.to_bytes(8, "little")
    return head + bytes([mode]) + n.to_bytes(4, "little") + len(payload).to_bytes(4, "little") + payload


def alprd_payload(oracle, n, seed):
    rng = np.random.default_rng(seed)
    bits = (np.uint64(0x3FF00) << np.uint64(46)) | rng.integers(0, 1 << 46, n, dtype=np.int64).astype(np.uint64)
    m = rng.random(n) < 0.13
    bits[m] = lcg_seq(seed, int(m.sum()))
    p = oracle.encode_mode(M_ALP_RD, bits, oracle.DT_F64, level=1)
    assert p is not None
    return bits, bytes(p)


def exception_records(p):
    """Byte offsets of the (varint position) fields of the payload's exception list."""
    nexc, pos = _varint(p, 2 + 8 * p[1])
    offs = []
    for _ in range(nexc):
        offs.append(pos)
        _, pos = _varint(p, pos)
        pos += 8
    return offs


@pytest.mark.parametrize("n,seed,min_exc", [(32768, 11, 4097), (131072, 12, 16385)])
def test_long_exception_lists(qb, oracle, n, seed, min_exc):
    bits, p = alprd_payload(oracle, n, seed)
    assert len(exception_records(p)) >= min_exc
    s = one_frame_stream(p, n)
    d = qb.decompress_column(s)
    assert np.ascontiguousarray(d.values).view(np.uint64).tobytes() == bits.tobytes()


def test_repeated_exception_position_later_record_wins(qb, oracle):
    n = 32768
    bits, p = alprd_payload(oracle, n, 13)
    offs = exception_records(p)
    b = bytearray(p)
    done = 0
    for k in range(1, len(offs) - 1, 997):  # give record k the position of record k - 1
        a0, a1 = offs[k - 1], offs[k]
        la, lb = _varint(p, a0)[1] - a0, _varint(p, a1)[1] - a1
        if la == lb:
            b[a1:a1 + lb] = p[a0:a0 + la]
            done += 1
    assert done >= 2
    s = one_frame_stream(bytes(b), n)
    want = oracle.decompress_column(s)[1]
    got = qb.decompress_column(s).values
    assert np.ascontiguousarray(got).view(np.uint8).tobytes() == np.ascontiguousarray(want).view(np.uint8).tobytes()


def _rebuilt(p, offs, k, new_varint):
    """The payload with record k's position varint replaced (the records after it shift)."""
    end = _varint(p, offs[k])[1]
    return p[:offs[k]] + bytes(new_varint) + p[end:]


def test_damaged_exception_lists_match_oracle(qb, oracle):
    from test_entropy_decode import _agree
    n = 32768
    bits, p = alprd_payload(oracle, n, 14)
    offs = exception_records(p)
    k = len(offs) // 2
    pos_k = _varint(p, offs[k])[0]
    cases = {
        "position_n": _rebuilt(p, offs, k, [n & 0x7F | 0x80, (n >> 7) & 0x7F | 0x80, n >> 14]),
        "position_last": _rebuilt(p, offs, k, [(n - 1) & 0x7F | 0x80, ((n - 1) >> 7) & 0x7F | 0x80, (n - 1) >> 14]),
        "varint_4_bytes": _rebuilt(p, offs, k, [pos_k & 0x7F | 0x80, (pos_k >> 7) & 0x7F | 0x80,
                                                (pos_k >> 14) | 0x80, 0]),
        "varint_6_bytes": _rebuilt(p, offs, k, [pos_k & 0x7F | 0x80, (pos_k >> 7) & 0x7F | 0x80,
                                                (pos_k >> 14) | 0x80, 0x80, 0x80, 0]),
        "varint_11_bytes": _rebuilt(p, offs, k, [0x80] * 10 + [0]),
        "cut_in_record": p[:offs[k] + 4],
        "cut_at_record": p[:offs[k]],
        "cut_last_record": p[:offs[-1] + 2],
    }
    kinds = {}
    for name, q in cases.items():
        kinds[name] = _agree(qb, oracle, one_frame_stream(q, n))
    assert kinds["position_n"] == "CorruptPayload"
    assert kinds["varint_4_bytes"] == "ok" and kinds["varint_6_bytes"] == "ok"
    assert kinds["varint_11_bytes"] == "CorruptPayload"
    assert kinds["cut_in_record"] == kinds["cut_at_record"] == "Truncated"
