"""The benchmark columns at their full size (67,108,864 values each, seeded
synthetic stand-ins for the integer-lane and float-lane workloads) at
Level::Fast: the GPU stream must equal the oracle's byte for byte, and its
decode must give back every value bit for bit (null slots as 0, the bitmap
unchanged).
"""
import numpy as np
import pytest

from quoin_b200 import synth

pytestmark = pytest.mark.gpu

N_FULL = 1 << 26
DEC128 = 6


def _expected(v, bm, n):
    raw = np.ascontiguousarray(v).view(np.uint8).reshape(n, -1).copy()
    if bm is not None:
        raw[~np.unpackbits(bm, bitorder="little")[:n].astype(bool)] = 0
    return raw.tobytes()


@pytest.mark.parametrize("kind", ["integer", "float"])
def test_full_size_columns_match_oracle_and_round_trip(qb, oracle, kind):
    for name, dt, v, bm in synth.benchmark_columns(kind, N_FULL):
        sc, pr = (4, 18) if dt == DEC128 else (0, 0)
        got = qb.compress_column(v, bm, qb.Config(level=qb.Level.FAST), dtype=dt, scale=sc, precision=pr)
        want = oracle.compress_column(v, dt, bm, level=1, scale=sc, precision=pr, threads=16)
        assert len(got) == len(want), name
        assert got == want, name
        del want
        d = qb.decompress_column(got)
        assert np.ascontiguousarray(d.values).view(np.uint8).tobytes() == _expected(v, bm, N_FULL), name
        if bm is not None:
            assert bytes(d.validity) == bm.tobytes(), name
        else:
            assert d.validity is None, name
