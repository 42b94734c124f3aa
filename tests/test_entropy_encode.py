"""GPU encoder at Level.BALANCED_INPOOL: Balanced's competition (lambda 2) with
the rANS-coded forms of FLOAT_MULT, ALP-RD and DICT and the BYTE_TRANSPOSE
candidate (reference encoder.rs:275-469, entropy/rans.rs:25-108), without the
Lz and Pco candidates.  Its streams must equal the oracle's Balanced in-pool
streams byte for byte and decode to the input.
"""
import numpy as np
import pytest

from conftest import lcg1_seq, lcg_seq
from test_entropy_decode import _dec_bytes, _expected, entropy_cases, frame_tags
from test_gpu_parity import shape_cases

pytestmark = pytest.mark.gpu

LEVEL_ORACLE = 2


def gpu_balanced(qb, v, dt, bm=None, block_size=None, scale=0, precision=0):
    cfg = qb.Config(level=qb.Level.BALANCED_INPOOL, block_size=block_size)
    return qb.compress_column(v, bm, cfg, dtype=dt, scale=scale, precision=precision)


def check(qb, oracle, v, dt, bm=None, block_size=None, scale=0, precision=0):
    want = oracle.compress_column(v, dt, bm, level=LEVEL_ORACLE, block_size=block_size, scale=scale,
                                  precision=precision)
    got = gpu_balanced(qb, v, dt, bm, block_size, scale, precision)
    if got != want:
        gf, wf = frame_tags(got), frame_tags(want)
        raise AssertionError(f"stream mismatch: {len(got)} vs {len(want)} bytes; tags {gf[:8]} vs {wf[:8]}")
    assert _dec_bytes(qb.decompress_column(got)) == _expected(v, dt, bm)
    return got


@pytest.mark.parametrize("case", entropy_cases(), ids=lambda c: c[0])
def test_entropy_shapes_match_oracle(qb, oracle, case):
    name, v, dt, bm, sc, pr = case
    check(qb, oracle, v, dt, bm, scale=sc, precision=pr)


@pytest.mark.parametrize("case", shape_cases(), ids=lambda c: c[0])
def test_shapes_match_oracle_balanced(qb, oracle, case):
    name, v, dt, bm = case
    check(qb, oracle, v, dt, bm)


@pytest.mark.parametrize("bs", [1, 7, 1000, 5000, 1 << 30])
def test_fixed_block_sizes_balanced(qb, oracle, bs):
    rng = np.random.default_rng(bs)
    cats = (lcg_seq(5, 300) >> np.uint64(8))[lcg1_seq(9, 20000) >> np.uint64(56)]
    check(qb, oracle, cats, 2, block_size=bs)
    walk = np.round(np.cumsum(rng.standard_normal(9000)), 3)
    check(qb, oracle, walk, 0, block_size=bs)


def test_every_entropy_part_is_emitted(qb, oracle):
    """The cases above make the GPU write every coded form (tags seen in its own streams)."""
    seen = set()
    for name, v, dt, bm, sc, pr in entropy_cases():
        seen.update(frame_tags(gpu_balanced(qb, v, dt, bm, scale=sc, precision=pr)))
    need = {("BT",), ("FM", 1), ("RD", 1, 0, True), ("RD", 1, 1, True), ("RD", 0, 1, False),
            ("DICT", 0, 1, 1), ("DICT", 1, 1, 2), ("DICT", 2, 1, 1), ("DICT", 2, 1, 2), ("DICT", 2, 0, 0)}
    assert need <= seen, sorted(need - seen)


def test_levels_other_than_inpool_balanced_are_refused(qb):
    v = np.arange(1000, dtype=np.int64)
    for lv in (qb.Level.BALANCED, qb.Level.HIGH, qb.Level.MAX):
        with pytest.raises(qb.Error) as ei:
            qb.compress_column(v, None, qb.Config(level=lv), dtype=1)
        assert ei.value.kind == "Unsupported"
