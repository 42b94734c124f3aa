"""Selection::Sample (reference src/encoder.rs:470-620) at Level::Fastest and
Level::Fast: each block's candidates are sized on a stratified sample (8 runs
of 64 values spread over the block, or the whole block up to 512 values) and
only the winner is encoded in full against RAW, CONST and STRIDE.  The GPU
stream must equal the oracle's (oracle/quoin_oracle.c encode_block_sampled)
byte for byte and decode to the input.

The CPU test pins the oracle: its sampled streams decode, and on these cases
the sampled winner differs from the full competition's somewhere, so the
GPU tests compare a selection that is really different.
"""
import numpy as np
import pytest

from conftest import bitmap_from_bools, lcg1_seq, lcg_seq
from test_entropy_decode import _dec_bytes, _expected, frame_tags
from test_gpu_parity import shape_cases

F64, I64, U64, I32, U32, F32 = 0, 1, 2, 3, 4, 5


def sample_cases():
    rng = np.random.default_rng(77)
    u12 = rng.random(100000) + 1.0
    u12[rng.integers(0, 100000, 900)] = rng.random(900) * 1e6
    vb = rng.random(100000) > 0.15
    return [
        ("runs_of_categories", np.repeat(lcg_seq(5, 900) >> np.uint64(50), 200).astype(np.int64)[:150000], I64, None),
        ("sine", np.sin(np.arange(70000) * 1e-3), F64, None),
        ("prices", np.floor(rng.random(100000) * 1e6 + 0.5) / 100.0, F64, None),
        ("alprd_nullable", u12, F64, bitmap_from_bools(vb)),
        ("dict_u64", (lcg_seq(31, 3000) >> np.uint64(8))[(lcg1_seq(32, 90000) >> np.uint64(40)) % 1800], U64, None),
        ("ramp_i32", (np.arange(80000) * 7 - 3).astype(np.int32), I32, None),
        ("random_u64", lcg_seq(3, 50000), U64, None),
        ("walk_f32", np.cumsum(rng.standard_normal(60000)).astype(np.float32), F32, None),
        ("timestamps_nullable", (1_700_000_000_000 + np.cumsum(1000 + rng.poisson(50, 100000))).astype(np.int64), I64,
         bitmap_from_bools(vb)),
    ]


def test_oracle_sampled_streams_decode(oracle):
    differs = 0
    for name, v, dt, bm in sample_cases():
        for level in (0, 1):
            s = oracle.compress_column(v, dt, bm, level=level, sample=True)
            d = oracle.decompress_column(s)
            assert np.ascontiguousarray(d[1]).view(np.uint8).tobytes() == _expected(v, dt, bm), (name, level)
            differs += s != oracle.compress_column(v, dt, bm, level=level)
    assert differs >= 4


def gpu_sampled(qb, v, dt, bm, level, block_size=None):
    cfg = qb.Config(level=qb.Level(level), block_size=block_size, selection=qb.Selection.SAMPLE)
    return qb.compress_column(v, bm, cfg, dtype=dt)


def check(qb, oracle, v, dt, bm, level, block_size=None):
    want = oracle.compress_column(v, dt, bm, level=level, block_size=block_size, sample=True)
    got = gpu_sampled(qb, v, dt, bm, level, block_size)
    if got != want:
        raise AssertionError(f"{len(got)} vs {len(want)} bytes; tags {frame_tags(got)[:6]} vs {frame_tags(want)[:6]}")
    assert _dec_bytes(qb.decompress_column(got)) == _expected(v, dt, bm)


@pytest.mark.gpu
@pytest.mark.parametrize("level", [0, 1])
@pytest.mark.parametrize("case", sample_cases(), ids=lambda c: c[0])
def test_sampled_streams_match_oracle(qb, oracle, case, level):
    name, v, dt, bm = case
    check(qb, oracle, v, dt, bm, level)


@pytest.mark.gpu
@pytest.mark.parametrize("case", shape_cases(), ids=lambda c: c[0])
def test_sampled_shapes_match_oracle(qb, oracle, case):
    name, v, dt, bm = case
    for level in (0, 1):
        check(qb, oracle, v, dt, bm, level)


@pytest.mark.gpu
@pytest.mark.parametrize("bs", [7, 300, 512, 513, 1000, 70000])
def test_sampled_fixed_block_sizes(qb, oracle, bs):
    rng = np.random.default_rng(bs)
    for name, v, dt, bm in sample_cases()[:4]:
        check(qb, oracle, v, dt, bm, 1, block_size=bs)
    check(qb, oracle, np.round(np.cumsum(rng.standard_normal(9000)), 2), F64, None, 0, block_size=bs)


@pytest.mark.gpu
def test_sample_selection_outside_fastest_and_fast_is_refused(qb):
    v = np.arange(1000, dtype=np.int64)
    with pytest.raises(qb.Error) as ei:
        gpu_sampled(qb, v, I64, None, int(qb.Level.BALANCED_INPOOL))
    assert ei.value.kind == "Unsupported"
