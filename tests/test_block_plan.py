"""The adaptive block plan (reference encoder.rs:154-178) over long window chains.

A column of 32,768-value windows, each a constant run (the probe sees repeats:
the block grows to 131,072 values) or a ramp (distinct values, no repeats: a
32,768-value block), in a seeded random order.  The frame sizes of the GPU
stream must follow the reference's chain: a block starts at window w, covers
four windows when w's probe grows it, else one.  More than 4,096 windows
exercise the plan's chunked scan across chunk boundaries.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W = 32768


def expected_sizes(grow, n):
    sizes, s = [], 0
    while s < n:
        end = min(s + (4 * W if grow[s // W] else W), n)
        sizes.append(end - s)
        s = end
    return sizes


def frame_sizes(stream):
    pos, out = 16, []
    while pos < len(stream):
        out.append(int.from_bytes(stream[pos + 1:pos + 5], "little"))
        pos += 9 + int.from_bytes(stream[pos + 5:pos + 9], "little")
    return out


@pytest.mark.parametrize("nwin,tail", [(37, 0), (4096, 0), (4101, 1234), (9000, 7)])
def test_block_plan_chain(qb, nwin, tail):
    rng = np.random.default_rng(nwin)
    grow = rng.random(nwin + 1) < 0.3
    n = nwin * W + tail
    v = np.empty(n, np.uint64)
    ramp = np.arange(W, dtype=np.uint64)
    for w in range(nwin + (1 if tail else 0)):
        a, b = w * W, min((w + 1) * W, n)
        v[a:b] = np.uint64(w) if grow[w] else (np.uint64(w) << np.uint64(32)) + ramp[:b - a]
    s = qb.compress_column(v, None, qb.Config(level=qb.Level.FAST), dtype=2)
    assert frame_sizes(s) == expected_sizes(grow, n)
