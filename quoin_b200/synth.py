"""Seeded synthetic columns with the shapes of the benchmark workloads.

The published benchmarks run on datasets that are not available here (the
ALP float corpus, ClickBench); these generators stand in for them with the
value distributions each workload names.  numpy PCG64, base seed
20261203 + 100 * column set + column index (column sets: 0 prices, 1 integer
lanes, 2 float lanes, 3 mixed columns, 4 served requests).
"""
from __future__ import annotations

import numpy as np

# Wire dtype ids of the stream header (reference src/dtype.rs:68-93), the same
# values as the package's constants.  Defined here so the generators load
# without the CUDA library (the CPU reference arm of the benchmark imports
# this file by path).
F64, I64, U64, I32, U32, F32, DECIMAL128, DECIMAL256 = range(8)

BASE_SEED = 20261203


def rng_for(column_set: int, column: int) -> np.random.Generator:
    return np.random.default_rng(BASE_SEED + 100 * column_set + column)


def bernoulli_bitmap(rng: np.random.Generator, n: int, p_valid: float = 0.9) -> np.ndarray:
    valid = rng.random(n) < p_valid
    return np.packbits(valid, bitorder="little")


def timestamps_i64(n: int, rng: np.random.Generator) -> np.ndarray:
    """i64 ns timestamps from 1.7e18 with steps 1,000,000 + Poisson(5000)."""
    d = 1_000_000 + rng.poisson(5000, n).astype(np.int64)
    d[0] = 0
    return 1_700_000_000_000_000_000 + np.cumsum(d)


def runs_u64(n: int, rng: np.random.Generator) -> np.ndarray:
    """u64 base + U[0, 2^k) with base ~ U[0, 2^40) and k ~ U{3..40} redrawn per 1024 values."""
    base = np.uint64(rng.integers(0, 1 << 40))
    nruns = (n + 1023) // 1024
    k = rng.integers(3, 41, nruns).astype(np.uint64)
    masks = (np.uint64(1) << k) - np.uint64(1)
    u = rng.integers(0, np.iinfo(np.int64).max, n, dtype=np.int64).astype(np.uint64)
    return base + (u & np.repeat(masks, 1024)[:n])


def categories_i32(n: int, rng: np.random.Generator, ncat: int = 64, s: float = 1.1, mean_run: int = 16):
    """i32 categories: Zipf(s) over `ncat` symbols, emitted in Geometric(1/mean_run) runs."""
    cats = np.unique(rng.integers(-(1 << 31), 1 << 31, 4 * ncat, dtype=np.int64))
    cats = rng.permutation(cats)[:ncat].astype(np.int32)
    p = np.arange(1, ncat + 1, dtype=np.float64) ** -s
    p /= p.sum()
    m = n // mean_run + 64
    out = np.empty(0, np.int32)
    parts = []
    total = 0
    while total < n:
        lens = rng.geometric(1.0 / mean_run, m)
        syms = rng.choice(ncat, m, p=p)
        parts.append(np.repeat(cats[syms], lens))
        total += int(lens.sum())
    out = np.concatenate(parts)[:n]
    return np.ascontiguousarray(out)


def prices_f64(n: int, rng: np.random.Generator, exc_frac: float = 0.03) -> np.ndarray:
    """Two-decimal prices round(U(0,10000)*100)/100 (half away from zero) with
    floor(exc_frac*n) positions replaced by random finite f64 bit patterns."""
    x = rng.random(n) * 10000.0 * 100.0
    v = np.floor(x + 0.5) / 100.0
    bits = v.view(np.uint64).copy()
    ne = int(exc_frac * n)
    pos = rng.permutation(n)[:ne]
    r = rng.integers(0, np.iinfo(np.int64).max, ne, dtype=np.int64).astype(np.uint64) * np.uint64(2)
    r |= rng.integers(0, 2, ne).astype(np.uint64)
    bad = ((r >> np.uint64(52)) & np.uint64(0x7FF)) == np.uint64(0x7FF)
    while bad.any():
        r2 = rng.integers(0, np.iinfo(np.int64).max, int(bad.sum()), dtype=np.int64).astype(np.uint64) * np.uint64(2)
        r[bad] = r2
        bad = ((r >> np.uint64(52)) & np.uint64(0x7FF)) == np.uint64(0x7FF)
    bits[pos] = r
    return bits.view(np.float64)


def random_walk_f64(n: int, rng: np.random.Generator) -> np.ndarray:
    return 20.0 + np.cumsum(np.concatenate([[0.0], rng.normal(0.0, 1e-3, n - 1)])) if n else np.zeros(0)


def sensor_f32(n: int, rng: np.random.Generator) -> np.ndarray:
    return (np.round(rng.normal(25.0, 5.0, n) * 10.0) / 10.0).astype(np.float32)


def decimal128_uniform(n: int, rng: np.random.Generator, lo: int = -10**14, hi: int = 10**14) -> np.ndarray:
    """Decimal128 significands uniform in [lo, hi), as (n, 2) little-endian int64 limbs."""
    v = rng.integers(lo, hi, n, dtype=np.int64)
    out = np.empty((n, 2), np.int64)
    out[:, 0] = v
    out[:, 1] = np.where(v < 0, -1, 0)
    return out


def benchmark_columns(kind: str, n: int):
    """[(name, wire dtype, values, validity bitmap or None)] of a benchmark column
    set: "prices" (one f64 column of two-decimal prices with 3 % random-bit
    values), "integer" (i64 timestamps, u64 runs, i32 categories, 10 % nulls) or
    "float" (f64 random walk, f32 sensor readings, Decimal128)."""
    if kind == "integer":
        r = [rng_for(1, c) for c in range(3)]
        return [
            ("timestamps_i64", I64, timestamps_i64(n, r[0]), bernoulli_bitmap(r[0], n)),
            ("runs_u64", U64, runs_u64(n, r[1]), bernoulli_bitmap(r[1], n)),
            ("categories_i32", I32, categories_i32(n, r[2]), bernoulli_bitmap(r[2], n)),
        ]
    if kind == "prices":
        return [("prices_f64", F64, prices_f64(n, rng_for(0, 0)), None)]
    if kind == "float":
        r = [rng_for(2, c) for c in range(3)]
        return [
            ("random_walk_f64", F64, random_walk_f64(n, r[0]), None),
            ("sensor_f32", F32, sensor_f32(n, r[1]), None),
            ("decimal128", DECIMAL128, decimal128_uniform(n, r[2]), None),
        ]
    raise ValueError(kind)


MIXED_DTYPES = [F64, F32, I64, U64, I32, U32, DECIMAL128]
NATIVE_BYTES = {F64: 8, F32: 4, I64: 8, U64: 8, I32: 4, U32: 4, DECIMAL128: 16}


def mixed_columns(ncols: int, max_len: int = 1 << 21, min_len: int = 1024):
    """Many uneven columns: `ncols` columns with lengths floor(exp(U[ln min_len,
    ln max_len])), dtype uniform over f64/f32/i64/u64/i32/u32/decimal128, the
    per-dtype generators of benchmark_columns, and a null rate U(0, 0.2) each.
    [(name, wire dtype, values, validity bitmap or None)]."""
    return _mixed_columns(3, ncols, lambda r, dt: int(np.floor(np.exp(r.uniform(np.log(min_len), np.log(max_len))))))


def request_columns(ncols: int, max_bytes: int = 256 << 20, min_bytes: int = 64 << 10):
    """Columns of the served request stream: sizes floor(exp(U[ln min_bytes,
    ln max_bytes])) bytes of native values, dtypes and generators as mixed_columns."""
    return _mixed_columns(4, ncols, lambda r, dt: max(
        int(np.floor(np.exp(r.uniform(np.log(min_bytes), np.log(max_bytes))))) // NATIVE_BYTES[dt], 1),
        size_first=False)


def _mixed_columns(column_set: int, ncols: int, length, size_first: bool = True):
    dtypes = MIXED_DTYPES
    out = []
    for c in range(ncols):
        r = rng_for(column_set, c)
        if size_first:
            n = length(r, None)
            dt = dtypes[int(r.integers(0, len(dtypes)))]
        else:
            dt = dtypes[int(r.integers(0, len(dtypes)))]
            n = length(r, dt)
        null_rate = float(r.uniform(0.0, 0.2))
        if dt == F64:
            v = prices_f64(n, r) if c % 2 == 0 else random_walk_f64(n, r)
        elif dt == F32:
            v = sensor_f32(n, r)
        elif dt == I64:
            v = timestamps_i64(n, r)
        elif dt == U64:
            v = runs_u64(n, r)
        elif dt == I32:
            v = categories_i32(n, r)
        elif dt == U32:
            v = categories_i32(n, r).view(np.uint32)
        else:
            v = decimal128_uniform(n, r)
        bm = bernoulli_bitmap(r, n, 1.0 - null_rate) if null_rate > 0 else None
        out.append((f"col{c}", dt, v, bm))
    return out
