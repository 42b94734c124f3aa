"""Regenerate the golden stream fixtures in this directory.

Each fixture is a small seeded input column and the exact stream the oracle
(the C restatement of the reference encoder, oracle/quoin_oracle.c) produces
for it at Level::Fastest and Level::Fast.  The GPU tests compare the CUDA
encoder's bytes against these files and decode them with the CUDA decoder,
so parity is checked against committed bytes, not only against a live oracle.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

M64 = (1 << 64) - 1


def lcg(seed, n):
    out = np.empty(n, dtype=np.uint64)
    s = seed
    for i in range(n):
        s = (s * 6364136223846793005 + 1442695040888963407) & M64
        out[i] = s
    return out


def cases():
    rng = np.random.default_rng(20261203)
    c = []
    c.append(("empty_f64", O.DT_F64, np.zeros(0), None, None))
    c.append(("single_f64", O.DT_F64, np.array([2.5]), None, None))
    c.append(("const_i64", O.DT_I64, np.full(5000, 7, np.int64), None, None))
    c.append(("stride_i64", O.DT_I64, np.arange(5000, dtype=np.int64), None, None))
    c.append(("ids_i64", O.DT_I64, (1000 + np.arange(8000) % 300).astype(np.int64), None, None))
    c.append(("wide_i64", O.DT_I64, lcg(1, 4000).view(np.int64), None, None))
    ts = 1_700_000_000_000 + np.cumsum(1000 + (lcg(0x12345678, 6000) >> np.uint64(52)).astype(np.int64))
    c.append(("timestamps_i64", O.DT_I64, ts, None, None))
    c.append(("lowcard_i32", O.DT_I32, (5000 + (lcg(0x9E37, 8000) >> np.uint64(60))).astype(np.int32), None, None))
    c.append(("runs_u64", O.DT_U64, np.repeat((10**6 + np.arange(40) * 7).astype(np.uint64), 250), None, None))
    c.append(("mixed_i32", O.DT_I32, ((np.arange(6000) % 400) - 200).astype(np.int32), None, None))
    c.append(("u32_noise", O.DT_U32, (lcg(3, 3000) >> np.uint64(32)).astype(np.uint32), None, None))
    c.append(("cents_f64", O.DT_F64, (np.arange(5000) % 1000) / 100.0, None, None))
    c.append(("sine_f64", O.DT_F64, np.sin(np.arange(5000) * 1e-3) * 100.0 + np.arange(5000) * 0.01, None, None))
    walk = 20.0 + np.cumsum(rng.normal(0, 1e-3, 5000))
    c.append(("randwalk_f64", O.DT_F64, walk, None, None))
    c.append(("special_f64", O.DT_F64, np.array([0.0, -0.0, np.nan, np.inf, -np.inf, 1e308, 1e-308, 3.14159]),
              None, None))
    c.append(("sensor_f32", O.DT_F32, (np.round(rng.normal(25, 5, 6000) * 10) / 10).astype(np.float32), None, None))
    vb = rng.random(5000) > 0.1
    c.append(("nullable_ts_i64", O.DT_I64, np.cumsum(1_000_000 + rng.poisson(5000, 5000)).astype(np.int64),
              np.packbits(vb, bitorder="little"), None))
    vb2 = np.ones(7000, bool)
    vb2[1000:3000] = False
    c.append(("clustered_nulls_u64", O.DT_U64, (77 + np.arange(7000) % 5).astype(np.uint64),
              np.packbits(vb2, bitorder="little"), None))
    d = np.zeros((3000, 2), np.int64)
    d[:, 0] = rng.integers(-10**14, 10**14, 3000)
    d[:, 1] = np.where(d[:, 0] < 0, -1, 0)
    c.append(("decimal128", O.DT_DEC128, d, None, (4, 18)))
    d4 = np.zeros((1500, 4), np.int64)
    d4[:, 0] = 1_000_000 + np.arange(1500) % 500
    c.append(("decimal256", O.DT_DEC256, d4, None, (2, 40)))
    c.append(("ids_fixed256_i64", O.DT_I64, (1000 + np.arange(6000) % 777).astype(np.int64), None, None, 256))
    return c


def main():
    manifest = []
    for case in cases():
        name, dt, vals, bm, sp = case[:5]
        bs = case[5] if len(case) > 5 else None
        vals = np.ascontiguousarray(vals)
        vals.tofile(os.path.join(HERE, f"{name}.in"))
        if bm is not None:
            bm.tofile(os.path.join(HERE, f"{name}.valid"))
        entry = {"name": name, "dtype": dt, "n": int(vals.nbytes // O.NATIVE_WIDTH[dt]),
                 "validity": bm is not None, "scale": sp[0] if sp else 0, "precision": sp[1] if sp else 0,
                 "block_size": bs, "streams": {}}
        for lvl in (O.LEVEL_FASTEST, O.LEVEL_FAST):
            s = O.compress_column(vals, dt, bm, level=lvl, block_size=bs, scale=entry["scale"],
                                  precision=entry["precision"])
            fn = f"{name}.L{lvl}.stream"
            with open(os.path.join(HERE, fn), "wb") as f:
                f.write(s)
            entry["streams"][str(lvl)] = fn
        manifest.append(entry)
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    total = sum(os.path.getsize(os.path.join(HERE, x)) for x in os.listdir(HERE))
    print(f"{len(manifest)} cases, {total} bytes")


if __name__ == "__main__":
    main()
