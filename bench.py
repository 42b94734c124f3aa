#!/usr/bin/env python3
"""Benchmark: quoin column compression/decompression on B200.

Workload (one "step"): the integer-lane configuration — three columns of
N = 67,108,864 values each (i64 ns timestamps with Poisson jitter, u64
base+U[0,2^k) runs, i32 Zipf categories in geometric runs), each 10 % null,
compressed at Level::Fast (the byte-identical level) and decompressed again.

  value   = uncompressed bytes of the three columns / (encode + decode time)
            with inputs resident in HBM (device API); the columns run
            concurrently on three CUDA streams (one context and host thread
            each); CUDA events joined across the streams, max over ranks;
  e2e     = the same metric through the host-buffer C ABI
            (quoin_b200_compress_column / quoin_b200_decompress_column) from
            pinned host memory, host<->device copies inside the timed region.

`--impl reference` times the reference algorithm's CPU implementation (the
C restatement in oracle/, since the Rust reference cannot be built here) on
all host cores, on a bounded sample of the same columns.

`--workload float-lanes` runs the float-lane columns (f64 random walk, f32
sensor readings, Decimal128) the same way; `--workload batched` compares
plain per-column calls with the batch calls on many uneven columns, and
`--workload served` drives the request server with an open-loop request
stream.

Run: python bench.py [--gpus N --steps K --warmup W] (torchrun for N > 1).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "encode+decode GB/s (uncompressed bytes; Level::Fast, bit-exact round trip)"
# --level: (C-ABI level id, oracle level id, name in the metric) for the
# single-column workloads; Fast is the headline.
LEVELS = {"fastest": (0, 0, "Fastest"), "fast": (1, 1, "Fast"), "balanced-inpool": (258, 2, "Balanced-in-pool")}


def metric_for(level: str) -> str:
    return METRIC.replace("Level::Fast", "Level::" + LEVELS[level][2])
N_DEFAULT = 67_108_864
N_PRICES = 1_048_576  # the prices column's length
L2_FLUSH_BYTES = 256 << 20  # written between timed phases when the inputs fit the 126 MB L2
TIMER_NAMES = ["compete", "emit", "decode", "finalize", "lower", "plan", "validity", "other", "read"]

# Single-column workloads: (synth config, description, arithmetic types).
WORKLOADS = {
    "integer-lanes": ("integer", "integer lanes: i64 timestamps (1e6+Poisson(5000) steps), u64 base+U[0,2^k) runs, "
                     "i32 Zipf(1.1) 64-category geometric runs; 10% nulls; Level::Fast", "int64/uint64/int32"),
    "prices": ("prices", "prices: one f64 column of two-decimal prices round(U(0,10000)*100)/100 with 3% "
                         "random-bit exceptions, no nulls; Level::Fast (the reference's Config::default() is Max, "
                         "whose Lz / Pco / range-coder candidates this encoder does not build)", "f64"),
    "float-lanes": ("float", "float lanes: f64 random walk x+N(0,1e-3) from 20.0 at full precision, f32 "
                     "round(N(25,5)*10)/10, Decimal128(18,4) uniform in [-1e14,1e14); no nulls; Level::Fast",
                "f64/f32/decimal128"),
}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per decode
# phase of the workload's three columns at the default 67,108,864 values per
# column: a one-pass ncu capture of every decode launch at 16,777,216 values
# per column (562.9 MB), scaled by the values processed (x4).
DECODE_TRAFFIC = {"integer-lanes": 2_251_622_400}


DECIMAL128_WIRE = 6  # wire dtype id of Decimal128 (reference src/dtype.rs:68-93)


def decimal_args(wire):
    """(scale, precision) of the benchmark's decimal columns; (0, 0) otherwise."""
    return (4, 18) if wire == DECIMAL128_WIRE else (0, 0)


def load_synth():
    """The column generators (quoin_b200/synth.py), loaded by path: importing
    the package would load the CUDA library, which the CPU reference arm must
    not touch."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("qb_synth", os.path.join(ROOT, "quoin_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Multi-rank plumbing (one process per GPU; every rank runs the same steps).
# ---------------------------------------------------------------------------
def max_over_ranks(values, world, device=None):
    """Element-wise maximum of a list of floats over all ranks (the slowest rank
    sets the job's time); identity for a single rank."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def whole_job_gbs(bytes_per_rank, world, steps, seconds):
    """Aggregate throughput: every rank processes bytes_per_rank per step."""
    return bytes_per_rank * world * steps / seconds / 1e9


# ---------------------------------------------------------------------------
# Reference arm: the reference's CPU algorithm (C restatement) on host cores.
# ---------------------------------------------------------------------------
def cpu_reference_run(cols, threads: int, sample: int, level: int = 1):
    from oracle import oracle as O
    enc_s = dec_s = 0.0
    nbytes = 0
    for name, dt, v, bm in cols:
        vs = v[:sample]
        bs = None if bm is None else bm[: (sample + 7) // 8]
        t0 = time.perf_counter()
        sc, pr = decimal_args(dt)
        s = O.compress_column(vs, dt, bs, level=level, scale=sc, precision=pr, threads=threads)
        t1 = time.perf_counter()
        O.decompress_column(s, threads=threads)
        t2 = time.perf_counter()
        enc_s += t1 - t0
        dec_s += t2 - t1
        nbytes += vs.nbytes
    return nbytes, enc_s, dec_s


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    synth = load_synth()
    olevel = LEVELS[args.level][1]
    threads = os.cpu_count() or 1
    # the GPU arm's workload: whole columns (batched / served: an equal share
    # of --cpu-sample per column)
    sample = args.cpu_sample if args.workload in ("batched", "served") else args.n
    if args.workload in ("batched", "served"):  # the columns, each cut to an equal share of the sample
        cols = (synth.mixed_columns(args.columns, args.max_len) if args.workload == "batched"
                else synth.request_columns(args.columns4, args.max_bytes))
        share = max(sample // len(cols), 1)
        cols = [(nm, dt, v[:share], None if bm is None else bm[: (min(len(v), share) + 7) // 8])
                for nm, dt, v, bm in cols]
        wl = (args.workload, f"{args.workload}: {len(cols)} columns of the workload, each cut to its "
                                 f"first {share} values; compress then decompress each; Level::Fast",
              "mixed (f64/f32/i64/u64/i32/u32/decimal128)")
    else:
        wl = WORKLOADS[args.workload]
        wl = (wl[0], wl[1].replace("Level::Fast", "Level::" + LEVELS[args.level][2]), wl[2])
        cols = synth.benchmark_columns(wl[0], sample)
    for _ in range(args.warmup):
        cpu_reference_run(cols, threads, sample, olevel)
    tot_b = 0
    tot_s = 0.0
    e_s = d_s = 0.0
    for _ in range(args.steps):
        b, e, d = cpu_reference_run(cols, threads, sample, olevel)
        tot_b += b
        tot_s += e + d
        e_s += e
        d_s += d
    gbs = tot_b / tot_s / 1e9
    # one host thread on a bounded part of the same columns, beside the
    # all-core figure
    one = max(min(args.single_thread_sample, sample), 1)
    cols1 = [(nm, dt, v[:one], None if bm is None else bm[: (min(len(v), one) + 7) // 8]) for nm, dt, v, bm in cols]
    b1, e1, d1 = cpu_reference_run(cols1, 1, one, olevel)
    line = {
        "impl": "reference", "metric": metric_for(args.level), "value": round(gbs, 4), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tot_s / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl[2],
        "data": "synthetic",
        "config": {"workload": wl[1], "values_per_column": sample, "columns": len(cols)},
        "encode_gbs": round(tot_b / e_s / 1e9, 4), "decode_gbs": round(tot_b / d_s / 1e9, 4),
        "cpu_baseline": {"value": round(gbs, 4), "unit": "GB/s", "cores": threads, "kind": "port",
                         "sample": (f"the whole {args.workload} columns ({sample} values each)"
                                    if sample == args.n and args.workload not in ("batched", "served") else
                                    f"first {sample} values of each {args.workload} column")
                                   + f", oracle C restatement, {threads} threads over plan_blocks ranges / frames",
                         "cpu_model": cpu_model(),
                         "single_thread": {"value": round(b1 / (e1 + d1) / 1e9, 4), "unit": "GB/s",
                                           "encode_gbs": round(b1 / e1 / 1e9, 4), "decode_gbs": round(b1 / d1 / 1e9, 4),
                                           "sample": f"first {one} values of each column, 1 thread"}},
        "e2e": {"value": round(gbs, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the Rust reference cannot be built here (no cargo, unvendored crates); its CPU path is timed "
                "through the repository's C restatement of the same algorithm",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu(args, rank, world, local):
    import torch
    import torch.distributed as dist
    import quoin_b200 as Q
    from quoin_b200 import synth

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    n = args.n
    wl = WORKLOADS[args.workload]
    wl = (wl[0], wl[1].replace("Level::Fast", "Level::" + LEVELS[args.level][2]), wl[2])
    cols = synth.benchmark_columns(wl[0], n)
    L = Q.lib
    # One context (CUDA stream + device arenas) and one host thread per column:
    # the columns' kernels overlap on the GPU, filling each other's tails.
    streams = [torch.cuda.Stream(device=dev) for _ in cols]
    ctxs = [ctypes.c_void_p(L.quoin_ctx_create(0)) for _ in cols]
    stream, ctx = streams[0], ctxs[0]
    pool = ThreadPoolExecutor(max_workers=len(cols))
    cfg = Q._QuoinConfig(LEVELS[args.level][0], 0, 16)
    P = ctypes.c_void_p

    gcols = []
    for ci, (name, wire, v, bm) in enumerate(cols):
        w = Q.NATIVE_WIDTH[wire]
        d_vals = torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).copy()).to(dev)
        d_bm = torch.from_numpy(bm.copy()).to(dev) if bm is not None else None
        cap = Q._stream_bound(wire, n, bm is not None)
        d_dst = torch.empty(cap, dtype=torch.uint8, device=dev)
        d_out = torch.empty(n * w, dtype=torch.uint8, device=dev)
        d_vout = torch.empty((n + 7) // 8, dtype=torch.uint8, device=dev)
        sc, pr = decimal_args(wire)
        gcols.append(dict(name=name, wire=wire, v=v, bm=bm, w=w, d_vals=d_vals, d_bm=d_bm, cap=cap, d_dst=d_dst,
                          d_out=d_out, d_vout=d_vout, len=0, idx=None, ctx=ctxs[ci], st=streams[ci], sc=sc, pr=pr))
    torch.cuda.synchronize()

    def compress_one(c):
        olen = ctypes.c_size_t()
        rc = L.quoin_b200_compress_column_device(
            c["ctx"], c["wire"], n, P(c["d_vals"].data_ptr()), P(c["d_bm"].data_ptr()) if c["d_bm"] is not None else None,
            c["sc"], c["pr"], ctypes.byref(cfg), P(c["d_dst"].data_ptr()), c["cap"], ctypes.byref(olen),
            P(c["st"].cuda_stream))
        if rc:
            raise Q.Error(rc)
        c["len"] = olen.value

    def decompress_one(c):
        # the stream is read on the device (header, validity, frame table)
        # inside every timed decode: no host copy, no prebuilt index
        w, nn = ctypes.c_int32(), ctypes.c_uint64()
        rc = L.quoin_b200_decompress_column_device(c["ctx"], P(c["d_dst"].data_ptr()), c["len"],
                                                   P(c["d_out"].data_ptr()), c["d_out"].numel(),
                                                   P(c["d_vout"].data_ptr()), ctypes.byref(w), ctypes.byref(nn),
                                                   P(c["st"].cuda_stream))
        if rc:
            raise Q.Error(rc)

    def compress_all():
        if args.serial_columns:
            for c in gcols:
                compress_one(c)
        else:
            list(pool.map(compress_one, gcols))

    def decompress_all():
        if args.serial_columns:
            for c in gcols:
                decompress_one(c)
        else:
            list(pool.map(decompress_one, gcols))

    def mark():
        """A timing event on stream 0 ordered after the work queued on every column stream."""
        for s in streams[1:]:
            e = torch.cuda.Event()
            e.record(s)
            streams[0].wait_event(e)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(streams[0])
        for s in streams[1:]:
            s.wait_event(ev)
        return ev

    # First pass: compress, decompress from the device stream, verify the
    # round trip bit for bit (null slots decode to 0).
    with torch.cuda.stream(stream):
        compress_all()
    with torch.cuda.stream(stream):
        decompress_all()
    torch.cuda.synchronize()
    bit_exact = True
    for c in gcols:
        got = c["d_out"].cpu().numpy()
        want = np.ascontiguousarray(c["v"]).view(np.uint8).reshape(n, c["w"]).copy()
        if c["bm"] is not None:
            valid = np.unpackbits(c["bm"], bitorder="little")[:n].astype(bool)
            want[~valid] = 0
            if c["d_vout"].cpu().numpy().tobytes() != c["bm"].tobytes():
                bit_exact = False
        if got.tobytes() != want.tobytes():
            bit_exact = False
    raw_bytes = sum(int(np.asarray(c["v"]).nbytes) for c in gcols)
    stream_bytes = sum(c["len"] for c in gcols)

    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            compress_all()
            decompress_all()
    torch.cuda.synchronize()
    # Inputs that fit in L2 (the prices column): a 256 MiB write on stream 0
    # before every timed compress and decompress, outside the timed intervals.
    flush_buf = (torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
                 if raw_bytes + stream_bytes < L2_FLUSH_BYTES else None)

    def flush():
        if flush_buf is not None:
            with torch.cuda.stream(streams[0]):
                flush_buf.fill_(1)

    # Timed region.
    L.quoin_b200_timing_enable(1)
    launches0 = Q.kernel_launches()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    if flush_buf is None:
        ev = [mark()]
        for k in range(args.steps):
            compress_all()
            ev.append(mark())
            decompress_all()
            ev.append(mark())
        enc_iv = [(ev[2 * k], ev[2 * k + 1]) for k in range(args.steps)]
        dec_iv = [(ev[2 * k + 1], ev[2 * k + 2]) for k in range(args.steps)]
    else:
        enc_iv, dec_iv = [], []
        for k in range(args.steps):
            flush()
            a = mark()
            compress_all()
            enc_iv.append((a, mark()))
            flush()
            a = mark()
            decompress_all()
            dec_iv.append((a, mark()))
    torch.cuda.synchronize()
    ms_arr = (ctypes.c_double * len(TIMER_NAMES))()
    calls_arr = (ctypes.c_uint64 * len(TIMER_NAMES))()
    L.quoin_b200_timing_read(ms_arr, calls_arr, len(TIMER_NAMES))
    L.quoin_b200_timing_enable(0)
    # The same K steps again with the columns pipelined: each column's thread
    # compresses and then decompresses on its own stream, with no join between
    # the phases, so one column's decode fills another's compress tail; the
    # steps are joined at their ends.  This loop gives `value`; the phased
    # loop above gives encode / decode GB/s, the kernel classes and the
    # roofline.  (Serial columns and L2-flushed inputs keep the phased total.)
    pipelined = flush_buf is None and not args.serial_columns and len(gcols) > 1
    if pipelined:
        def step_one(c):
            compress_one(c)
            decompress_one(c)
        pev = [mark()]
        for k in range(args.steps):
            list(pool.map(step_one, gcols))
            pev.append(mark())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    launches = Q.kernel_launches() - launches0
    enc_ms = sum(a.elapsed_time(b) for a, b in enc_iv)
    dec_ms = sum(a.elapsed_time(b) for a, b in dec_iv)
    phased_ms = ev[0].elapsed_time(ev[-1]) if flush_buf is None else enc_ms + dec_ms
    total_ms = pev[0].elapsed_time(pev[-1]) if pipelined else phased_ms
    total_ms, enc_ms, dec_ms, phased_ms = max_over_ranks([total_ms, enc_ms, dec_ms, phased_ms], world, dev)
    value = whole_job_gbs(raw_bytes, world, args.steps, total_ms / 1e3)

    # Roofline of the decode kernels (the largest kernel class per step): the
    # three columns' decode launches run together, so achieved = the decode
    # phase's algorithmic bytes (stream read + native values written + bitmap
    # copied) / the phase's event time.
    peak, peak_kind = load_peaks()
    dec_alg = stream_bytes + sum(n * c["w"] + ((n + 7) // 8 if c["bm"] is not None else 0) for c in gcols)
    achieved = dec_alg * args.steps / (dec_ms / 1e3) / 1e9 if dec_ms else 0.0
    per_class = {TIMER_NAMES[i]: (ms_arr[i], int(calls_arr[i])) for i in range(len(TIMER_NAMES))}

    # Per-column kernel-class breakdown (one untimed extra pass per column).
    per_column = {}
    for c in gcols:
        L.quoin_b200_timing_enable(1)
        compress_one(c)
        decompress_one(c)
        torch.cuda.synchronize()
        L.quoin_b200_timing_read(ms_arr, calls_arr, len(TIMER_NAMES))
        per_column[c["name"]] = {TIMER_NAMES[i]: round(ms_arr[i], 4) for i in range(len(TIMER_NAMES)) if ms_arr[i] > 0}
        per_column[c["name"]]["stream_bytes"] = c["len"]
    L.quoin_b200_timing_enable(0)

    # e2e through the host-buffer C ABI with pinned host memory.  Each column
    # runs --e2e-lanes two-stage pipelines, lane li taking steps li, li +
    # lanes, ...: one host thread compresses the lane's steps (its context),
    # another decompresses each step's stream as it arrives (a second
    # context), with two stream buffers between them, so decompresses (mostly
    # device -> host) overlap compresses (mostly host -> device) and several
    # copies are in flight per column.  --serial-columns runs compress then
    # decompress of one column at a time from one thread.
    import queue
    import threading

    lanes = 1 if args.serial_columns else max(args.e2e_lanes, 1)
    # per column and lane: a compress context, a decompress context, two
    # stream buffers and the output buffers; the inputs are shared
    cctxs = [[c["ctx"]] + [ctypes.c_void_p(L.quoin_ctx_create(0)) for _ in range(lanes - 1)] for c in gcols]
    dctxs = [[ctypes.c_void_p(L.quoin_ctx_create(0)) for _ in range(lanes)] for _ in gcols]
    pinned = []
    for c in gcols:
        hv = torch.from_numpy(np.ascontiguousarray(c["v"]).view(np.uint8).copy()).pin_memory()
        hb = torch.from_numpy(c["bm"].copy()).pin_memory() if c["bm"] is not None else None
        per_lane = []
        for _ in range(lanes):
            hdst = [torch.empty(c["len"] + (1 << 20), dtype=torch.uint8).pin_memory() for _ in range(2)]
            hout = torch.empty(n * c["w"], dtype=torch.uint8).pin_memory()
            hvout = torch.empty((n + 7) // 8, dtype=torch.uint8).pin_memory()
            per_lane.append((hdst, hout, hvout))
        pinned.append((hv, hb, per_lane))

    def e2e_compress(ci, li, slot):
        c = gcols[ci]
        hv, hb, per_lane = pinned[ci]
        hdst = per_lane[li][0]
        olen = ctypes.c_size_t()
        rc = L.quoin_b200_compress_column(cctxs[ci][li], c["wire"], n, P(hv.data_ptr()),
                                          P(hb.data_ptr()) if hb is not None else None, c["sc"], c["pr"],
                                          ctypes.byref(cfg),
                                          P(hdst[slot].data_ptr()), hdst[slot].numel(), ctypes.byref(olen))
        if rc:
            raise Q.Error(rc)
        return olen.value

    def e2e_decompress(ci, li, slot, olen):
        hdst, hout, hvout = pinned[ci][2][li]
        rc = L.quoin_b200_decompress_column(dctxs[ci][li], P(hdst[slot].data_ptr()), olen, P(hout.data_ptr()),
                                            P(hvout.data_ptr()))
        if rc:
            raise Q.Error(rc)

    def e2e_bytes():
        h2d = d2h = 0
        for c, (hv, hb, per_lane) in zip(gcols, pinned):
            hout, hvout = per_lane[0][1], per_lane[0][2]
            h2d += hv.numel() + (hb.numel() if hb is not None else 0) + c["len"]
            d2h += c["len"] + hout.numel() + (hvout.numel() if hb is not None else 0)
        return h2d, d2h

    def e2e_run(steps):
        if args.serial_columns:
            for _ in range(steps):
                for ci in range(len(gcols)):
                    e2e_decompress(ci, 0, 0, e2e_compress(ci, 0, 0))
            return
        errors = []

        def lane(ci, li, count):
            q = queue.Queue()
            free = threading.Semaphore(2)

            def produce():
                try:
                    for k in range(count):
                        free.acquire()
                        q.put((k % 2, e2e_compress(ci, li, k % 2)))
                except Exception as e:  # noqa: BLE001 - reported after the join
                    errors.append(e)
                q.put(None)

            prod = threading.Thread(target=produce)
            prod.start()
            try:
                while True:
                    item = q.get()
                    if item is None:
                        break
                    e2e_decompress(ci, li, item[0], item[1])
                    free.release()
            except Exception as e:  # noqa: BLE001
                errors.append(e)
                while prod.is_alive():  # let the producer finish its queued work
                    free.release()
                    if q.get() is None:
                        break
            prod.join()

        # lane li of a column takes steps li, li + lanes, ...
        threads = [threading.Thread(target=lane, args=(ci, li, len(range(li, steps, lanes))))
                   for ci in range(len(gcols)) for li in range(lanes)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        if errors:
            raise errors[0]

    e2e_run(1)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_run(args.steps)
    e2e_s = time.perf_counter() - t0
    h2d, d2h = e2e_bytes()
    e2e_s = max_over_ranks([e2e_s], world, dev)[0]
    e2e_gbs = whole_job_gbs(raw_bytes, world, args.steps, e2e_s)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sample = args.cpu_sample
        runs = [cpu_reference_run(cols, threads, sample, LEVELS[args.level][1]) for _ in range(3)]
        gb = sorted(b / (e + d) / 1e9 for b, e, d in runs)[1]
        cpu = {"value": round(gb, 4), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"first {sample} values of each column (of {n}), oracle C restatement, {threads} threads, "
                         f"median of 3 compress+decompress runs"}

    if rank == 0:
        line = {
            "metric": metric_for(args.level), "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl[2], "data": "synthetic",
            "config": {"workload": wl[1], "values_per_column": n, "columns": len(gcols),
                       "global_values": n * len(gcols) * world,
                       "l2": (f"inputs ({raw_bytes / 2**30:.2f} GiB per rank) exceed the 126 MB L2; no flush needed"
                              if flush_buf is None else
                              f"inputs ({raw_bytes / 2**20:.1f} MiB) fit in L2: a {L2_FLUSH_BYTES >> 20} MiB write "
                              "flushes it before every timed compress and decompress (outside the timed intervals)"),
                       "parallelism": f"replicas x{world} (each rank encodes and decodes its own copy of the columns)",
                       "concurrency": ("the three columns run one after another (--serial-columns)" if args.serial_columns
                                       else "the three columns run on three CUDA streams (one context and host "
                                            "thread each); value: every step compresses and decompresses each "
                                            "column on its stream, the columns overlapping, steps joined at their "
                                            "ends; encode/decode GB/s, kernel classes and roofline: a second K "
                                            "steps that compress all three, join, then decompress all three"
                                            if pipelined else
                                            "the three columns run on three CUDA streams (one context and host "
                                            "thread each); every step compresses all three, then decompresses "
                                            "all three")},
            "ms_per_step_phased": round(phased_ms / args.steps, 3),
            "encode_gbs": round(raw_bytes * world * args.steps / (enc_ms / 1e3) / 1e9, 3),
            "decode_gbs": round(raw_bytes * world * args.steps / (dec_ms / 1e3) / 1e9, 3),
            "ratio": round(raw_bytes / stream_bytes, 4), "bit_exact": bit_exact,
            "kernel_ms_per_step": {k: round(v[0] / args.steps, 4) for k, v in per_class.items()},
            "per_column_ms": per_column,
            "roofline": {"bound": "hbm", "kernel": "decode phase: the device stream reader (k_dp_head, "
                                                   "k_dp_bitmap, k_word_popcount, scans, k_select_table, "
                                                   "k_dp_cand_scan, k_dp_cand_compact, k_dp_succ, k_dp_marks, "
                                                   "k_dp_items, k_dp_layout, k_dp_expand) "
                                                   "and the block decoder (k_walk_frames, k_prepass, "
                                                   "k_prepass_scan, k_decode_items, k_decode_frames, "
                                                   "k_decimal_combine) of the three columns in flight together",
                         "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": DECODE_TRAFFIC.get(args.workload) if n == N_DEFAULT else None,
                         "traffic_note": ("DRAM bytes per decode phase (three decode calls): a one-pass ncu capture "
                                          "at 16,777,216 values per column scaled x4"
                                          if args.workload in DECODE_TRAFFIC and n == N_DEFAULT
                                          else "not captured for this workload and size"),
                         "decode_calls_per_step": per_class["decode"][1] // max(args.steps, 1)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "timing": ("wall clock around synchronous host-buffer C-ABI calls, pinned host memory; "
                               + ("one column at a time" if args.serial_columns else
                                  f"per column {lanes} pipeline(s), each one thread compressing its steps and "
                                  "another decompressing each step's stream (two stream buffers), so the two copy "
                                  "directions overlap"))},
            "gpu_launches": int(launches // max(args.steps, 1) * args.steps),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    pool.shutdown()
    for cx in ctxs + [x for row in cctxs for x in row[1:]] + [x for row in dctxs for x in row]:
        L.quoin_ctx_free(cx)
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Batched columns (--workload batched): many columns of uneven length
# and mixed dtype, plain per-column calls on one context vs batch calls over
# a pool of contexts (quoin_b200_*_batch_device).
# ---------------------------------------------------------------------------
def run_gpu_batched(args, rank, world, local):
    import torch
    import torch.distributed as dist
    import quoin_b200 as Q
    from quoin_b200 import synth

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    L = Q.lib
    P, S = ctypes.c_void_p, ctypes.c_size_t

    class CompressJob(ctypes.Structure):
        _fields_ = [("wire_dtype", ctypes.c_int32), ("scale", ctypes.c_int8), ("precision", ctypes.c_uint8),
                    ("n", S), ("d_values", P), ("d_validity", P), ("d_dst", P), ("dst_cap", S), ("out_len", S),
                    ("status", ctypes.c_int32)]

    L.quoin_b200_batch_create.restype = P
    L.quoin_b200_batch_create.argtypes = [ctypes.c_int]
    L.quoin_b200_batch_free.argtypes = [P]
    L.quoin_b200_compress_batch_device.argtypes = [P, ctypes.POINTER(CompressJob), S,
                                                   ctypes.POINTER(Q._QuoinConfig)]
    cfg = Q._QuoinConfig(int(Q.Level.FAST), 0, 16, 0)
    cols = synth.mixed_columns(args.columns, args.max_len)
    ctx = P(L.quoin_ctx_create(0))
    batch = P(L.quoin_b200_batch_create(args.workers))
    raw_bytes = 0
    gc = []
    for name, dt, v, bm in cols:
        nb = np.ascontiguousarray(v).nbytes
        raw_bytes += nb
        dv = torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).reshape(-1).copy()).to(dev)
        db = torch.from_numpy(bm.copy()).to(dev) if bm is not None else None
        cap = Q._stream_bound(dt, len(v), bm is not None)
        gc.append(dict(dt=dt, n=len(v), sc=4 if dt == Q.DECIMAL128 else 0, pr=18 if dt == Q.DECIMAL128 else 0,
                       dv=dv, db=db, cap=cap, dd=torch.empty(cap, dtype=torch.uint8, device=dev),
                       dout=torch.empty(max(nb, 8), dtype=torch.uint8, device=dev),
                       dvb=torch.empty(max((len(v) + 7) // 8, 1), dtype=torch.uint8, device=dev), v=v, bm=bm))
    cjobs = (CompressJob * len(gc))()
    for j, c in enumerate(gc):
        cjobs[j] = CompressJob(c["dt"], c["sc"], c["pr"], c["n"], c["dv"].data_ptr(),
                               c["db"].data_ptr() if c["db"] is not None else None, c["dd"].data_ptr(), c["cap"],
                               0, 0)
    torch.cuda.synchronize()
    # first pass: batched compress, then the batched device decode, bit-exact
    # round trip
    if L.quoin_b200_compress_batch_device(batch, cjobs, len(gc), ctypes.byref(cfg)):
        raise Q.Error(next(cjobs[j].status for j in range(len(gc)) if cjobs[j].status))

    class QueueJob(ctypes.Structure):
        _fields_ = [("d_src", P), ("src_len", S), ("d_values_out", P), ("values_cap_bytes", S),
                    ("d_validity_out", P), ("wire", ctypes.c_int32), ("n", ctypes.c_uint64),
                    ("status", ctypes.c_int32)]

    L.quoin_b200_decompress_queue_device.argtypes = [P, ctypes.POINTER(QueueJob), S, P]
    stream_bytes = 0
    qjobs = (QueueJob * len(gc))()
    for j, c in enumerate(gc):
        c["len"] = cjobs[j].out_len
        stream_bytes += c["len"]
        qjobs[j] = QueueJob(c["dd"].data_ptr(), c["len"], c["dout"].data_ptr(), c["dout"].numel(),
                            c["dvb"].data_ptr(), 0, 0, 0)
    if L.quoin_b200_decompress_queue_device(ctx, qjobs, len(gc), None):
        raise Q.Error(next(qjobs[j].status for j in range(len(gc)) if qjobs[j].status))
    torch.cuda.synchronize()
    bit_exact = True
    for c in gc:
        raw = np.ascontiguousarray(c["v"]).view(np.uint8).reshape(c["n"], -1).copy()
        if c["bm"] is not None:
            raw[~np.unpackbits(c["bm"], bitorder="little")[: c["n"]].astype(bool)] = 0
        if c["dout"][: raw.size].cpu().numpy().tobytes() != raw.tobytes():
            bit_exact = False
    rstats = (ctypes.c_uint64 * 6)()
    L.quoin_b200_reader_stats(rstats)
    queue_cols0 = rstats[5]

    def plain_compress():
        for c in gc:
            olen = ctypes.c_size_t()
            rc = L.quoin_b200_compress_column_device(
                ctx, c["dt"], c["n"], P(c["dv"].data_ptr()), P(c["db"].data_ptr()) if c["db"] is not None else None,
                c["sc"], c["pr"], ctypes.byref(cfg), P(c["dd"].data_ptr()), c["cap"], ctypes.byref(olen), None)
            if rc:
                raise Q.Error(rc)

    def plain_decompress():
        for c in gc:
            w, nn = ctypes.c_int32(), ctypes.c_uint64()
            rc = L.quoin_b200_decompress_column_device(ctx, P(c["dd"].data_ptr()), c["len"], P(c["dout"].data_ptr()),
                                                       c["dout"].numel(), P(c["dvb"].data_ptr()), ctypes.byref(w),
                                                       ctypes.byref(nn), None)
            if rc:
                raise Q.Error(rc)

    def plain():
        plain_compress()
        plain_decompress()

    def batched_decompress():
        if L.quoin_b200_decompress_queue_device(ctx, qjobs, len(gc), None):
            raise Q.Error(-14)

    def batched():
        if L.quoin_b200_compress_batch_device(batch, cjobs, len(gc), ctypes.byref(cfg)):
            raise Q.Error(-14)
        batched_decompress()

    stream = torch.cuda.current_stream(dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            fn()  # every call returns after its columns' device work completed
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks([e0.elapsed_time(e1)], world, dev)[0]

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    batched_ms = timed(batched)
    clocks = sampler.stop()
    plain_ms = timed(plain)
    dec_batched_ms = timed(batched_decompress)
    dec_plain_ms = timed(plain_decompress)
    L.quoin_b200_reader_stats(rstats)
    queue_cols = (rstats[5] - queue_cols0) // max(2 * (args.warmup + args.steps), 1)
    value = whole_job_gbs(raw_bytes, world, args.steps, batched_ms / 1e3)
    plain_gbs = whole_job_gbs(raw_bytes, world, args.steps, plain_ms / 1e3)
    L.quoin_b200_batch_free(batch)
    L.quoin_ctx_free(ctx)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(batched_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "mixed (f64/f32/i64/u64/i32/u32/decimal128)",
            "data": "synthetic",
            "config": {"workload": f"batched: {len(gc)} columns, lengths floor(exp(U[ln 1024, ln {args.max_len}])), "
                                   "dtype uniform over 7, null rate U(0,0.2); Level::Fast",
                       "columns": len(gc), "global_values": int(sum(c["n"] for c in gc)) * world,
                       "uncompressed_bytes": raw_bytes, "workers": args.workers,
                       "parallelism": f"replicas x{world}"},
            "plain_gbs": round(plain_gbs, 3), "batched_over_plain": round(value / plain_gbs, 3) if plain_gbs else None,
            "decode": {"batched_gbs": round(whole_job_gbs(raw_bytes, world, args.steps, dec_batched_ms / 1e3), 3),
                       "plain_gbs": round(whole_job_gbs(raw_bytes, world, args.steps, dec_plain_ms / 1e3), 3),
                       "columns_per_batched_call": int(queue_cols)},
            "ratio": round(raw_bytes / stream_bytes, 4), "bit_exact": bit_exact,
            "cpu_baseline": None, "clocks": clocks,
            "note": "plain = per-column compress_column_device / decompress_column_device calls on one context; "
                    "value = the same columns through the batch compress (a pool of contexts) and the batched "
                    "device decode (quoin_b200_decompress_queue_device: one launch per kernel class for the "
                    "batch)",
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# Served requests (--workload served): an open-loop Poisson request
# stream (70% decompress, 30% compress) over resident columns, served by the
# request server (a pool of contexts, FIFO admission against a 120 GB device
# budget) and by the plain per-request path (one context, one request at a
# time), at offered loads from 10% to 100% of the server's measured peak.
# ---------------------------------------------------------------------------
def run_gpu_served(args, rank, world, local):
    import torch
    import torch.distributed as dist
    import quoin_b200 as Q
    from quoin_b200 import synth

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    L = Q.lib
    P, S, U64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64

    class Request(ctypes.Structure):
        _fields_ = [("op", ctypes.c_int32), ("wire_dtype", ctypes.c_int32), ("scale", ctypes.c_int8),
                    ("precision", ctypes.c_uint8), ("n", S), ("d_values", P), ("d_validity", P), ("d_dst", P),
                    ("dst_cap", S), ("idx", P), ("d_src", P), ("d_values_out", P), ("d_validity_out", P),
                    ("device_bytes", U64), ("out_len", S), ("status", ctypes.c_int32), ("done", ctypes.c_int32),
                    ("t_submit_ns", U64), ("t_start_ns", U64), ("t_end_ns", U64)]

    L.quoin_b200_server_create.restype = P
    L.quoin_b200_server_create.argtypes = [ctypes.c_int, U64, ctypes.POINTER(Q._QuoinConfig)]
    L.quoin_b200_server_submit.argtypes = [P, ctypes.POINTER(Request)]
    L.quoin_b200_server_wait.argtypes = [P, ctypes.POINTER(Request), ctypes.c_int]
    L.quoin_b200_server_peak_bytes.argtypes = [P]
    L.quoin_b200_server_peak_bytes.restype = U64
    L.quoin_b200_server_free.argtypes = [P]
    cfg = Q._QuoinConfig(int(Q.Level.FAST), 0, 16, 0)
    budget = 120 << 30

    # Resident columns: values, a compressed copy (source of the decompress
    # requests) with its decode index, and output buffers.  Concurrent requests
    # on one column write the same bytes to its shared outputs.
    cols = synth.request_columns(args.columns4, args.max_bytes)
    ctx = P(L.quoin_ctx_create(0))
    tpl = []
    resident = 0
    for name, dt, v, bm in cols:
        n = len(v)
        nb = np.ascontiguousarray(v).nbytes
        dv = torch.from_numpy(np.ascontiguousarray(v).view(np.uint8).reshape(-1).copy()).to(dev)
        db = torch.from_numpy(bm.copy()).to(dev) if bm is not None else None
        cap = Q._stream_bound(dt, n, bm is not None)
        dd = torch.empty(cap, dtype=torch.uint8, device=dev)
        sc, pr = (4, 18) if dt == Q.DECIMAL128 else (0, 0)
        olen = ctypes.c_size_t()
        rc = L.quoin_b200_compress_column_device(ctx, dt, n, P(dv.data_ptr()), P(db.data_ptr()) if db is not None else None,
                                                 sc, pr, ctypes.byref(cfg), P(dd.data_ptr()), cap, ctypes.byref(olen), None)
        if rc:
            raise Q.Error(rc)
        hs = dd[: olen.value].cpu().numpy().tobytes()
        ds = torch.from_numpy(np.frombuffer(hs, np.uint8).copy()).to(dev)
        idx = P()
        if L.quoin_b200_index_create(ctx, hs, len(hs), ctypes.byref(idx)):
            raise Q.Error(-14)
        dout = torch.empty(max(nb, 8), dtype=torch.uint8, device=dev)
        dvb = torch.empty(max((n + 7) // 8, 1), dtype=torch.uint8, device=dev)
        resident += dv.numel() + cap + ds.numel() + dout.numel() + dvb.numel()
        tpl.append(dict(dt=dt, n=n, nb=nb, sc=sc, pr=pr, dv=dv, db=db, dd=dd, cap=cap, ds=ds, slen=len(hs), idx=idx,
                        dout=dout, dvb=dvb))
    torch.cuda.synchronize()

    def request(t, op):
        c = tpl[t]
        if op == 0:
            return Request(op=0, wire_dtype=c["dt"], scale=c["sc"], precision=c["pr"], n=c["n"],
                           d_values=c["dv"].data_ptr(), d_validity=c["db"].data_ptr() if c["db"] is not None else None,
                           d_dst=c["dd"].data_ptr(), dst_cap=c["cap"], device_bytes=c["nb"] + c["cap"])
        return Request(op=1, idx=c["idx"], d_src=c["ds"].data_ptr(), d_values_out=c["dout"].data_ptr(),
                       d_validity_out=c["dvb"].data_ptr(), device_bytes=c["slen"] + c["nb"])

    rng = np.random.default_rng(20261203 + 400)

    def draw(k):
        """k requests: (column, op) with 70% decompress."""
        return [(int(rng.integers(0, len(tpl))), 0 if rng.random() < 0.3 else 1) for _ in range(k)]

    def serve(srv, reqs, arrivals):
        """Submits reqs at the arrival offsets (seconds; None = all at once), waits for all;
        returns (GB/s, latencies in ms)."""
        rs = [request(t, op) for t, op in reqs]
        t0 = time.perf_counter()
        for i, r in enumerate(rs):
            if arrivals is not None:
                d = t0 + arrivals[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            rc = L.quoin_b200_server_submit(srv, ctypes.byref(r))
            if rc:
                raise Q.Error(rc)
        for r in rs:
            rc = L.quoin_b200_server_wait(srv, ctypes.byref(r), -1)
            if rc:
                raise Q.Error(rc)
        nbytes = sum(tpl[t]["nb"] for t, _ in reqs)
        span = (max(r.t_end_ns for r in rs) - min(r.t_submit_ns for r in rs)) / 1e9
        lat = np.array([(r.t_end_ns - r.t_submit_ns) / 1e6 for r in rs])
        return nbytes / span / 1e9, lat

    pool = P(L.quoin_b200_server_create(args.workers, budget, ctypes.byref(cfg)))
    plain = P(L.quoin_b200_server_create(1, budget, ctypes.byref(cfg)))
    # Warm-up: every context meets the largest columns (its arenas grow once,
    # outside the timed loads), then every column.
    big = sorted(range(len(tpl)), key=lambda t: -tpl[t]["nb"])[:2]
    for _ in range(max(args.warmup, 1)):
        for t in big:
            for op in (0, 1):
                serve(pool, [(t, op)] * args.workers, None)
        serve(pool, [(t, op) for t in range(len(tpl)) for op in (0, 1)] * 2, None)
        serve(plain, [(t, op) for t in range(len(tpl)) for op in (0, 1)], None)
    peak_reqs = draw(args.requests)
    peak_gbs, _ = serve(pool, peak_reqs, None)
    mean_bytes = float(np.mean([tpl[t]["nb"] for t, _ in peak_reqs]))
    sampler = ClockSampler(local)
    sampler.start()
    loads = []
    for pct in range(10, 101, 10):
        reqs = draw(args.requests)
        rate = pct / 100.0 * peak_gbs * 1e9 / mean_bytes  # requests per second
        arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
        row = {"offered": pct / 100.0, "offered_gbs": round(pct / 100.0 * peak_gbs, 3)}
        for key, srv in (("server", pool), ("plain", plain)):
            gbs, lat = serve(srv, reqs, arrivals)
            row[key] = {"gbs": round(gbs, 3), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                        "p99_ms": round(float(np.percentile(lat, 99)), 3)}
        loads.append(row)
    clocks = sampler.stop()
    peak_held = L.quoin_b200_server_peak_bytes(pool)
    L.quoin_b200_server_free(pool)
    L.quoin_b200_server_free(plain)
    for c in tpl:
        L.quoin_b200_index_free(c["idx"])
    L.quoin_ctx_free(ctx)
    top = loads[-1]
    if rank == 0:
        line = {
            "metric": "served GB/s (uncompressed bytes; 70% decompress / 30% compress, Level::Fast, open-loop "
                      "Poisson arrivals at 100% of the measured peak)",
            "value": top["server"]["gbs"], "unit": "GB/s", "n_gpus": world, "steps": len(loads),
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "mixed (f64/f32/i64/u64/i32/u32/decimal128)", "data": "synthetic",
            "config": {"workload": f"served: {len(tpl)} resident columns, sizes floor(exp(U[ln 64 KiB, "
                                   f"ln {args.max_bytes >> 20} MiB])) bytes, dtypes and generators of the batched "
                                   "columns; "
                                   f"{args.requests} requests per offered load",
                       "workers": args.workers, "budget_bytes": budget, "resident_bytes": resident,
                       "mean_request_bytes": int(mean_bytes), "parallelism": f"replicas x{world}"},
            "peak_gbs": round(peak_gbs, 3), "loads": loads, "peak_admitted_bytes": int(peak_held),
            "server_over_plain_at_100pct": round(top["server"]["gbs"] / top["plain"]["gbs"], 3)
            if top["plain"]["gbs"] else None,
            "cpu_baseline": None, "clocks": clocks,
            "note": "server = the request server over a pool of contexts; plain = the same arrivals served one "
                    "request at a time on one context; latency = completion - submission (queueing included)",
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=None,
                    help="values per column (default 67,108,864; 1,048,576 for the prices workload)")
    ap.add_argument("--cpu-sample", type=int, default=1 << 24,
                    help="values per column of the GPU arm's cpu_baseline leg (and of the batched / served "
                         "reference arm)")
    ap.add_argument("--single-thread-sample", type=int, default=1 << 21,
                    help="reference arm: values per column of the one-thread run")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--e2e-lanes", type=int, default=1,
                    help="e2e: compress/decompress pipelines per column (each its own contexts and buffers)")
    ap.add_argument("--serial-columns", action="store_true",
                    help="one host thread runs the columns one after another (for profilers)")
    ap.add_argument("--workload", default="integer-lanes",
                    choices=["integer-lanes", "float-lanes", "prices", "batched", "served"],
                    help="batched: many uneven columns (plain vs batch calls); served: the request stream")
    ap.add_argument("--level", default="fast", choices=list(LEVELS),
                    help="single-column workloads: compression level (Fast is the headline)")
    ap.add_argument("--columns", type=int, default=256, help="batched: number of columns")
    ap.add_argument("--max-len", type=int, default=1 << 21, help="batched: longest column")
    ap.add_argument("--workers", type=int, default=8, help="batched / served: contexts in the batch / server")
    ap.add_argument("--columns4", type=int, default=24, help="served: resident columns")
    ap.add_argument("--max-bytes", type=int, default=256 << 20, help="served: largest column")
    ap.add_argument("--requests", type=int, default=600, help="served: requests per offered load")
    args = ap.parse_args()
    if args.level != "fast" and args.workload in ("batched", "served"):
        ap.error("--level applies to the single-column workloads")
    if args.n is None:
        args.n = N_PRICES if args.workload == "prices" else N_DEFAULT
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batched":
        return run_gpu_batched(args, rank, world, local)
    if args.workload == "served":
        return run_gpu_served(args, rank, world, local)
    return run_gpu(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
