"""Multi-rank host logic of the benchmark on CPU (gloo, world size 2): the
max-over-ranks reduction, the whole-job throughput, and the reference arm's
rank-0-only output.  No GPU is touched."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    got = bench.max_over_ranks([1.0 + rank, 5.0 - rank], world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == [2.0, 5.0] and res[1] == [2.0, 5.0]


def test_whole_job_throughput_is_weak_scaling():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.whole_job_gbs(1e9, 1, 2, 1.0) == pytest.approx(2.0)
    assert bench.whole_job_gbs(1e9, 4, 2, 1.0) == pytest.approx(8.0)
    assert bench.max_over_ranks([3.0, 1.0], 1) == [3.0, 1.0]


def test_reference_arm_nonzero_rank_is_silent():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
