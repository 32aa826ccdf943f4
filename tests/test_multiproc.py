"""The multi-process (one process per GPU, replicas) plumbing of bench.py,
exercised on CPU with the gloo backend and world size 2: the slowest rank's
time is the job's, the job value counts every rank's transforms, and under
torchrun the reference arm prints one line from rank 0 while the other ranks
exit without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v = bench.max_over_ranks(dist, 10.0 + 5.0 * rank)
        q.put((rank, v))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_gloo_world_size_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 15.0, 1: 15.0}


def test_job_value_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench
    one = bench.job_value(1, 1e9, 10, 100.0)
    assert abs(one - 100.0) < 1e-9                      # 10 GFLOP in 0.1 s
    assert abs(bench.job_value(4, 1e9, 10, 100.0) - 4 * one) < 1e-9


def test_reference_arm_under_torchrun_prints_one_line():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", "--impl", "reference",
           "--gpus", "2", "--log2n", "16", "--segments", "8", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    if "unavailable" not in line:
        assert line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
        assert line["cpu_baseline"]["kind"] in ("reference", "port")
