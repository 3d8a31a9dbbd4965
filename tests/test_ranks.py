"""The multi-rank host logic of bench.py on CPU, world size 2 over gloo: the max-over-ranks time and
the whole-job rate of independent replicas, and the reference arm under torchrun (rank 0 alone
measures and prints one line; the other rank exits 0 without work)."""

import datetime
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))  # fmt: skip
    try:
        ms = bench.reduce_max(10.0 + 5.0 * rank, dist)  # rank 1 is the slow one
        rate = bench.whole_job_rate(world, 1000, 4, ms * 1e-3)
        dist.barrier()
        out.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate in got:
        assert ms == 15.0  # every rank sees the slowest rank's time
        assert rate == pytest.approx(2 * 1000 * 4 / 0.015)


def test_single_process_reduce_is_identity():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench.reduce_max(3.5) == 3.5
    assert bench.whole_job_rate(1, 10, 2, 0.5) == 40.0


def test_reference_arm_under_torchrun_two_ranks():
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), "bench.py",
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
           "--workload", "hex", "--cpu-threads", "2"]  # fmt: skip
    r = subprocess.run(cmd, cwd=REPO, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2
    assert line["metric"] == "cell-iterations/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 2
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_cases_shard_whole_and_balanced():
    """The batch workload's sharding: every case on exactly one rank, ranks' cell totals within
    the largest case of each other, the same draws whatever the number of ranks."""
    sys.path.insert(0, str(REPO))
    from autan_b200 import cases

    params = cases.batch_parameters(256, 0, (20_000, 500_000))
    size = [1.111 * float(np.prod(p["boxes"])) for p in params]
    for ranks in (1, 2, 4, 8):
        parts = cases.shard_cases(params, ranks)
        flat = sorted(k for part in parts for k in part)
        assert flat == list(range(256))
        loads = [sum(size[k] for k in part) for part in parts]
        assert max(loads) - min(loads) <= max(size)
    assert cases.batch_parameters(256, 0, (20_000, 500_000)) == params


def test_reduce_sum_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_sum_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [30.0, 30.0]


def _sum_rank(rank: int, world: int, port: int, out) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))  # fmt: skip
    try:
        out.put((rank, bench.reduce_sum(10.0 + 10.0 * rank, dist)))
    finally:
        dist.destroy_process_group()
