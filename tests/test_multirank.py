"""The replicas-only multi-GPU path of bench.py: each rank times its own
replica and rank 0 reports all ranks' work over the slowest rank's time.
Exercised here with two gloo ranks on the CPU (no GPU, no NCCL)."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    ms = [40.0, 55.0][rank]  # rank 1 is the slowest replica
    bench.barrier(world)
    mx = bench.all_max(ms, world)
    rate = bench.whole_job_rate(1_000_000, 10, world, mx)
    out[rank] = (mx, rate)
    dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    for r in range(2):
        mx, rate = out[r]
        assert mx == 55.0
        assert rate == pytest.approx(2 * 10 * 1_000_000 / 0.055)
