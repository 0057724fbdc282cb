"""The multi-GPU bench path on the host: two gloo ranks (world size 2) run
bench.py's rank helpers -- barrier, the max-over-ranks time and the
whole-job throughput of independent replicas -- exactly as N GPUs do under
torchrun with NCCL (replicas only: no data-path collective)."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        bench.barrier(2)
        # rank r "took" 1 + r seconds for its replica of 1000 units
        t = bench.allreduce_max(1.0 + rank, 2)
        rate = bench.job_rate(1000.0, t, 2)
        bench.barrier(2)
        q.put((rank, t, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_as_the_slowest_replica():
    import multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, rate in out:
        assert t == 2.0, "every rank sees the slowest replica's time"
        assert rate == pytest.approx(2 * 1000.0 / 2.0)
