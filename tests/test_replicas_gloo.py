"""Multi-rank path of bench.py on the CPU (gloo, world size 2): the workload is replicated, one
independent grid per rank, so the only cross-rank step is the reduction of the timing (max)
and of the work (sum)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms, acc = bench.aggregate_over_ranks(dist, ms=10.0 + 5.0 * rank, accepted=500 - rank, device=torch.device("cpu"))
    q.put((rank, ms, acc))
    dist.barrier()
    dist.destroy_process_group()


def test_aggregate_over_two_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, acc in res:
        assert ms == 15.0 and acc == 999
