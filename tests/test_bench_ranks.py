"""The multi-rank plumbing of bench.py on the host: two gloo ranks take the
maximum of their timings, aggregate whole-job throughput from it, and the
CPU reference arm runs on rank 0 alone.  (On the GPU the same helpers run
over NCCL, one replica per GPU: the path does not shard.)"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = 10.0 + 5.0 * rank                        # the slower rank sets the time
    slowest = bench.max_over_ranks(ms, world)
    bench.barrier(world)
    value = bench.aggregate(world, 1000, 4, slowest)

    class A:
        steps, warmup = 1, 1
    rc = bench.run_reference(A()) if rank != 0 else 0   # rank 1 of the CPU arm leaves without work
    dist.destroy_process_group()
    out.put((rank, slowest, value, rc))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value, rc in res:
        assert slowest == 15.0
        assert value == pytest.approx(2 * 1000 * 4 / 0.015)
        assert rc == 0
