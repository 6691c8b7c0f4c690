"""The multi-GPU benchmark path (replicas, no data exchange) as two gloo
ranks on the CPU: rank-local work sums and the max-over-ranks time."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        samples = 1000.0 * (rank + 1)
        ms = 10.0 + 5.0 * rank
        tot, mx = bench.reduce_replicas(dist, samples, ms, torch.device("cpu"))
        q.put((rank, tot, mx))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replica_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, tot, mx in res:
        assert tot == 3000.0 and mx == 15.0
