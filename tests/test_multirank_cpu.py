"""The multi-GPU host path on CPU: two gloo ranks shard the batched solves
(independent, no collective on the data path) and take the max-over-ranks
time the way bench.py does under torchrun."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch

    from mumaxplus_b200 import batch as B
    from mumaxplus_b200 import workloads as W

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    pool = W.batch_instances(64 * world)
    mine = B.shard(pool, rank, world)
    cells = sum(W.ncells(pool[i]) for i in mine)
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, cells))
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((gathered, float(t.item()), len(pool)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_solves_and_reduce_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax, n = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (a, ca), (b, cb) = gathered
    assert sorted(a + b) == list(range(n)) and not set(a) & set(b)
    assert max(ca, cb) / min(ca, cb) < 1.05  # cell-balanced
    assert tmax == pytest.approx(2.0)
