"""World-size-2 gloo run of the multi-GPU plumbing on the CPU: every estimation lands on
exactly one rank, seeds differ across ranks, and the job time is the max over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_items, q):
    sys.path.insert(0, os.path.join(REPO, "parallelkde.jl_b200"))
    import datetime

    import torch
    import torch.distributed as dist
    from pkde_b200 import multi
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = multi.shard(n_items, rank, world)
    seeds = [multi.estimation_seed(rank, k) for k in range(len(mine))]
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, seeds))
    t = multi.max_over_ranks(10.0 * (rank + 1), dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, gathered, t))


@pytest.mark.parametrize("n_items", [1, 7, 8])
def test_two_rank_sharding(n_items):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n_items, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, t in out:
        assert t == 20.0  # max over ranks
        items = [i for shard, _ in gathered for i in shard]
        assert sorted(items) == list(range(n_items))  # each estimation on exactly one rank
        seeds = [s for _, ss in gathered for s in ss]
        assert len(set(seeds)) == len(seeds)
