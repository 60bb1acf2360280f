"""Sweep sharding over ranks (host logic, CPU): the greedy partition covers
every instance exactly once, balances the estimated cost, and two gloo ranks
that compute it independently agree and gather the full result set."""
import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from fgpe_b200 import sweep

SIZES = (64, 96, 128, 192, 256, 384, 512)


def shapes(n=256, seed=4):
    rng = np.random.default_rng(seed)
    return [(int(s), int(s), 1) for s in rng.choice(SIZES, size=n)]


def test_partition_covers_and_balances():
    sh = shapes()
    for world in (1, 2, 3, 4, 8):
        own = sweep.partition(sh, world)
        assert sorted(i for r in range(world) for i in sweep.my_instances(sh, r, world)) == list(range(len(sh)))
        loads = [sum(sweep.instance_cost(sh[i]) for i in range(len(sh)) if own[i] == r) for r in range(world)]
        biggest = max(sweep.instance_cost(s) for s in sh)
        assert max(loads) - min(loads) <= biggest  # greedy LPT bound


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sh = shapes(40)
    mine = sweep.my_instances(sh, rank, world)
    # stand-in for each instance's result (its converged mu): a function of its index
    results = {i: float(i) * 0.5 for i in mine}
    gathered = [None] * world
    dist.all_gather_object(gathered, results)
    if rank == 0:
        merged = {}
        for g in gathered:
            assert not set(g) & set(merged)
            merged.update(g)
        out.put(sorted(merged.items()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_instance():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    items = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert items == [(i, i * 0.5) for i in range(40)]
