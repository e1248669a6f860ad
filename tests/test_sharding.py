"""Box placement for the multi-GPU batched form, and its host-side exchange on two gloo
ranks (the step itself has no collective)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import ics
from sharding import lpt_shard, shard_loads


def test_lpt_covers_every_box_once_and_balances():
    specs = ics.batch_mix(64)
    costs = [sp["n"] ** 3 * 30 for sp in specs]
    for world in (1, 2, 3, 4, 8):
        sh = lpt_shard(costs, world)
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(costs)))
        loads = shard_loads(costs, sh)
        # LPT bound: max load <= (4/3 - 1/(3m)) OPT, and OPT >= mean
        assert max(loads) <= (4 / 3) * max(np.mean(loads), max(costs)) + 1e-9
        assert lpt_shard(costs, world) == sh  # deterministic
    assert lpt_shard([5, 5, 5], 5) == [[0], [1], [2], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        specs = ics.batch_mix(64)
        costs = [sp["n"] ** 3 * 30 for sp in specs]
        mine = lpt_shard(costs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = torch.tensor([float(sum(costs[i] for i in mine))])  # stands in for this rank's time
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put((gathered, float(t.item()), lpt_shard(costs, world), max(shard_loads(costs, lpt_shard(costs, world)))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_placement():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    gathered, tmax, expect, maxload = q.get()
    assert gathered == expect
    assert sorted(i for s in gathered for i in s) == list(range(64))
    assert tmax == maxload
