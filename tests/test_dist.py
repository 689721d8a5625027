"""CPU tests of the multi-process plumbing with world size 2 over gloo:
max-over-ranks timing and the batch sharding (no GPU, no collective on the
data path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gb_b200 import dist, synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = dist.max_over_ranks(10.0 + rank)
        mats = [synth.random_macaulay(10 + 5 * i, 5 + i, 12, 101, seed=i) for i in range(7)]
        shards = dist.shard_batch(mats, world)
        q.put((rank, got, shards))
    finally:
        td.destroy_process_group()


def test_max_over_ranks_and_sharding_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [11.0, 11.0]          # max over ranks on every rank
    assert res[0][2] == res[1][2]                       # same deterministic shards
    shards = res[0][2]
    assert sorted(i for s in shards for i in s) == list(range(7))


def test_shard_batch_balances_work():
    mats = [synth.random_macaulay(20, 10, 30, 101, seed=i) for i in range(9)]
    shards = dist.shard_batch(mats, 3)
    loads = [sum(dist.work_estimate(mats[i]) for i in s) for s in shards]
    assert max(loads) <= 2.5 * min(loads)
    assert dist.max_over_ranks(3.5) == 3.5  # not distributed: identity
