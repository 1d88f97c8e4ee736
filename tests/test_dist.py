"""Replica sharding and max-over-ranks timing on CPU with gloo, world size 2."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from motioncorr1exp_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, n_items, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = D.shard(n_items, rank, world)
        t_local = 10.0 + 5.0 * rank           # per-rank "device time"
        frames_local = 40.0 * len(mine)
        out[rank] = (mine, D.max_over_ranks(t_local), D.sum_over_ranks(frames_local))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world, n_items = 2, 5
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, n_items, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    shards = [res[r][0] for r in range(world)]
    assert sorted(sum(shards, [])) == list(range(n_items))
    assert not set(shards[0]) & set(shards[1])
    assert all(res[r][1] == 15.0 for r in range(world))         # max over ranks
    assert all(res[r][2] == 40.0 * n_items for r in range(world))


def test_shard_validation():
    assert D.shard(7, 2, 3) == [2, 5]
    with pytest.raises(ValueError):
        D.shard(3, 3, 3)


def test_single_process_reductions_are_identity():
    assert D.max_over_ranks(3.5) == 3.5
    assert D.sum_over_ranks(2.0) == 2.0
