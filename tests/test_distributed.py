"""Multi-rank host logic on CPU: 2 gloo ranks (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_scenes_partitions_and_balances():
    from physgrad_b200.distributed import shard_scenes

    counts = [4096 * (1 + (7 * i) % 13) for i in range(64)]
    for world in (1, 2, 3, 8):
        shards = [shard_scenes(counts, world, r) for r in range(world)]
        allidx = sorted(i for s in shards for i in s)
        assert allidx == list(range(64))
        loads = [sum(counts[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(counts)
    with pytest.raises(ValueError):
        shard_scenes(counts, 2, 2)


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from physgrad_b200.distributed import max_over_ranks, shard_scenes, sum_over_ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        counts = [10, 40, 30, 20, 50]
        mine = shard_scenes(counts, world, rank)
        local_particles = sum(counts[i] for i in mine)
        t_max = max_over_ranks(1.5 + rank)          # each rank's "device time"
        total = sum_over_ranks(local_particles)
        out[rank] = (mine, t_max, total)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    s0, s1 = res[0][0], res[1][0]
    assert sorted(s0 + s1) == [0, 1, 2, 3, 4] and not set(s0) & set(s1)
    assert res[0][1] == res[1][1] == 2.5          # max over ranks
    assert res[0][2] == res[1][2] == 150          # every particle counted once
