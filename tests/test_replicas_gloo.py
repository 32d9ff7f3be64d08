"""The N>1 path on CPU: two gloo ranks partition the units without
communication and agree on the max-over-ranks time."""
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


def _worker(rank, world, port, costs, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from cudalatticegauge_b200.replicas import max_over_ranks, rank_seed, shard_units

    mine = shard_units(costs, world, rank)
    t = max_over_ranks(1.0 + rank)
    q.put((rank, mine, t, rank_seed(0xC1A60001, rank)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding():
    # 12 point sources + 16 noise sources on 32^3x32, plus the five uneven lattices
    costs = [1.0] * 28 + [4096, 20736, 65536, 131072, 221184]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    parts = [set(r[1]) for r in res]
    assert parts[0].isdisjoint(parts[1])
    assert parts[0] | parts[1] == set(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.2
    assert all(r[2] == 2.0 for r in res)
    assert res[0][3] != res[1][3]


def test_sharding_single_rank_is_everything():
    from cudalatticegauge_b200.replicas import shard_units

    assert shard_units([3, 1, 2], 1, 0) == [0, 1, 2]
    with pytest.raises(ValueError):
        shard_units([1], 2, 2)
