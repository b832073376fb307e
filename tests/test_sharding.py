"""Rank logic of the multi-GPU path, on CPU: the forest split by problem
(each problem on exactly one rank, loads within one problem of the even
share) and the max-over-ranks timing reduction, run as two gloo ranks."""
import os

import numpy as np
import pytest

from fmma_b200.sharding import forest_shard, max_over_ranks, sub_forest


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_forest_shard_covers_every_problem_once(world):
    sizes = np.exp(np.random.default_rng(world).uniform(np.log(1e3), np.log(2e5), 512)).astype(np.int64)
    shards = [forest_shard(sizes, world, r) for r in range(world)]
    allp = np.sort(np.concatenate(shards))
    assert np.array_equal(allp, np.arange(len(sizes)))
    loads = np.array([sizes[s].sum() for s in shards])
    assert loads.max() - sizes.sum() / world <= sizes.max()


def test_sub_forest_gathers_the_problems():
    toff = np.array([0, 3, 3, 7, 10])
    soff = np.array([0, 2, 5, 5, 9])
    st, ss, ti, si = sub_forest(toff, soff, [2, 0])
    assert st.tolist() == [0, 4, 7] and ss.tolist() == [0, 0, 2]
    assert ti.tolist() == [3, 4, 5, 6, 0, 1, 2] and si.tolist() == [0, 1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = np.arange(1, 41) * 100
        mine = forest_shard(sizes, world, rank)
        got = max_over_ranks([1.0 + rank, 10.0 - rank])
        gathered = [None] * world
        dist.all_gather_object(gathered, mine.tolist())
        q.put((rank, got, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_split():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, gathered in res:
        assert got == [2.0, 10.0]
        assert sorted(gathered[0] + gathered[1]) == list(range(40))
        assert not set(gathered[0]) & set(gathered[1])
