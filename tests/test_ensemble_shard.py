"""Instance sharding of an ensemble over ranks (no collective in the data
path): a world-size-2 gloo run checks that the ranks' shares cover every box
exactly once, that each rank gets a near-equal share of every size, and that
every box is seeded by its global index on whichever rank runs it (the union
of the ranks' seeds is seed_base + b for every box b, with no duplicates)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

GROUPS = [(64, 16), (96, 16), (128, 16)]


SEED_BASE = 1234


def _shard(groups, world, rank):
    # qaxions_b200.shard_groups / shard_seeds, imported lazily in the children
    from qaxions_b200 import shard_groups, shard_seeds
    g, mine = shard_groups(groups, world, rank)
    return g, mine, shard_seeds(groups, world, rank, SEED_BASE)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = [None] * world
        dist.all_gather_object(got, _shard(GROUPS, world, rank))
        if rank == 0:
            out.put(got)
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_shard_groups_gloo_world2():
    pytest.importorskip("qaxions_b200")
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), q), nprocs=world, join=True, start_method="spawn")
    got = q.get()
    all_boxes = sorted(b for _, mine, _ in got for b in mine)
    nbox = sum(c for _, c in GROUPS)
    assert all_boxes == list(range(nbox))
    all_seeds = [x for _, _, seeds in got for x in seeds]
    assert sorted(all_seeds) == [SEED_BASE + b for b in range(nbox)]  # no duplicates, none missing
    size_of = [n for n, c in GROUPS for _ in range(c)]
    for groups, mine, seeds in got:
        assert sum(c for _, c in groups) == len(mine) == len(seeds)
        for n, c in groups:
            assert c == 8  # 16 boxes of each size split evenly over 2 ranks
        # local box i (numbered group by group, as Ensemble does) is global box mine[i]
        local_sizes = [n for n, c in groups for _ in range(c)]
        assert local_sizes == [size_of[b] for b in mine]
        assert seeds == [SEED_BASE + b for b in mine]


def test_shard_groups_repeated_sizes():
    from qaxions_b200 import shard_groups
    groups = [(64, 3), (96, 2), (64, 4)]
    size_of = [n for n, c in groups for _ in range(c)]
    seen = []
    for rank in range(3):
        g, mine = shard_groups(groups, 3, rank)
        assert [n for n, c in g for _ in range(c)] == [size_of[b] for b in mine]
        seen += mine
    assert sorted(seen) == list(range(9))
