"""Instance sharding of an ensemble over ranks (no collective in the data
path): a world-size-2 gloo run checks that the ranks' shares cover every box
exactly once and that each rank gets a near-equal share of every size."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

GROUPS = [(64, 16), (96, 16), (128, 16)]


def _shard(groups, world, rank):
    # same rule as qaxions_b200.shard_groups, imported lazily in the children
    from qaxions_b200 import shard_groups
    return shard_groups(groups, world, rank)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        groups, mine = _shard(GROUPS, world, rank)
        got = [None] * world
        dist.all_gather_object(got, (groups, mine))
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
    all_boxes = sorted(b for _, mine in got for b in mine)
    assert all_boxes == list(range(sum(c for _, c in GROUPS)))
    for groups, mine in got:
        assert sum(c for _, c in groups) == len(mine)
        for n, c in groups:
            assert c == 8  # 16 boxes of each size split evenly over 2 ranks
