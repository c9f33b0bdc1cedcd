"""The multi-rank plumbing on CPU (gloo, world size 2): the max-over-ranks
timing reduction of bench.py and the instance partition that shards batches
(plates, RVEs) over ranks with no data-path collective."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), AKB_DIST_BACKEND="gloo")
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist

    import bench
    from akantu_b200.batch import partition_instances
    d = bench.Dist(world)
    try:
        mine = partition_instances(sizes, world)[rank]
        elems = float(sum(sizes[i] for i in mine))
        t_rank = 1.0 + rank  # a "device time" that differs per rank
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out[rank] = dict(max=d.max(t_rank), total=d.sum(elems), parts=gathered)
    finally:
        d.close()


def test_partition_covers_and_balances():
    from akantu_b200.batch import partition_instances
    rng = np.random.default_rng(0)
    sizes = np.exp(rng.uniform(np.log(100), np.log(20000), 4096)).astype(int)
    for world in (1, 2, 3, 8):
        parts = partition_instances(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) - min(loads) <= sizes.max()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_agree():
    sizes = list(np.random.default_rng(1).integers(100, 5000, 300))
    world, port = 2, _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, sizes, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0]["max"] == res[1]["max"] == 2.0
    assert res[0]["total"] == res[1]["total"] == float(sum(sizes))
    assert res[0]["parts"] == res[1]["parts"]
    a, b = res[0]["parts"]
    assert not set(a) & set(b) and len(a) + len(b) == len(sizes)
