"""Host-side logic of the batched ensemble: box sizes, LPT sharding across ranks, and a
two-rank gloo run in which every rank takes its shard and the ranks agree on the
partition (the only exchange the ensemble needs is a gather of per-box results)."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from warpsph_b200.ensemble import box_sizes, shard_boxes


def test_box_sizes_log_uniform_and_square():
    s = box_sizes(256, seed=0)
    assert len(s) == 256 and all(int(round(np.sqrt(v))) ** 2 == v for v in s)
    assert 4000 <= min(s) and max(s) <= 66000
    total = sum(s)
    assert 4.8e6 < total < 6.6e6          # E[N] ~ 22,160 per box
    assert box_sizes(256, seed=0) == s and box_sizes(256, seed=1) != s


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_lpt_shards_cover_and_balance(world):
    s = box_sizes(256, seed=0)
    parts = shard_boxes(s, world)
    flat = sorted(b for p in parts for b in p)
    assert flat == list(range(256))
    loads = [sum(s[b] for b in p) for p in parts]
    assert max(loads) - min(loads) <= max(s)           # LPT bound
    assert max(loads) <= sum(s) / world + max(s)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = box_sizes(64, seed=3)
        mine = shard_boxes(s, world)[rank]
        t = torch.zeros(64, dtype=torch.int64)
        t[mine] = rank + 1
        dist.all_reduce(t)
        out[rank] = t.tolist()
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + os.getpid() % 1000
        ps = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in ps:
            p.start()
        for p in ps:
            p.join(120)
        assert all(p.exitcode == 0 for p in ps)
        a, b = out[0], out[1]
        assert a == b and all(v in (1, 2) for v in a)    # every box on exactly one rank
