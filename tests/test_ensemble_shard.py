"""Host logic of the ensemble split over ranks (no data exchange between ranks): every
block is owned by exactly one rank, the particle counts are balanced, and two gloo ranks
agree on the split."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hidem_b200 import workloads


def test_ensemble_sizes_follow_the_configuration():
    edges, max_load = workloads.ensemble_sizes(256)
    n = 4 * edges ** 3
    assert len(n) == 256
    assert n.min() >= 4 * 11 ** 3 and n.max() <= 4 * 28 ** 3  # 5k..80k rounded to cells
    assert 5e6 < n.sum() < 8e6
    assert abs(np.median(max_load) / 5e-4 - 1) < 0.1
    assert abs(np.std(np.log(max_load)) - 0.3) < 0.05


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_partition_and_balance(world):
    edges, _ = workloads.ensemble_sizes(256)
    sizes = 4 * edges ** 3
    parts = [workloads.ensemble_shard(sizes, world, r) for r in range(world)]
    owned = sorted(i for p in parts for i in p)
    assert owned == list(range(256))
    loads = [int(sizes[p].sum()) for p in parts]
    assert max(loads) - min(loads) <= int(sizes.max())


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    edges, _ = workloads.ensemble_sizes(64)
    mine = workloads.ensemble_shard(4 * edges ** 3, world, rank)
    got = [None] * world
    dist.all_gather_object(got, mine)
    dist.destroy_process_group()
    q.put((rank, got))


def test_two_gloo_ranks_agree_on_the_split():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    views = [g for _, g in res]
    assert views[0] == views[1]
    owned = sorted(i for part in views[0] for i in part)
    assert owned == list(range(64))
