"""The multi-rank host path on CPU: two `gloo` ranks (world size 2) agree on
the job time (maximum over ranks) and split an uneven batch of slices into
disjoint, cost-balanced ranges, as `bench.py --gpus N` does with NCCL."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mr_recon_b200.shard import max_over_ranks, shard_slices


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, costs, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = max_over_ranks(10.0 + 5.0 * rank)
        b, e = shard_slices(costs, world, rank)
        out.put((rank, t, b, e))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_max_time_and_disjoint_slices():
    rng = np.random.RandomState(4)
    costs = [float(c * m) for c, m in zip(rng.randint(8, 33, 64), rng.randint(10000, 100001, 64))]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    (_, _, b0, e0), (_, _, b1, e1) = res
    assert b0 == 0 and e0 == b1 and e1 == len(costs)
    total = sum(costs)
    for b, e in ((b0, e0), (b1, e1)):
        assert abs(sum(costs[b:e]) - total / 2) <= max(costs)


@pytest.mark.parametrize("world", [1, 3, 8])
def test_shard_slices_partition(world):
    rng = np.random.RandomState(world)
    costs = list(rng.rand(37) * 10 + 1)
    ranges = [shard_slices(costs, world, r) for r in range(world)]
    covered = [i for b, e in ranges for i in range(b, e)]
    assert covered == list(range(len(costs)))
    assert shard_slices([], 2, 1) == (0, 0)
    with pytest.raises(ValueError):
        shard_slices(costs, 2, 2)


def test_max_over_ranks_without_group():
    assert max_over_ranks(3.5) == 3.5
