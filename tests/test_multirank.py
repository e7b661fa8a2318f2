"""The multi-rank host path on CPU: two `gloo` ranks (world size 2) agree on
the job time (maximum over ranks), split an uneven batch of slices into
disjoint, cost-balanced ranges, solve their own slices and gather the
results in slice order, as `bench.py --gpus N` does with NCCL for the
batched configuration (there the solve runs on each rank's GPU)."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mr_recon_b200.shard import gather_slices, max_over_ranks, shard_slices


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


def _uneven_batch():
    """Five independent slices of different sizes, coils and sample counts."""
    from mr_recon_b200 import synth
    rng = np.random.RandomState(21)
    sizes = [(12, 12), (16, 10), (12, 12), (14, 14), (10, 16)]
    coils = [2, 1, 3, 1, 2]
    slices = []
    for s, c in zip(sizes, coils):
        m = int(rng.randint(60, 140))
        trj = ((rng.rand(1, m, 2) - 0.5) * np.array(s)).astype(np.float32)
        mps = synth.gaussian_coil_maps(s, c)
        x = synth.randn_complex(s, rng)
        slices.append((s, trj, mps, x))
    return slices


def _solve(sl):
    """A^H A x of one slice with the oracle's SENSE model (CPU)."""
    import torch
    from oracle import nufft_oracle as O
    s, trj, mps, x = sl
    A = O.SenseOracle(trj[0], mps, O.KBNufftOracle(s, 1.25, 6))
    return torch.from_numpy(A.normal(x))


def _rank_solve(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        slices = _uneven_batch()
        costs = [float(sl[2].shape[0] * sl[1].shape[1]) for sl in slices]
        b, e = shard_slices(costs, world, rank)
        res = gather_slices([_solve(sl) for sl in slices[b:e]], b, e, len(slices))
        out.put((rank, b, e, [r.numpy() for r in res]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_and_gather_an_uneven_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_solve, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, b0, e0, r0), (_, b1, e1, r1) = res
    assert 0 < e0 == b1 < e1 == 5  # both ranks have work
    ref = [_solve(sl).numpy() for sl in _uneven_batch()]
    for got in (r0, r1):  # every rank holds every slice's result, in slice order
        assert len(got) == 5
        for g, r in zip(got, ref):
            assert np.array_equal(g, r)


def test_gather_slices_without_group():
    import torch
    t = [torch.ones(3), torch.zeros(2)]
    assert gather_slices(t, 0, 2, 2) == t
    with pytest.raises(ValueError):
        gather_slices(t, 0, 1, 2)
