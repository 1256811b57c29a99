"""Batched problems split over ranks by cost (partition_problems): the split
is the same on every rank without communication, covers every problem once
and is balanced to within one problem's cost; on gloo CPU ranks each rank
runs its share with the oracle and the gathered results equal the serial
run's.  (On GPUs each rank builds Batch.shard(...) on its own device; not
run on more than one GPU here.)"""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fluidity_b200.batch import batched_workload, partition_problems, problem_cost


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_and_balances(world):
    probs = batched_workload(seed=3, n1d=300, n2d=40)
    parts = partition_problems(probs, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(probs)))
    loads = [sum(problem_cost(probs[i][0]) for i in p) for p in parts]
    biggest = max(problem_cost(s) for s, _ in probs)
    assert max(loads) - min(loads) <= biggest
    assert parts == partition_problems(probs, world)   # deterministic


def test_partition_more_ranks_than_problems():
    probs = batched_workload(seed=1, n1d=3, n2d=0)
    parts = partition_problems(probs, 5)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1, 1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _small_workload():
    return batched_workload(seed=5, n1d=12, n2d=3, lo1=16, hi1=200, lo2=8, hi2=24)


def _run_share(probs, idx, steps):
    from oracle import oracle
    out = {}
    for i in idx:
        shape, states = probs[i]
        u = oracle.fill_riemann(shape, states, 1.4)
        res, it, rt, _ = oracle.simulate(shape, u, 1.4, 0.8, 1.0 / shape[0], 1e30, steps)
        out[i] = (res, it, rt)
    return out


def _rank_main(rank, world, port, steps, path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        probs = _small_workload()
        parts = partition_problems(probs, world)
        mine = _run_share(probs, parts[rank], steps)
        got = [None] * world
        dist.all_gather_object(got, (parts, mine))
        if rank == 0:
            np.save(path, np.array(got, dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def test_sharded_batch_on_two_ranks_matches_serial(tmp_path):
    world, steps = 2, 5
    path = str(tmp_path / "shares.npy")
    mp.start_processes(_rank_main, args=(world, _free_port(), steps, path), nprocs=world,
                       join=True, start_method="spawn")
    got = np.load(path, allow_pickle=True)
    probs = _small_workload()
    assert got[0][0] == got[1][0]                       # same split on both ranks
    merged = {}
    for _, mine in got:
        assert not set(mine) & set(merged)
        merged.update(mine)
    want = _run_share(probs, range(len(probs)), steps)
    assert sorted(merged) == sorted(want)
    for i, (res, it, rt) in want.items():
        r2, it2, rt2 = merged[i]
        assert it2 == it and rt2 == rt and np.array_equal(r2, res)


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_shards_on_one_gpu_match_whole_batch(cuda, world):
    """Batch.shard for every rank, run one after another on this GPU: each
    problem's final state, step count and time equal those of the whole
    batch (NaN where the whole batch has NaN)."""
    import torch
    from fluidity_b200.batch import Batch
    probs = batched_workload(seed=7, n1d=40, n2d=8, lo1=16, hi1=2000, lo2=16, hi2=96)
    steps = 10

    def run(b):
        b.fill()
        b.begin(0.8, 1e30, steps)
        b.steps(steps)
        # some random problems of this workload blow up: compared as they are
        it, rt, done, _ = b.status(allow_nan=True)
        torch.cuda.synchronize()
        return [(b.state(k).cpu().numpy(), it[k], rt[k]) for k in range(len(b.problems))]

    whole = run(Batch(probs, dtype="f64"))
    seen = []
    for r in range(world):
        b, idx = Batch.shard(probs, world, r, dtype="f64")
        for k, (u, it, rt) in zip(idx, run(b)):
            wu, wit, wrt = whole[k]
            assert it == wit and (rt == wrt or (np.isnan(rt) and np.isnan(wrt)))
            assert np.array_equal(u, wu, equal_nan=True)
        seen += idx
    assert sorted(seen) == list(range(len(probs)))
