"""Systems and served requests spread over ranks (mfix_dem.partition): the
greedy size balance, and the metrics gather across two gloo ranks on CPU
(the only collective of the partitioned batched and served runs)."""
import os

import numpy as np
import pytest

from mfix_dem import configs
from mfix_dem.partition import gather_list, gather_metrics, loads, partition_requests, partition_work


def test_partition_covers_every_system_once_and_balances():
    rng = np.random.default_rng(3)
    work = np.exp(rng.uniform(np.log(2000), np.log(200000), 256))
    for n_ranks in (1, 2, 4, 8):
        part = partition_work(work, n_ranks)
        flat = sorted(i for p in part for i in p)
        assert flat == list(range(256))
        ld = loads(work, part)
        # LPT: the largest load is within 4/3 of the optimum, which is at
        # least the mean load and at least the largest item
        lower = max(sum(work) / n_ranks, max(work))
        assert max(ld) <= 4.0 / 3.0 * lower + 1e-9
        assert partition_work(work, n_ranks) == part  # every rank computes the same


def test_partition_of_the_batched_workload():
    systems, info = configs.batched(n_sys=64, total=400_000)
    sizes = [s[2]["pos"].shape[1] for s in systems]
    part = partition_work(sizes, 4)
    ld = loads(sizes, part)
    assert max(ld) / min(ld) < 1.05
    assert sum(ld) == sum(sizes)


def test_requests_split_in_arrival_order():
    reqs = configs.hopper_requests(40, 20.0, steps=100)
    part = partition_requests(reqs, 3)
    assert sorted(r["rid"] for p in part for r in p) == list(range(40))
    for p in part:
        arr = [r["arrival"] for r in p]
        assert arr == sorted(arr)
    ld = [sum(r["n"] * r["steps"] for r in p) for p in part]
    assert max(ld) - min(ld) <= max(r["n"] * r["steps"] for r in reqs)


def _rank_main(rank, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=2)
    try:
        rng = np.random.default_rng(11)
        work = rng.uniform(1.0, 10.0, 33)
        part = partition_work(work, 2)
        mine = part[rank]
        m = gather_metrics({"ms": 10.0 + rank, "particle_steps": float(sum(work[i] for i in mine))}, 2)
        lat = gather_list([0.1 * (rank + 1)] * (rank + 2), 2)
        out[rank] = (max(m["ms"]), sum(m["particle_steps"]), float(sum(work)), sorted(lat))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_the_partitioned_metrics():
    import torch.multiprocessing as mp
    port = 31500 + os.getpid() % 1000
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(port, out), nprocs=2, join=True)
        r0, r1 = out[0], out[1]
    assert r0 == r1
    ms, ps, total, lat = r0
    assert ms == 11.0
    assert abs(ps - total) < 1e-9 * total
    assert lat == pytest.approx([0.1, 0.1, 0.2, 0.2, 0.2])
