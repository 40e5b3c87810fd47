"""Replica path (binder_b200.replicas) as two gloo ranks on CPU: static partition of the work
list, per-unit seeds, max-over-ranks timing and the gather of per-unit results."""
import os
import socket

import numpy as np
import pytest

from binder_b200 import replicas


def test_partition_covers_every_unit_once():
    for n in (0, 1, 5, 32, 33, 64):
        for world in (1, 2, 3, 8):
            got = [u for r in range(world) for u in replicas.partition(n, r, world)]
            assert got == list(range(n))
            sizes = [len(replicas.partition(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.partition(4, 2, 2)


def test_unit_seed_independent_of_world():
    a = [replicas.unit_seed(1000, u) for r in range(2) for u in replicas.partition(32, r, 2)]
    b = [replicas.unit_seed(1000, u) for r in range(4) for u in replicas.partition(32, r, 4)]
    assert a == b == list(range(1000, 1032))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, n_units, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local = {}
        for u in replicas.partition(n_units, rank, world):
            rng = np.random.default_rng(replicas.unit_seed(1000, u))
            local[u] = rng.standard_normal(4)          # stands in for a chain's mean field
        t = replicas.max_over_ranks(0.5 + rank, dist)
        merged = replicas.gather_results(local, n_units, dist)
        if rank == 0:
            np.save(out, np.stack([merged[u] for u in range(n_units)] + [np.full(4, t)]))
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_time_and_gather(tmp_path):
    import torch.multiprocessing as mp
    n_units, world = 7, 2
    out = str(tmp_path / "merged.npy")
    mp.spawn(_worker, args=(world, _free_port(), n_units, out), nprocs=world, join=True)
    got = np.load(out)
    want = np.stack([np.random.default_rng(1000 + u).standard_normal(4) for u in range(n_units)])
    assert np.array_equal(got[:n_units], want)
    assert np.all(got[n_units] == 1.5)                 # max over ranks of 0.5 + rank


def test_gather_without_group_checks_coverage():
    assert set(replicas.gather_results({0: 1, 1: 2}, 2)) == {0, 1}
    with pytest.raises(RuntimeError):
        replicas.gather_results({0: 1}, 2)
