"""Sharding of independent systems over ranks: the partition (host logic)
and the end-of-run gather, the latter with two gloo ranks on CPU."""

import os
import socket

import numpy as np
import pytest

from amigo_b200.shard import gather_by_system, partition_systems, shard_systems
from amigo_b200.workloads import batched_optimal_control


def test_partition_covers_every_system_once_and_balances():
    rng = np.random.default_rng(1)
    costs = rng.integers(50, 400, size=97).astype(float)
    for world in (1, 2, 3, 4, 8):
        parts = partition_systems(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        assert all(p == sorted(p) for p in parts)
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max()
    # deterministic: the same partition on every call
    assert partition_systems(costs, 4) == partition_systems(list(costs), 4)


def test_partition_edge_cases():
    assert partition_systems([], 3) == [[], [], []]
    assert partition_systems([5.0], 2) == [[0], []]
    # equal costs go round-robin from rank 0
    assert partition_systems([1.0] * 5, 2) == [[0, 2, 4], [1, 3]]
    with pytest.raises(ValueError):
        partition_systems([1.0], 0)


def test_gather_without_process_group():
    out = gather_by_system(["a", "b"], [1, 0], 2)
    assert out == ["b", "a"]
    with pytest.raises(ValueError):
        gather_by_system(["a"], [0], 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, result_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = batched_optimal_control(num_systems=24, seed=0)
        idx, mine = shard_systems(systems, rank, world)
        # a per-system result that only the owning rank computes
        local = [(q.n, q.expected_inertia) for q in mine]
        out = gather_by_system(local, idx, len(systems))
        np.save(os.path.join(result_dir, f"rank{rank}.npy"),
                np.array([[n, p, m] for n, (p, m) in out]))
        np.save(os.path.join(result_dir, f"idx{rank}.npy"), np.array(idx))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_gather(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    systems = batched_optimal_control(num_systems=24, seed=0)
    want = np.array([[q.n, *q.expected_inertia] for q in systems])
    idx = [np.load(tmp_path / f"idx{r}.npy") for r in range(world)]
    assert sorted(np.concatenate(idx).tolist()) == list(range(len(systems)))
    for r in range(world):
        # every rank holds every system's result, in the batch's order
        assert np.array_equal(np.load(tmp_path / f"rank{r}.npy"), want)
