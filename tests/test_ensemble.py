"""Scene sharding over ranks (host logic; world size 2 over gloo on CPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mtlphys_b200 import configs
from mtlphys_b200.ensemble import gather_scene_scalars, partition_scenes, shard_workload


def test_partition_covers_every_scene_once_and_balances():
    counts = configs.batch_counts(256, 2000, 64000, seed=7)
    for world in (1, 2, 3, 4, 8):
        shards = partition_scenes(counts, world)
        flat = sorted(s for sh in shards for s in sh)
        assert flat == list(range(len(counts)))
        loads = [int(sum(counts[s] for s in sh)) for sh in shards]
        # greedy LPT: the spread is at most the largest single scene
        assert max(loads) - min(loads) <= int(max(counts))
        assert all(sh == sorted(sh) for sh in shards)
        assert shards == partition_scenes(counts, world)  # deterministic


def test_partition_edge_cases():
    assert partition_scenes([], 3) == [[], [], []]
    assert partition_scenes([5], 2) == [[0], []]
    assert partition_scenes([3, 3, 3, 3], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition_scenes([1], 0)


def test_shard_workload_keeps_per_scene_parameters():
    w = configs.batch_cubes(num=9, lo=200, hi=3000)
    seen = []
    for r in range(2):
        sub, idx = shard_workload(w, r, 2)
        seen += idx
        assert sub.counts == [w.counts[i] for i in idx]
        assert sub.dts == [w.dts[i] for i in idx]
        assert [p.epsilon for p in sub.params] == [w.params[i].epsilon for i in idx]
    assert sorted(seen) == list(range(9))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_worker(rank, world, port, counts, out_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        idx = partition_scenes(counts, world)[rank]
        vals = [1000.0 * s + 0.125 for s in idx]  # exact in FP64
        full = gather_scene_scalars(vals, idx, len(counts), world)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array(full))
    finally:
        dist.destroy_process_group()


def test_gather_scene_scalars_over_two_gloo_ranks(tmp_path):
    counts = [int(c) for c in configs.batch_counts(11, 100, 5000, seed=3)]
    mp.start_processes(_gather_worker, args=(2, _free_port(), counts, str(tmp_path)), nprocs=2,
                       start_method="spawn")
    want = np.array([1000.0 * s + 0.125 for s in range(len(counts))])
    for r in range(2):
        np.testing.assert_array_equal(np.load(tmp_path / f"r{r}.npy"), want)


def test_gather_scene_scalars_without_a_process_group():
    assert gather_scene_scalars([2.5, -1.0], [2, 0], 3, 1) == [-1.0, 0.0, 2.5]
