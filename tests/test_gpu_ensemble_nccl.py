"""The ensemble's scalar all-gather over NCCL on a GPU (the path `bench.py
--gpus N` and multi-GPU rollouts take).  Only one GPU is available to a
test, so the process group has one rank: the collective itself runs on the
device through NCCL, with CUDA FP64 tensors, over the per-scene gradients
of a real batched sphere-drop rollout."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, out_dir):
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from mtlphys_b200 import configs
    from mtlphys_b200.batch import Batch
    from mtlphys_b200.ensemble import gather_scene_scalars, shard_workload

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=rank, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        full = configs.batch_spheres(num=3, lo=2000, hi=6000, steps=4)
        w, idx = shard_workload(full, rank, 1)
        b = Batch(0)
        b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        b.rollout_forward(w.steps, 2)
        g = torch.zeros((b.particle_count(), 4), device="cuda")
        g[:, 1] = 1.0 / b.particle_count()
        _, _, per_scene = b.rollout_backward(g, None)
        assert b.check_errors() == 0
        local = per_scene[:, 0].double().cpu().numpy()
        gathered = gather_scene_scalars(local.tolist(), idx, len(full.counts), 1)
        b.close()
        np.save(os.path.join(out_dir, "local.npy"), local)
        np.save(os.path.join(out_dir, "gathered.npy"), np.array(gathered))
        np.save(os.path.join(out_dir, "idx.npy"), np.array(idx))
        np.save(os.path.join(out_dir, "backend.npy"), np.array([dist.get_backend() == "nccl"]))
    finally:
        dist.destroy_process_group()


def test_scene_scalars_gathered_over_nccl(tmp_path, cuda):
    mp.start_processes(_worker, args=(_free_port(), str(tmp_path)), nprocs=1, start_method="spawn")
    assert bool(np.load(tmp_path / "backend.npy")[0])
    local, idx = np.load(tmp_path / "local.npy"), np.load(tmp_path / "idx.npy")
    got = np.load(tmp_path / "gathered.npy")
    assert len(got) == 3 and sorted(idx.tolist()) == [0, 1, 2]
    assert np.isfinite(local).all() and np.abs(local).max() > 0.0
    np.testing.assert_array_equal(got[idx], local)
