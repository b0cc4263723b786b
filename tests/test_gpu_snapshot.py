"""Snapshots on the GPU: saving, restoring into a fresh engine or batch and
stepping on reproduces the uninterrupted run bit for bit."""
import numpy as np
import pytest

from mtlphys_b200 import Engine, MPError, _abi, configs, snapshot
from mtlphys_b200.batch import Batch

pytestmark = pytest.mark.gpu


def test_engine_snapshot_restore_continues_bit_for_bit(cuda, tmp_path):
    w = configs.cube_drop(side=20)
    e = Engine(0)
    e.set_params(w.params)
    e.reset(w.n, w.scene, w.desc)
    for _ in range(5):
        e.step(w.dt)
    path = str(tmp_path / "engine.snap")
    e.save(path)
    saved = snapshot.read(path)
    assert saved.kind == snapshot.KIND_ENGINE and saved.particles == w.n
    np.testing.assert_array_equal(saved.positions, e.positions())
    np.testing.assert_array_equal(saved.velocities, e.velocities())
    assert abs(saved.scenes[0].params.scorr_k - w.params.scorr_k) == 0
    for _ in range(5):
        e.step(w.dt)
    want_p, want_v = e.positions(), e.velocities()
    f = Engine(0)
    f.load(path)
    assert f.particle_count() == w.n and f.current_scene() == w.scene
    for _ in range(5):
        f.step(w.dt)
    np.testing.assert_array_equal(f.positions(), want_p)
    np.testing.assert_array_equal(f.velocities(), want_v)
    e.close()
    f.close()


def test_batch_snapshot_restore_continues_bit_for_bit(cuda):
    w = configs.batch_cubes(num=3, lo=500, hi=4000)
    sp = configs.batch_spheres(num=1, lo=3000, hi=3001)
    b = Batch(0)
    b.reset(w.counts + sp.counts, w.params + sp.params, w.dts + sp.dts, w.scenes + sp.scenes,
            w.descs + sp.descs)
    for _ in range(4):
        b.step()
    data = b.snapshot_bytes()
    for _ in range(4):
        b.step()
    want_p, want_v, want_s = b.positions(), b.velocities(), b.sphere(3)
    c = Batch(0)
    c.restore_bytes(data)
    assert c.scene_count() == 4 and c.particle_count() == b.particle_count()
    for _ in range(4):
        c.step()
    np.testing.assert_array_equal(c.positions(), want_p)
    np.testing.assert_array_equal(c.velocities(), want_v)
    np.testing.assert_array_equal(c.sphere(3), want_s)
    # a batch snapshot is not an engine snapshot
    e = Engine(0)
    with pytest.raises(MPError):
        e.restore_bytes(data)
    with pytest.raises(MPError):
        c.restore_bytes(data[:100])
    for x in (b, c, e):
        x.close()
