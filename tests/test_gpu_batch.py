"""The multi-scene batch on the GPU (no reference counterpart): one
persistent launch per step gives, bit for bit, what the same kernel launched
scene by scene gives and what a single-scene Engine gives each scene; a step
of every scene matches the FP64 oracle."""
import numpy as np
import pytest

from mtlphys_b200 import Engine, _abi, configs
from mtlphys_b200.batch import Batch
from oracle import oracle as O
from parity import assert_equal_u32, assert_positions, position_tolerance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch(cuda):
    b = Batch(0)
    yield b
    b.close()


def small_cubes(num=10, steps=8):
    return configs.batch_cubes(num=num, lo=200, hi=9000, steps=steps)


def small_spheres(num=3):
    w = configs.batch_spheres(num=num, lo=3000, hi=12000, steps=6)
    return w


def load(b, w):
    b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)


def run(b, w, steps):
    for _ in range(steps):
        b.step()
    assert b.check_errors() == 0
    return b.positions(), b.velocities()


def test_batched_and_serial_are_bit_identical(batch):
    w = small_cubes()
    load(batch, w)
    batch.set_serial(False)
    a = run(batch, w, w.steps)
    load(batch, w)
    batch.set_serial(True)
    b = run(batch, w, w.steps)
    batch.set_serial(False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_batch_gives_each_scene_the_single_engine_result(batch, cuda):
    w = small_cubes(num=6, steps=6)
    load(batch, w)
    pos, vel = run(batch, w, w.steps)
    e = Engine(0)
    try:
        for s in range(len(w.counts)):
            e.set_params(w.params[s])
            e.reset(w.counts[s], w.scenes[s], w.descs[s])
            for _ in range(w.steps):
                e.step(w.dts[s])
            f, n = batch.scene_range(s)
            assert n == w.counts[s]
            assert np.array_equal(e.positions(), pos[f:f + n]), f"scene {s} positions"
            assert np.array_equal(e.velocities(), vel[f:f + n]), f"scene {s} velocities"
    finally:
        e.close()


def test_batch_step_matches_the_oracle_per_scene(batch):
    w = small_cubes(num=5, steps=4)
    w.params = [p.copy() for p in w.params]
    for p in w.params:
        p.scorr_k = 1e-4  # a well-conditioned step: the strict bound applies
    load(batch, w)
    pos, vel = run(batch, w, 4)
    batch.step()
    assert batch.check_errors() == 0
    got = batch.positions()
    for s in range(len(w.counts)):
        f, n = batch.scene_range(s)
        p, v = pos[f:f + n], vel[f:f + n]
        o = O.step(w.params[s], w.dts[s], p, v)
        tol = position_tolerance(w.params[s], w.dts[s], p, v)
        assert_positions(got[f:f + n], o["pos"], tol, what=f"scene {s} positions")


def test_graph_mode_and_launch_shapes_give_identical_results(batch):
    w = small_cubes(num=8, steps=5)
    ref = None
    for block, graph in ((256, False), (128, True), (512, False)):
        load(batch, w)
        batch.set_launch(block, 0)
        batch.set_graph_mode(graph)
        out = run(batch, w, w.steps)
        batch.set_graph_mode(False)
        if ref is None:
            ref = out
        else:
            assert np.array_equal(ref[0], out[0]) and np.array_equal(ref[1], out[1])
    batch.set_launch(256, 0)


def test_autotune_picks_a_shape_without_advancing_the_scenes(batch):
    w = small_cubes(num=8, steps=3)
    load(batch, w)
    before = batch.positions()
    t = batch.autotune(steps=2)
    assert t["block"] in (128, 256, 512) and t["blocks_per_sm"] >= 1 and t["ms_per_step"] > 0
    assert np.array_equal(before, batch.positions())
    assert batch.launch()[0] == t["block"]


def test_sphere_scenes_match_single_engines(batch, cuda):
    w = small_spheres()
    load(batch, w)
    pos, vel = run(batch, w, w.steps)
    e = Engine(0)
    try:
        for s in range(len(w.counts)):
            e.set_params(w.params[s])
            e.reset(w.counts[s], w.scenes[s], w.descs[s])
            for _ in range(w.steps):
                e.step(w.dts[s])
            f, n = batch.scene_range(s)
            assert np.array_equal(e.positions(), pos[f:f + n]), f"scene {s}"
            assert np.array_equal(e.sphere(), batch.sphere(s))
    finally:
        e.close()


def test_empty_and_single_particle_scenes(batch):
    w = small_cubes(num=4, steps=3)
    w.counts[1] = 0
    w.counts[2] = 1
    load(batch, w)
    pos, vel = run(batch, w, 3)
    assert batch.scene_range(1)[1] == 0
    assert np.isfinite(pos).all()


def test_random_cloud_scenes(batch, cuda):
    """Three seeded random clouds (tight clumps, points outside the grid,
    random velocities) as scenes of one batch: each scene's bounding box of
    cells holds outliers and crowded cells, and particles leave it during the
    step.  Batched and scene-by-scene launches agree bit for bit, each scene
    equals a single-scene engine bit for bit, and each meets the oracle."""
    from parity import random_scene

    p = _abi.default_params()
    clouds = [random_scene(seed, n) for seed, n in ((5, 800), (6, 2500), (7, 1500))]
    counts = [len(c[0]) for c in clouds]
    dt = 1.0 / 240.0
    results = []
    for serial in (False, True):
        batch.reset(counts, [p] * 3, [dt] * 3, [_abi.MP_SCENE_CUBE_DROP] * 3, None)
        batch.set_serial(serial)
        pos0, vel0 = batch.positions(), batch.velocities()
        for s, (cp, cv) in enumerate(clouds):
            f, n = batch.scene_range(s)
            pos0[f:f + n], vel0[f:f + n] = cp, cv
        batch.write(_abi.MP_BUF_POSITIONS, pos0)
        batch.write(_abi.MP_BUF_VELOCITIES, vel0)
        for _ in range(2):
            batch.step()
        assert batch.check_errors() == 0
        results.append((batch.positions(), batch.velocities()))
    batch.set_serial(False)
    for x, y in zip(*results):
        assert np.array_equal(x, y)
    pos, vel = results[0]
    e = Engine(0)
    try:
        for s, (cp, cv) in enumerate(clouds):
            e.set_params(p)
            e.reset(len(cp), _abi.MP_SCENE_CUBE_DROP)
            e.set_positions(cp)
            e.set_velocities(cv)
            e.step(dt)
            mid_p, mid_v = e.positions(), e.velocities()
            e.step(dt)
            f, n = batch.scene_range(s)
            assert np.array_equal(e.positions(), pos[f:f + n]), f"scene {s} positions"
            assert np.array_equal(e.velocities(), vel[f:f + n]), f"scene {s} velocities"
            o = O.step(p, dt, mid_p, mid_v)
            assert_positions(pos[f:f + n], o["pos"], position_tolerance(p, dt, mid_p, mid_v))
    finally:
        e.close()
