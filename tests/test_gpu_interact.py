"""The interactive and legacy Engine passes on the GPU: Engine::integrate
(Integrate.metal) and Engine::applyMousePulse (Constraints.metal:231-253),
against the reference's own shaders (golden vectors) and the FP32 oracle."""
import numpy as np
import pytest

from mtlphys_b200 import Engine, _abi
from oracle import oracle as O
from parity import golden

pytestmark = pytest.mark.gpu


def engine_with(pos, vel, params=None):
    e = Engine(0)
    if params is not None:
        e.set_params(params)
    e.reset(len(pos))
    e.write(_abi.MP_BUF_POSITIONS, pos)
    e.write(_abi.MP_BUF_VELOCITIES, vel)
    return e


def test_integrate_equals_the_reference_shader(cuda):
    g = golden()
    e = engine_with(g["integrate/many/pos_in"], g["integrate/many/vel_in"])
    for _ in range(3):
        e.integrate(1.0 / 60.0)
    np.testing.assert_array_equal(e.positions(), g["integrate/many/pos"])
    np.testing.assert_array_equal(e.velocities(), g["integrate/many/vel"])
    e.close()


def test_integrator_reference_cases(cuda):
    """test_integrator.cpp: 100 free-fall steps at dt = 0.01 from (0, 5, 0);
    a particle at y = -2.95 moving down at 10 m/s is clamped to the floor and
    bounces upwards."""
    g = golden()
    e = engine_with(np.array([[0, 5, 0, 1]], np.float32), np.zeros((1, 4), np.float32))
    for _ in range(100):
        e.integrate(0.01)
    np.testing.assert_array_equal(e.positions(), g["integrate/freefall/pos"])
    np.testing.assert_array_equal(e.velocities(), g["integrate/freefall/vel"])
    e.write(_abi.MP_BUF_POSITIONS, np.array([[0, -2.95, 0, 1]], np.float32))
    e.write(_abi.MP_BUF_VELOCITIES, np.array([[0, -10.0, 0, 0]], np.float32))
    e.integrate(0.05)
    p, v = e.positions(), e.velocities()
    assert p[0, 1] == -3.0 and v[0, 1] > 0.0
    np.testing.assert_array_equal(v, g["integrate/bounce/vel"])
    before = e.positions()
    e.integrate(0.0)  # dt <= 0: no-op
    np.testing.assert_array_equal(e.positions(), before)
    e.close()


def test_mouse_pulse_matches_the_reference_shader_and_the_oracle(cuda):
    g = golden()
    r = g["mouse/ray"]
    radius = float(g["mouse/radius"])
    e = engine_with(g["mouse/pos"], g["mouse/vel_in"])
    e.apply_mouse_pulse(r[0], r[1], r[2], radius)
    v = e.velocities()
    np.testing.assert_allclose(v, g["mouse/vel"], rtol=1e-6, atol=1e-6)
    want = O.mouse_pulse_f32(_abi.default_params(), r[0], r[1], r[2], radius, g["mouse/pos"],
                             g["mouse/vel_in"])
    np.testing.assert_allclose(v, want, rtol=1e-6, atol=1e-6)
    # particles outside the cylinder or behind the origin keep their velocity bit for bit
    moved = np.abs(want - g["mouse/vel_in"]).max(1) > 0
    np.testing.assert_array_equal(v[~moved], g["mouse/vel_in"][~moved])
    assert moved.sum() > 10
    # positions are untouched
    np.testing.assert_array_equal(e.positions(), g["mouse/pos"])
    e.close()


def test_mouse_pulse_at_scale_and_after_a_step(cuda):
    """A pulse into the 1M-particle dam break between two steps: the velocity
    change equals the oracle's pulse of the same state."""
    from mtlphys_b200 import configs

    w = configs.dam_break()
    e = Engine(0)
    e.set_params(w.params)
    e.reset(w.n, w.scene, w.desc)
    e.step(w.dt)
    pos, vel = e.positions(), e.velocities()
    origin, direction, force = (1.6, 4.0, -1.0), (0.0, -0.6, 0.8), (0.0, 5.0, 2.0)
    d = np.array(direction, np.float32) / np.float32(np.linalg.norm(direction))
    e.apply_mouse_pulse(origin, d, force, 0.8)
    got = e.velocities()
    want = O.mouse_pulse_f32(w.params, origin, d, force, 0.8, pos, vel)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6)
    assert (np.abs(want - vel).max(1) > 0).sum() > 1000
    e.step(w.dt)
    e.check_errors()
    e.close()


@pytest.mark.parametrize("seed", [1, 2])
def test_integrate_and_pulse_on_random_clouds(cuda, seed):
    """Seeded random clouds (points outside the box included, so the
    integrator's wall clamps and reflections fire on every face): integrate
    is bit-exact against the FP32 oracle over several calls, and a pulse
    through the cloud matches it within 1e-6."""
    from parity import random_scene

    p = _abi.default_params()
    pos, vel = random_scene(seed, 20_000)
    vel[:, :3] *= 20.0  # fast enough to cross walls within a call
    e = engine_with(pos, vel, p)
    want_p, want_v = pos, vel
    for dt in (1.0 / 60.0, 1.0 / 30.0, 1.0 / 120.0):
        e.integrate(dt)
        want_p, want_v = O.integrate_f32(p, dt, want_p, want_v)
        np.testing.assert_array_equal(e.positions(), want_p)
        np.testing.assert_array_equal(e.velocities(), want_v)
    rng = np.random.default_rng(seed)
    d = rng.normal(size=3).astype(np.float32)
    d /= np.float32(np.linalg.norm(d))
    origin = (0.0, 1.0, 0.0) - 2.0 * d
    cur_p, cur_v = e.positions(), e.velocities()
    e.apply_mouse_pulse(tuple(origin), tuple(d), (1.0, 3.0, -2.0), 0.6)
    want = O.mouse_pulse_f32(p, tuple(origin), tuple(d), (1.0, 3.0, -2.0), 0.6, cur_p, cur_v)
    np.testing.assert_allclose(e.velocities(), want, rtol=1e-6, atol=1e-6)
    assert (np.abs(want - cur_v).max(1) > 0).sum() > 100
    e.close()
