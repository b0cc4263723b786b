"""The CPU oracle against the reference: golden vectors produced by the
reference's own compute shaders (tests/golden/make_golden.py) and the
reference tests' known answers (tests/test_scan.cpp, test_spatial.cpp,
test_pbf.cpp).  Runs without a GPU."""
import math

import numpy as np
import pytest

from mtlphys_b200 import _abi, configs
from oracle import oracle as O
from parity import (H, POS_TOL, assert_equal_u32, assert_lambdas, assert_positions,
                    assert_velocities, golden, position_tolerance, random_scene)

G = golden()


def ref_params():
    return _abi.default_params()


# ---- scan (tests/test_scan.cpp) -----------------------------------------------------

def np_exclusive(x):
    x = np.asarray(x, np.uint32)
    return (np.cumsum(x, dtype=np.uint64) - x).astype(np.uint32)


@pytest.mark.parametrize("n,seed,maxval", [(1024, 0xA, 7), (700, 0xB, 7), (2048, 0xC, 7),
                                           (635626, 0xD, 3)])
def test_oracle_scan_random(n, seed, maxval):
    x = np.random.RandomState(seed).randint(0, maxval + 1, size=n).astype(np.uint32)
    assert_equal_u32(O.exclusive_scan(x), np_exclusive(x), "scan")


def test_oracle_scan_zeros_and_ones():
    assert not O.exclusive_scan(np.zeros(100, np.uint32)).any()
    assert_equal_u32(O.exclusive_scan(np.ones(500, np.uint32)), np.arange(500, dtype=np.uint32), "ones")


def test_oracle_scan_wraps_mod_2_32():
    x = np.full(5, 0xFFFFFFFF, np.uint32)
    assert_equal_u32(O.exclusive_scan(x), np_exclusive(x), "wrap")


# ---- spatial hash (tests/test_spatial.cpp) ------------------------------------------

LAYOUTS = ["hash_points", "three_cells", "isolated", "close_pair", "lattice_099"]


@pytest.mark.parametrize("name", LAYOUTS)
def test_oracle_spatial_matches_reference_shaders(name):
    k = f"spatial/{name}/"
    h, cs, si, nc = O.build_spatial_hash(ref_params(), G[k + "pos"])
    assert_equal_u32(h, G[k + "hashes"], "hashes")
    occ = np.nonzero(np.diff(cs))[0]
    assert_equal_u32(occ, G[k + "occupied_cells"], "occupied cells")
    assert_equal_u32(cs[occ], G[k + "occupied_start"], "cell starts")
    assert cs[-1] == G[k + "cell_start_total"] == len(h)
    assert_equal_u32(si, G[k + "sorted_index"], "sortedIndex")
    assert_equal_u32(nc, G[k + "neighbor_counts"], "neighbor counts")


def test_oracle_spatial_known_answers():
    p = ref_params()
    assert (O.build_spatial_hash(p, G["spatial/isolated/pos"])[3] == 0).all()
    assert list(O.build_spatial_hash(p, G["spatial/close_pair/pos"])[3]) == [1, 1]
    nc = O.build_spatial_hash(p, G["spatial/lattice_099/pos"])[3]
    assert nc[13] == 6 and nc[0] < nc[13] and nc[26] < nc[13]


def test_oracle_hash_formula_and_clamping():
    p = ref_params()
    g = O.grid(p)
    assert list(g.dims) == [60, 90, 60] and g.cells == 324000
    pos = np.array([[0, 0, 0, 1], [-100, -100, -100, 1], [100, 100, 100, 1],
                    [np.nan, 0, 0, 1], [-3.0, -3.0, -3.0, 1]], np.float32)
    h = O.hash_f32(p, pos)
    assert h[1] == 0 and h[4] == 0 and h[3] == 0 + 30 * 60 + 30 * 60 * 90
    assert h[2] == 59 + 89 * 60 + 59 * 60 * 90
    cfg_grid = O.grid(configs.base_params(3))
    assert list(cfg_grid.dims) == [86, 86, 86] and cfg_grid.cells == 636056


# ---- PBF (tests/test_pbf.cpp) ---------------------------------------------------------

def test_oracle_isolated_particle_falls():
    p = ref_params()
    pos = np.array([[0, 1, 0, 1]], np.float32)
    o = O.step(p, 0.01, pos, np.zeros_like(pos))
    assert o["pos"][0, 1] == pytest.approx(0.99902, rel=1e-3)
    assert o["vel"][0, 1] < 0
    assert_positions(o["pos"], G["pbf/isolated/pos"])
    assert_velocities(o["vel"], G["pbf/isolated/vel"], 0.01)


def test_oracle_lambda_sign_and_isolated_value():
    p = ref_params()
    pos = G["pbf/lambda/pos_in"]
    o = O.step(p, 1e-6, pos, np.zeros_like(pos))
    lam = o["lambda"]
    assert lam[13] < 0
    # isolated: -(W(0)/rho0 - 1)/epsilon with the engine's epsilon (800)
    h = np.float64(np.float32(0.1))
    w0 = 315.0 / (64.0 * math.pi * h ** 9) * h ** 6
    assert lam[-1] == pytest.approx(-(w0 / p.rest_density - 1.0) / p.epsilon, rel=1e-6)
    assert_lambdas(lam, G["pbf/lambda/lambda"])


TRAJ = sorted({k.rsplit("/", 2)[0] + "/" + k.rsplit("/", 2)[1] for k in G if k.startswith("traj/")})


@pytest.mark.parametrize("key", TRAJ)
def test_oracle_step_matches_reference_shaders(key):
    p = ref_params()
    k = key + "/"
    dt = float(G[k + "dt"])
    sphere = None
    if k + "sphere_in" in G:
        sphere = G[k + "sphere_in"].astype(np.float64)
    tol = position_tolerance(p, dt, G[k + "pos_in"], G[k + "vel_in"], sphere)
    o = O.step(p, dt, G[k + "pos_in"], G[k + "vel_in"], None if sphere is None else sphere.copy())
    assert_equal_u32(o["hashes"], G[k + "hashes"], "hashes")
    assert_equal_u32(o["sorted_index"], G[k + "sorted_index"], "sortedIndex")
    assert_equal_u32(o["neighbor_counts"], G[k + "neighbor_counts"], "neighbor counts")
    assert_positions(o["pos"], G[k + "pos"], tol)
    assert_velocities(o["vel"], G[k + "vel"], dt, tol)
    if tol == POS_TOL:
        assert_lambdas(o["lambda"], G[k + "lambda"])
        assert np.abs(o["foam"] - G[k + "foam"]).max() < 1e-3
    if sphere is not None:
        O.step(p, dt, G[k + "pos_in"], G[k + "vel_in"], sphere)
    if sphere is not None:
        assert np.abs(sphere[:6] - G[k + "sphere_out"][:6]).max() < 1e-5


def test_oracle_dt_zero_is_a_noop():
    p = ref_params()
    pos = O.seed_scene(p, 0, 10)
    o = O.step(p, 0.0, pos, np.zeros_like(pos))
    # no outputs written for dt <= 0 (Engine.cpp:686): arrays are uninitialised,
    # the call simply returns 0
    assert o is not None


# ---- seeding (Engine.cpp:454-549) -------------------------------------------------

def test_oracle_seeding_reference_scenes():
    p = ref_params()
    cube = O.seed_scene(p, _abi.MP_SCENE_CUBE_DROP, 1000)   # side 10, top at y = 2
    assert cube[:, 1].max() == pytest.approx(2.0) and cube[:, 1].min() == pytest.approx(2.0 - 9 * 0.05)
    assert cube[:, 0].mean() == pytest.approx(0.0, abs=1e-6)
    dam = O.seed_scene(p, _abi.MP_SCENE_DAM_BREAK, 11000)   # 110 layers, 100 per layer
    assert dam[:, 0].min() == pytest.approx(-2.95) and dam[:, 1].min() == pytest.approx(-2.95)
    assert len(np.unique(dam[:, 1])) == 110
    lake = O.seed_scene(p, _abi.MP_SCENE_SPHERE_DROP, 5000)
    assert lake[:, 1].min() == pytest.approx(-2.95)


def test_oracle_config_lattices():
    w = configs.dam_break()
    pos = O.seed_scene(w.params, w.scene, w.n, w.desc)
    assert len(pos) == 1003520
    assert pos[:, 0].min() == pytest.approx(0.05, abs=0.0011)
    assert pos[:, 1].max() == pytest.approx(8.0, abs=0.0011)
    assert (pos[:, :3] >= 0).all() and (pos[:, :3] <= configs.BOX).all()
    w = configs.cube_drop()
    pos = O.seed_scene(w.params, w.scene, w.n, w.desc)
    assert pos[:, 0].min() == pytest.approx(2.0, abs=0.0011)


@pytest.mark.skipif(not O.has_ref(), reason="reference sources not built here (oracle/_ref)")
def test_oracle_matches_reference_shaders_live_config_box():
    """FP64 oracle vs the reference's shader code on a cube in the 86h box
    (the reference hard-codes s_corr k = 1e-4, so the check uses that)."""
    w = configs.cube_drop(side=12, iterations=3)
    p = w.params.copy()
    p.scorr_k = 1e-4
    pos = O.seed_scene(p, w.scene, w.n, w.desc)
    vel = np.zeros_like(pos)
    O.ref_set_threads(1)
    for _ in range(20):
        r = O.ref_step(p, w.dt, pos, vel)
        o = O.step(p, w.dt, pos, vel)
        assert_equal_u32(o["sorted_index"], r["sorted_index"], "sortedIndex")
        assert_positions(o["pos"], r["pos"])
        pos, vel = r["pos"], r["vel"]


@pytest.mark.skipif(not O.has_ref(), reason="reference sources not built here (oracle/_ref)")
@pytest.mark.parametrize("seed,n", [(1, 600), (2, 2000), (3, 3000)])
def test_oracle_matches_reference_shaders_random_clouds(seed, n):
    """FP64 oracle vs the reference's shader code on seeded random clouds
    (uniform, tight clumps, points outside the grid; random velocities), two
    steps from each state: hash, cellStart, sortedIndex and neighbour counts
    bit-exact, positions within the step's bound (1e-5 h, or 4x the measured
    1-ulp sensitivity where the clumps make the step ill-conditioned)."""
    p = ref_params()
    dt = 1.0 / 240.0
    pos, vel = random_scene(seed, n)
    O.ref_set_threads(1)
    for _ in range(2):
        r = O.ref_step(p, dt, pos, vel)
        o = O.step(p, dt, pos, vel)
        for key in ("hashes", "cell_start", "sorted_index", "neighbor_counts"):
            assert_equal_u32(o[key], r[key], key)
        assert_positions(o["pos"], r["pos"], position_tolerance(p, dt, pos, vel))
        pos, vel = r["pos"], r["vel"]


@pytest.mark.skipif(not O.has_ref(), reason="reference sources not built here (oracle/_ref)")
@pytest.mark.parametrize("seed", [5, 6])
def test_oracle_matches_reference_shaders_random_cloud_with_sphere(seed):
    """The same random clouds with the moving sphere inside them: the
    oracle's sphere kinematics and per-iteration push against the reference's
    (host kinematics restated by the harness, sphereCollision compiled from
    its shader), two steps."""
    p = ref_params()
    dt = 1.0 / 240.0
    pos, vel = random_scene(seed, 2000)
    rng = np.random.default_rng(seed)
    sph_r = np.array([0.05, 1.0, -0.05, *rng.normal(0.0, 1.0, 3), 0.25], np.float32)
    sph_o = sph_r.astype(np.float64)
    O.ref_set_threads(1)
    for _ in range(2):
        tol = position_tolerance(p, dt, pos, vel, sph_o.copy())
        o = O.step(p, dt, pos, vel, sph_o)
        r = O.ref_step(p, dt, pos, vel, sph_r)
        for key in ("hashes", "cell_start", "sorted_index", "neighbor_counts"):
            assert_equal_u32(o[key], r[key], key)
        assert_positions(o["pos"], r["pos"], tol)
        assert np.abs(sph_o[:6] - sph_r[:6]).max() < 1e-5
        pos, vel = r["pos"], r["vel"]


def test_integrate_matches_the_reference_shader():
    """Engine::integrate restated in FP32 equals the reference's Integrate.metal
    (compiled as C++) bit for bit, including box clamps and reflections."""
    g = golden()
    p = _abi.default_params()
    pos, vel = g["integrate/many/pos_in"], g["integrate/many/vel_in"]
    for _ in range(3):
        pos, vel = O.integrate_f32(p, 1.0 / 60.0, pos, vel)
    np.testing.assert_array_equal(pos, g["integrate/many/pos"])
    np.testing.assert_array_equal(vel, g["integrate/many/vel"])
    # test_integrator.cpp: 100 free-fall steps, and the floor bounce
    pos, vel = np.array([[0, 5, 0, 1]], np.float32), np.zeros((1, 4), np.float32)
    for _ in range(100):
        pos, vel = O.integrate_f32(p, 0.01, pos, vel)
    np.testing.assert_array_equal(pos, g["integrate/freefall/pos"])
    np.testing.assert_array_equal(vel, g["integrate/freefall/vel"])
    pos, vel = O.integrate_f32(p, 0.05, np.array([[0, -2.95, 0, 1]], np.float32),
                               np.array([[0, -10.0, 0, 0]], np.float32))
    assert pos[0, 1] == -3.0 and vel[0, 1] > 0.0
    np.testing.assert_array_equal(vel, g["integrate/bounce/vel"])


def test_mouse_pulse_matches_the_reference_shader():
    """applyMousePulse restated in FP32; the reference's shader, compiled as
    C++, evaluates its exponent in double, hence the 1e-6 relative bound."""
    g = golden()
    p = _abi.default_params()
    r = g["mouse/ray"]
    v = O.mouse_pulse_f32(p, r[0], r[1], r[2], float(g["mouse/radius"]), g["mouse/pos"], g["mouse/vel_in"])
    np.testing.assert_allclose(v, g["mouse/vel"], rtol=1e-6, atol=1e-6)
    moved = np.abs(g["mouse/vel"] - g["mouse/vel_in"]).max(1) > 0
    assert 10 < moved.sum() < len(moved)  # the case exercises both branches


def test_planted_self_density_fault_changes_the_oracle():
    """The mistake the GPU parity tests plant in the oracle (or_plant_fault 1:
    the density starts at W(0) only when the particle's own slot lies in the
    stencil of its current cell) really changes the step where particles
    drift two cells within it (the exploding clumps of a random cloud), and
    the context manager takes it out again."""
    p = ref_params()
    pos, vel = random_scene(3, 3000)
    good = O.step(p, 1.0 / 240.0, pos, vel)["pos"]
    with O.planted_fault(1):
        bad = O.step(p, 1.0 / 240.0, pos, vel)["pos"]
    again = O.step(p, 1.0 / 240.0, pos, vel)["pos"]
    moved = np.abs(bad - good).max(axis=1)
    assert (moved > 1e-4).sum() >= 10, (moved > 1e-4).sum()
    assert np.array_equal(good, again)
