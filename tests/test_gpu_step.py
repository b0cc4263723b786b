"""Engine::step on the GPU (engine/src/Engine.cpp:685-811) through the C ABI,
against the reference's known answers (tests/test_pbf.cpp), the golden
vectors of its shaders, and the FP64 oracle per step from the same FP32
state: positions within 1e-5 h, integer outputs bit-exact."""
import numpy as np
import pytest

from mtlphys_b200 import Engine, _abi, configs
from oracle import oracle as O
from parity import (POS_TOL, assert_equal_u32, assert_lambdas, assert_position_distribution,
                    assert_positions, assert_velocities, golden, neighbourhood_max,
                    position_tolerance, random_scene, sensitivity, sensitivity_field)

pytestmark = pytest.mark.gpu
G = golden()


@pytest.fixture(scope="module")
def eng(cuda):
    e = Engine(0)
    yield e
    e.close()


def load_state(e, pos, vel, params=None, scene=_abi.MP_SCENE_CUBE_DROP):
    if params is not None:
        e.set_params(params)
    e.reset(len(pos), scene)
    e.set_positions(pos)
    e.set_velocities(vel)


def gpu_step(e, dt):
    e.step(dt)
    assert e.check_errors() == 0
    return {"pos": e.positions(), "vel": e.velocities(), "lambda": e.lambdas(),
            "neighbor_counts": e.neighbor_counts(), "foam": e.foam(), "hashes": e.cell_hashes(),
            "sorted_index": e.sorted_index(), "cell_start": e.cell_start()}


def compare_with_distribution(p, dt, pos, vel, got, dist, oracle_params=None):
    """The workloads' per-step check (k = 0.1: free surfaces and the 0.3h
    clamp make the step chaotic in places).  Integers bit-exact; positions:
    a ceiling of 4x the largest 1-ulp sensitivity, every particle within 10x
    (99.9% within 1x) the sensitivity of its neighbourhood of cells, at least
    dist[0] of the particles within 1e-5 h and the 99th percentile within
    dist[1] (floors measured on these workloads); lambda and foam where the
    step is well conditioned (kappa_i <= 1e-5 h).  oracle_params: the
    oracle runs with these instead (a test plants a wrong constant there)."""
    q = p if oracle_params is None else oracle_params
    o, kappa = sensitivity_field(q, dt, pos, vel)
    assert_equal_u32(got["hashes"], o["hashes"], "hashes")
    assert_equal_u32(got["cell_start"], o["cell_start"], "cellStart")
    assert_equal_u32(got["sorted_index"], o["sorted_index"], "sortedIndex")
    assert_equal_u32(got["neighbor_counts"], o["neighbor_counts"], "neighbor counts")
    err = np.abs(got["pos"][:, :3] - o["pos"]).max(axis=1)
    ceiling = max(POS_TOL, 4.0 * float(kappa.max()))
    assert err.max() <= ceiling, f"max |dpos| {err.max():.3e} > {ceiling:.3e}"
    g = O.grid(q)
    near = neighbourhood_max(kappa, o["hashes"], list(g.dims))
    stats = assert_position_distribution(err, near, dist[0], dist[1])
    assert_velocities(got["vel"], o["vel"], dt, ceiling)
    well = kappa <= POS_TOL
    if well.any():
        assert_lambdas(got["lambda"][well], o["lambda"][well])
        assert np.abs(got["foam"][well] - o["foam"][well]).max() < 1e-3
    stats["well"] = float(well.mean())
    print("  " + " ".join(f"{k}={v:.3e}" for k, v in stats.items()))
    return stats


def compare_with_oracle(p, dt, pos, vel, got, sphere=None, check_lambda=True):
    tol = position_tolerance(p, dt, pos, vel, sphere)
    o = O.step(p, dt, pos, vel, None if sphere is None else np.array(sphere, np.float64))
    d = np.abs(got["pos"][:, :3] - o["pos"]).max(axis=1)
    print(f"  n={len(pos)} max|dpos|={d.max():.3e} p99.9={np.percentile(d, 99.9):.3e} "
          f"p50={np.median(d):.3e} tol={tol:.3e}")
    assert_equal_u32(got["hashes"], o["hashes"], "hashes")
    assert_equal_u32(got["cell_start"], o["cell_start"], "cellStart")
    assert_equal_u32(got["sorted_index"], o["sorted_index"], "sortedIndex")
    assert_equal_u32(got["neighbor_counts"], o["neighbor_counts"], "neighbor counts")
    err = assert_positions(got["pos"], o["pos"], tol)
    assert_velocities(got["vel"], o["vel"], dt, tol)
    if check_lambda and tol == POS_TOL:
        assert_lambdas(got["lambda"], o["lambda"])
        assert np.abs(got["foam"] - o["foam"]).max() < 1e-3
    assert (got["pos"][:, 3] == 1.0).all() and (got["vel"][:, 3] == 0.0).all()
    return err


# ---- tests/test_pbf.cpp ------------------------------------------------------------

def test_isolated_particle_falls(eng):
    load_state(eng, np.array([[0, 1, 0, 1]], np.float32), np.zeros((1, 4), np.float32),
               _abi.default_params())
    g = gpu_step(eng, 0.01)
    assert g["pos"][0, 1] == pytest.approx(0.99902, rel=1e-3)
    assert g["vel"][0, 1] < 0
    assert_positions(g["pos"], G["pbf/isolated/pos"])


def test_lambda_sign_and_isolated_value(eng):
    p = _abi.default_params()
    pos = G["pbf/lambda/pos_in"]
    load_state(eng, pos, np.zeros_like(pos), p)
    g = gpu_step(eng, 1e-6)
    lam = g["lambda"]
    assert lam[13] < 0
    h = np.float64(np.float32(0.1))
    w0 = 315.0 / (64.0 * np.pi * h ** 9) * h ** 6
    assert lam[-1] == pytest.approx(-(w0 / p.rest_density - 1.0) / p.epsilon, rel=1e-5)
    assert_lambdas(lam, G["pbf/lambda/lambda"])


def test_fifty_steps_stay_finite_and_in_box(eng):
    eng.set_params(_abi.default_params())
    eng.reset(1024, _abi.MP_SCENE_CUBE_DROP)
    for _ in range(50):
        eng.step(1.0 / 240.0)
    assert eng.check_errors() == 0
    pos = eng.positions()
    assert np.isfinite(pos).all()
    assert (pos[:, 0] >= -3.01).all() and (pos[:, 0] <= 3.01).all()
    assert (pos[:, 1] >= -3.01).all() and (pos[:, 1] <= 6.01).all()


TRAJ = sorted({k.rsplit("/", 2)[0] + "/" + k.rsplit("/", 2)[1] for k in G if k.startswith("traj/")})


@pytest.mark.parametrize("key", TRAJ)
def test_step_matches_reference_shaders(eng, key):
    k = key + "/"
    p = _abi.default_params()
    dt = float(G[k + "dt"])
    sphere = G.get(k + "sphere_in")
    scene = _abi.MP_SCENE_SPHERE_DROP if sphere is not None else _abi.MP_SCENE_CUBE_DROP
    load_state(eng, G[k + "pos_in"], G[k + "vel_in"], p, scene)
    if sphere is not None:
        eng.set_sphere(sphere[:3], sphere[3:6], sphere[6])
    g = gpu_step(eng, dt)
    tol = position_tolerance(p, dt, G[k + "pos_in"], G[k + "vel_in"], sphere)
    assert_equal_u32(g["hashes"], G[k + "hashes"], "hashes")
    assert_equal_u32(g["sorted_index"], G[k + "sorted_index"], "sortedIndex")
    assert_equal_u32(g["neighbor_counts"], G[k + "neighbor_counts"], "neighbor counts")
    # two FP32 implementations, each within the bound of the FP64 oracle
    assert_positions(g["pos"], G[k + "pos"], 2 * tol)
    if sphere is not None:
        s = eng.sphere()
        assert np.abs(s[:6] - G[k + "sphere_out"][:6]).max() < 1e-5
    compare_with_oracle(p, dt, G[k + "pos_in"], G[k + "vel_in"], g, sphere)


# ---- the benchmark workloads, per step against the FP64 oracle ------------------------

def run_and_check(e, w, check_at, steps, seed_check=True, dist=None, oracle_params=None):
    """Steps the workload and checks the steps in check_at against the oracle
    (dist: step -> (within-1e-5h floor, p99 bound) for the distribution
    checks of the k = 0.1 workloads)."""
    e.set_params(w.params)
    e.reset(w.n, w.scene, w.desc)
    pos = e.positions()
    if seed_check:
        want = O.seed_scene(w.params, w.scene, w.n, w.desc)
        assert np.array_equal(pos, want), "seeded lattice differs from the oracle's"
    errs = []
    for st in range(steps):
        if st in check_at:
            pos, vel = e.positions(), e.velocities()
            sphere = e.sphere() if w.scene == _abi.MP_SCENE_SPHERE_DROP else None
            g = gpu_step(e, w.dt)
            if dist is not None:
                errs.append(compare_with_distribution(w.params, w.dt, pos, vel, g, dist[st], oracle_params))
            else:
                errs.append(compare_with_oracle(w.params, w.dt, pos, vel, g, sphere))
        else:
            e.step(w.dt)
    assert e.check_errors() == 0
    return errs


# Distribution floors of the k = 0.1 workloads, per checked step: (fraction of
# particles within 1e-5 h, bound on the 99th percentile of |dpos|).  Measured
# on a B200: cube drop 0.987 / 1.1e-6 (step 0), 0.998 / 4.1e-7 (25), 0.999 /
# 4.3e-7 (79); dam break 0.488 / 1.3e-5 (step 0, the compressed column),
# 0.864 / 5.1e-6 (12).  A rest density off by 1e-4 gives 0.010-0.62 / 5e-5-9e-5
# (cube) and 0.000-0.009 / 5e-4-6e-4 (dam break).
CUBE_DIST = {0: (0.97, 3e-6), 25: (0.97, 3e-6), 79: (0.97, 3e-6)}
DAM_DIST = {0: (0.40, 4e-5), 12: (0.75, 2e-5)}


def test_cube_drop_97k_per_step_parity(eng):
    errs = run_and_check(eng, configs.cube_drop(), set(CUBE_DIST), 80, dist=CUBE_DIST)
    print("cube_drop:", errs)


def test_dam_break_1m_per_step_parity(eng):
    errs = run_and_check(eng, configs.dam_break(), set(DAM_DIST), 13, dist=DAM_DIST)
    print("dam_break:", errs)


@pytest.mark.parametrize("workload,dist,steps", [("cube_drop", {25: (0.97, 3e-6)}, 26),
                                                 ("dam_break", {12: (0.75, 2e-5)}, 13)])
def test_workload_checks_reject_a_wrong_rest_density(eng, workload, dist, steps):
    """A mistake planted in the oracle, on the CPU: its rest density 1e-4
    too large (a wrong constant, ~1e-4 m on most particles).  The workloads'
    per-step checks at k = 0.1 must reject the (correct) GPU step against it;
    a bound on the largest error alone (4x the largest 1-ulp sensitivity)
    would accept it."""
    w = configs.WORKLOADS[workload]()
    wrong = w.params.copy()
    wrong.rest_density = w.params.rest_density * (1.0 + 1e-4)
    with pytest.raises(AssertionError):
        run_and_check(eng, w, set(dist), steps, dist=dist, oracle_params=wrong)


def test_random_cloud_checks_reject_the_self_density_fault(eng):
    """The mistake the self-density fix removed (the density starts at W(0)
    only when the particle's own slot lies in its current stencil), planted
    in the oracle on the CPU: on the random cloud whose clumps explode (149
    particles move by up to 2.3 mm under it), the per-step check rejects the
    (correct) GPU step.  At the k = 0.1 workloads this fault moves 22-175 of
    1M dam-break particles by ~5 mm inside regions where a one-ulp change of
    the input alone moves the oracle by as much, so no per-step check there
    can single it out."""
    p = _abi.default_params()
    pos, vel = random_scene(3, 3000)
    load_state(eng, pos, vel, p)
    g = gpu_step(eng, 1.0 / 240.0)
    compare_with_oracle(p, 1.0 / 240.0, pos, vel, g)  # the real oracle: accepted
    with O.planted_fault(1):
        with pytest.raises(AssertionError):
            compare_with_oracle(p, 1.0 / 240.0, pos, vel, g)


def test_reference_sphere_drop_scene(eng):
    eng.set_params(_abi.default_params())
    eng.reset(30_000, _abi.MP_SCENE_SPHERE_DROP)
    s = eng.sphere()
    assert s[1] == pytest.approx(4.5) and s[6] == pytest.approx(0.6)
    for st in range(3):
        pos, vel, sph = eng.positions(), eng.velocities(), eng.sphere()
        g = gpu_step(eng, 1.0 / 120.0)
        compare_with_oracle(_abi.default_params(), 1.0 / 120.0, pos, vel, g, sph)


def test_zero_iterations(eng):
    p = _abi.default_params()
    p.solver_iterations = 0
    eng.set_params(p)
    eng.reset(5000, _abi.MP_SCENE_DAM_BREAK)
    pos, vel = eng.positions(), eng.velocities()
    g = gpu_step(eng, 1.0 / 240.0)
    compare_with_oracle(p, 1.0 / 240.0, pos, vel, g, check_lambda=False)


def test_graph_mode_is_bit_identical(eng):
    w = configs.cube_drop(side=30)
    outs = []
    for graph in (False, True):
        eng.set_params(w.params)
        eng.reset(w.n, w.scene, w.desc)
        eng.set_graph_mode(graph)
        for _ in range(20):
            eng.step(w.dt)
        assert eng.check_errors() == 0
        outs.append((eng.positions(), eng.velocities(), eng.foam()))
        eng.set_graph_mode(False)
    for a, b in zip(*outs):
        assert np.array_equal(a, b)


def test_steps_are_deterministic(eng):
    w = configs.cube_drop(side=24)
    outs = []
    for _ in range(2):
        eng.set_params(w.params)
        eng.reset(w.n, w.scene, w.desc)
        for _ in range(15):
            eng.step(w.dt)
        outs.append(eng.positions())
    assert np.array_equal(outs[0], outs[1])


def test_host_round_trip_every_step_is_bit_identical(eng):
    """The state held on the host (positions and velocities uploaded before
    and downloaded after every step, as a caller keeping its own buffers
    does) gives the device-resident trajectory bit for bit."""
    w = configs.cube_drop(side=24)
    eng.set_params(w.params)
    eng.reset(w.n, w.scene, w.desc)
    eng.set_graph_mode(True)
    for _ in range(3):
        eng.step(w.dt)
    pos, vel = eng.positions(), eng.velocities()
    for _ in range(12):
        eng.step(w.dt)
    resident = (eng.positions(), eng.velocities())
    for _ in range(12):
        eng.set_positions(pos)
        eng.set_velocities(vel)
        eng.step(w.dt)
        pos, vel = eng.positions(), eng.velocities()
    eng.set_graph_mode(False)
    assert eng.check_errors() == 0
    assert np.array_equal(pos, resident[0])
    assert np.array_equal(vel, resident[1])


def test_dt_le_zero_is_a_noop(eng):
    eng.set_params(_abi.default_params())
    eng.reset(1000)
    before = eng.positions()
    eng.step(0.0)
    eng.step(-1.0)
    assert np.array_equal(before, eng.positions())


def test_nan_input_sets_the_device_error_word(eng):
    eng.set_params(_abi.default_params())
    eng.reset(1000)
    pos = eng.positions()
    pos[17, 0] = np.nan
    eng.set_positions(pos)
    eng.step(1.0 / 240.0)
    bits = eng.error_bits()
    assert bits & _abi.MP_DEVERR_NAN
    assert eng.error_bits() == 0  # cleared


@pytest.mark.parametrize("spacing,epsilon", [(0.35, 800.0), (0.22, 1e5)])
def test_crowded_stencil_rows(eng, spacing, epsilon):
    """A lattice packed at `spacing` h puts ~70 (0.35h) or ~250 (0.22h)
    candidates in every stencil row: the lambda pass takes each row in
    chunks of 32, and the delta pass walks the first chunk's recorded bits
    and distance-tests the rest of the row.  Per step against the oracle
    (epsilon raised for the denser lattice, where the default one makes the
    step ill-conditioned and only the adaptive bound would apply)."""
    p = _abi.default_params()
    p.epsilon = epsilon
    rng = np.random.default_rng(11)
    side = int(round(3.0 / spacing))  # a cube of ~3h on a side
    g = np.stack(np.meshgrid(*(np.arange(side),) * 3, indexing="ij"), -1).reshape(-1, 3)
    pos = np.zeros((len(g), 4), np.float32)
    pos[:, :3] = g * spacing * p.h + np.array([0.1, 1.0, 0.2]) + rng.uniform(-1e-2, 1e-2, g.shape) * p.h
    pos[:, 3] = 1.0
    vel = np.zeros_like(pos)
    load_state(eng, pos, vel, p)
    for _ in range(2):
        pos, vel = eng.positions(), eng.velocities()
        g = gpu_step(eng, 1.0 / 240.0)
        compare_with_oracle(p, 1.0 / 240.0, pos, vel, g)


@pytest.mark.parametrize("seed,n", [(1, 600), (2, 2000), (3, 3000), (4, 50_000)])
def test_random_clouds(eng, seed, n):
    """Seeded random clouds (uniform, tight clumps of hundreds of particles
    per cell, points outside the grid; random velocities), two steps, each
    from the GPU's own state, against the oracle.  The clumps explode, so
    some particles drift two cells from their hash cells within a step and
    leave their own slot out of their stencil: their density must still
    start from their own W(0), as the reference's does."""
    p = _abi.default_params()
    pos, vel = random_scene(seed, n)
    load_state(eng, pos, vel, p)
    for _ in range(2):
        pos, vel = eng.positions(), eng.velocities()
        g = gpu_step(eng, 1.0 / 240.0)
        compare_with_oracle(p, 1.0 / 240.0, pos, vel, g)


@pytest.mark.parametrize("seed", [5, 6])
def test_random_clouds_with_sphere(eng, seed):
    """A seeded random cloud with the kinematic sphere inside it (moving):
    every iteration pushes the particles it overlaps out to its surface.  Two
    steps against the oracle, sphere state included."""
    p = _abi.default_params()
    pos, vel = random_scene(seed, 2000)
    load_state(eng, pos, vel, p, _abi.MP_SCENE_SPHERE_DROP)
    rng = np.random.default_rng(seed)
    eng.set_sphere((0.05, 1.0, -0.05), tuple(rng.normal(0.0, 1.0, 3)), 0.25)
    for _ in range(2):
        pos, vel, sph = eng.positions(), eng.velocities(), eng.sphere()
        g = gpu_step(eng, 1.0 / 240.0)
        compare_with_oracle(p, 1.0 / 240.0, pos, vel, g, sph)
        s_gpu = eng.sphere()
        s_or = np.array(sph, np.float64)
        O.step(p, 1.0 / 240.0, pos, vel, s_or)
        assert np.abs(s_gpu[:6] - s_or[:6]).max() < 1e-5


def test_empty_engine_steps(eng):
    eng.set_params(_abi.default_params())
    eng.reset(0)
    eng.step(1.0 / 240.0)
    eng.build_spatial_hash()
    assert eng.check_errors() == 0
    assert eng.particle_count() == 0


def with_reference_k(w):
    """The same workload with the reference engine's s_corr k = 1e-4
    (Constraints.metal:158), where the step is well conditioned."""
    w.params = w.params.copy()
    w.params.scorr_k = 1e-4
    return w


def test_cube_drop_97k_reference_k_strict_parity(eng):
    errs = run_and_check(eng, with_reference_k(configs.cube_drop()), {0, 40, 99}, 100)
    assert max(errs) <= POS_TOL
    print("cube_drop (k=1e-4) max |dpos|:", errs)


def test_dam_break_1m_reference_k_strict_parity(eng):
    errs = run_and_check(eng, with_reference_k(configs.dam_break()), {0, 20}, 21)
    assert max(errs) <= POS_TOL
    print("dam_break (k=1e-4) max |dpos|:", errs)


@pytest.mark.parametrize("workload", ["dam_break", "cube_drop"])
def test_full_length_runs_stay_valid(eng, workload):
    """The configs' full runs (dam break 300 steps at 1M particles, cube drop
    200 steps) under graph replay: no device error word, every position and
    velocity finite, inside the box, speeds under the CFL cap, and at the end
    the hash invariants of the reference's spatial tests hold."""
    w = configs.WORKLOADS[workload]()
    eng.set_params(w.params)
    eng.reset(w.n, w.scene, w.desc)
    eng.set_graph_mode(True)
    for t in range(w.steps):
        eng.step(w.dt)
        if t % 50 == 49:
            assert eng.check_errors() == 0, t
    eng.set_graph_mode(False)
    pos, vel = eng.positions(), eng.velocities()
    assert np.isfinite(pos).all() and np.isfinite(vel).all()
    lo, hi = np.array(w.params.bounds_min[:]), np.array(w.params.bounds_max[:])
    assert (pos[:, :3] >= lo).all() and (pos[:, :3] <= hi).all()
    vmax = w.params.vmax * w.params.h / w.dt
    assert (np.linalg.norm(vel[:, :3], axis=1) <= vmax * (1 + 1e-5)).all()
    eng.build_spatial_hash()
    cs, si, hs = eng.cell_start(), eng.sorted_index(), eng.cell_hashes()
    assert cs[0] == 0 and cs[-1] == w.n and (np.diff(cs.astype(np.int64)) >= 0).all()
    assert np.array_equal(np.sort(si), np.arange(w.n, dtype=si.dtype))
    # slots of a cell hold exactly that cell's particles, in increasing index
    cell_of_slot = np.repeat(np.arange(len(cs) - 1), np.diff(cs.astype(np.int64)))
    assert np.array_equal(hs[si], cell_of_slot)
    same = cell_of_slot[1:] == cell_of_slot[:-1]
    assert (si[1:][same] > si[:-1][same]).all()


@pytest.mark.parametrize("graph", [True, False])
def test_profiling_times_every_kernel_and_keeps_the_bits(eng, graph):
    """Per-kernel timing, kernel by kernel or captured with the step's graph
    (event nodes), times each launch of the step and gives the same state as
    an untimed step."""
    w = configs.cube_drop(side=24)
    k = int(w.params.solver_iterations)
    outs = []
    for profile in (False, True):
        eng.set_params(w.params)
        eng.reset(w.n, w.scene, w.desc)
        eng.set_graph_mode(graph)
        eng.set_profiling(profile)
        for _ in range(4):
            eng.step(w.dt)
        if profile:
            times = eng.kernel_times()
            launches = sum(v[0] for v in times.values())
            assert launches == 4 * int(_abi.load().mp_step_launch_count(k)), times
            assert all(v[1] > 0.0 for v in times.values()), times
            assert times["lambda_count"][0] == 4 and times["delta_finalize"][0] == 4
            eng.set_profiling(False)
        assert eng.check_errors() == 0
        outs.append((eng.positions(), eng.velocities()))
        eng.set_graph_mode(False)
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
