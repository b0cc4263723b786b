"""Tolerances and comparison helpers shared by the parity tests.

Positions: within 1e-5 * h of the FP64 oracle per step, from the same FP32
input state (the acceptance bound of the step).  Velocities are
(p - p_prev) / dt * damping, so their bound is the position bound / dt.
Integer outputs (cell hashes, cell starts, sorted order, neighbour counts)
are compared bit for bit.
"""
from __future__ import annotations

import os

import numpy as np

H = 0.1
POS_TOL = 1e-5 * H
LAMBDA_ATOL = 2e-7
LAMBDA_RTOL = 1e-4
FOAM_ATOL = 1e-3

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_shaders.npz")


def golden() -> dict:
    z = np.load(GOLDEN)
    return {k: z[k] for k in z.files}


def max_abs(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max()) if a.size else 0.0


def assert_positions(got, want, tol: float = POS_TOL, what: str = "positions") -> float:
    err = max_abs(np.asarray(got)[:, :3], np.asarray(want)[:, :3])
    assert err <= tol, f"{what}: max |diff| {err:.3e} > {tol:.3e}"
    return err


def assert_velocities(got, want, dt: float, tol: float = POS_TOL, what: str = "velocities") -> float:
    bound = tol / dt
    err = max_abs(np.asarray(got)[:, :3], np.asarray(want)[:, :3])
    assert err <= bound, f"{what}: max |diff| {err:.3e} > {bound:.3e}"
    return err


def assert_lambdas(got, want) -> None:
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    bound = LAMBDA_ATOL + LAMBDA_RTOL * np.abs(want)
    bad = np.abs(got - want) > bound
    assert not bad.any(), f"lambda: {bad.sum()} outside tolerance, worst {np.abs(got - want).max():.3e}"


def assert_equal_u32(got, want, what: str) -> None:
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, f"{what}: shape {got.shape} != {want.shape}"
    if not np.array_equal(got, want):
        i = int(np.nonzero(got != want)[0][0])
        raise AssertionError(f"{what}: first mismatch at {i}: got {got[i]} want {want[i]}")


def sensitivity(p, dt: float, pos4, vel4, sphere=None, seed: int = 0) -> float:
    """How far the FP64 oracle's step moves when every input coordinate is
    nudged by one FP32 ulp: the conditioning of the step at this state.  A
    deep first contact with the sphere amplifies it by ~10^4 in the
    reference algorithm itself (FP32 and FP64 alike)."""
    from oracle import oracle as O

    pos4 = np.asarray(pos4, np.float32)
    rng = np.random.default_rng(seed)
    pert = pos4.copy()
    sgn = np.where(rng.random(pert[:, :3].shape) < 0.5, -np.inf, np.inf).astype(np.float32)
    pert[:, :3] = np.nextafter(pert[:, :3], sgn)
    s0 = None if sphere is None else np.array(sphere, np.float64)
    s1 = None if sphere is None else np.array(sphere, np.float64)
    a = O.step(p, dt, pos4, vel4, s0)["pos"]
    b = O.step(p, dt, pert, vel4, s1)["pos"]
    return max_abs(a, b)


def sensitivity_field(p, dt: float, pos4, vel4, sphere=None, seeds=(0, 1, 2)):
    """Per-particle conditioning of the FP64 oracle's step at this state: for
    each seed, every input coordinate is nudged by one FP32 ulp in a random
    direction and each particle's result is compared with the unperturbed
    step; kappa_i is the largest move over the seeds.  Returns (the
    unperturbed oracle output, kappa)."""
    from oracle import oracle as O

    pos4 = np.asarray(pos4, np.float32)
    s = None if sphere is None else np.array(sphere, np.float64)
    base = O.step(p, dt, pos4, vel4, s)
    kappa = np.zeros(len(pos4))
    for seed in seeds:
        rng = np.random.default_rng(seed)
        pert = pos4.copy()
        sgn = np.where(rng.random(pert[:, :3].shape) < 0.5, -np.inf, np.inf).astype(np.float32)
        pert[:, :3] = np.nextafter(pert[:, :3], sgn)
        s1 = None if sphere is None else np.array(sphere, np.float64)
        moved = np.abs(O.step(p, dt, pert, vel4, s1)["pos"] - base["pos"]).max(axis=1)
        kappa = np.maximum(kappa, moved)
    return base, kappa


def neighbourhood_max(values, hashes, dims, reach: int = 2):
    """For every particle, the largest value over the particles whose hash
    cells lie within `reach` cells of its own (a (2 reach + 1)^3 block of the
    grid): a particle's FP32 rounding reaches its neighbours' results, so its
    own 1-ulp move can understate how far it may go."""
    from scipy.ndimage import maximum_filter

    dims = [int(d) for d in dims]
    g = np.zeros(dims[0] * dims[1] * dims[2])
    hashes = np.asarray(hashes, np.int64)
    np.maximum.at(g, hashes, values)
    g = maximum_filter(g.reshape(dims[2], dims[1], dims[0]), size=2 * reach + 1, mode="nearest")
    return g.ravel()[hashes]


def assert_position_distribution(err, kappa_near, frac_floor=None, p99_bound=None,
                                 ratio_cap: float = 10.0, beyond_frac: float = 1e-3) -> dict:
    """Checks of an ill-conditioned step, particle by particle and over the
    distribution (err: per-particle max |GPU - oracle|, kappa_near: the
    neighbourhood sensitivity):
      - every particle within ratio_cap x max(1e-5 h, kappa_near_i), and at
        most a fraction beyond_frac beyond 1 x;
      - at least frac_floor of the particles within 1e-5 h and the 99th
        percentile of the error at most p99_bound (when given: measured
        floors of a workload, which a wrong constant or formula breaks)."""
    r = err / np.maximum(kappa_near, POS_TOL)
    stats = {"within_tol": float((err <= POS_TOL).mean()), "p50": float(np.median(err)),
             "p99": float(np.quantile(err, 0.99)), "max": float(err.max()), "ratio_max": float(r.max()),
             "beyond_kappa": float((r > 1.0).mean())}
    assert stats["ratio_max"] <= ratio_cap, f"a particle is {stats['ratio_max']:.1f}x its neighbourhood sensitivity"
    assert stats["beyond_kappa"] <= beyond_frac, f"{stats['beyond_kappa']:.2e} of particles beyond their sensitivity"
    if frac_floor is not None:
        assert stats["within_tol"] >= frac_floor, f"only {stats['within_tol']:.4f} within 1e-5 h (floor {frac_floor})"
    if p99_bound is not None:
        assert stats["p99"] <= p99_bound, f"p99 {stats['p99']:.2e} > {p99_bound:.2e}"
    return stats


def position_tolerance(p, dt: float, pos4, vel4, sphere=None) -> float:
    """1e-5 h where the step is well conditioned (a 1-ulp input change moves
    it by less than that); otherwise 4x the measured sensitivity."""
    kappa = sensitivity(p, dt, pos4, vel4, sphere)
    return POS_TOL if kappa <= POS_TOL else 4.0 * kappa


def random_scene(seed: int, n: int):
    """A seeded random cloud in the reference's default box ([-3, 3] x [-3, 6]
    x [-3, 3]): 60% uniform in a 1 m cube, 30% in three tight clumps (cells of
    dozens to hundreds of particles: long stencil rows and long cell
    segments), 10% anywhere in a slightly larger box (positions outside the
    grid, clamped by the hash); velocities N(0, 0.5 m/s).  Returns float32
    (n, 4) positions (w = 1) and velocities (w = 0)."""
    rng = np.random.default_rng(seed)
    n_u, n_c = int(0.6 * n), int(0.3 * n)
    n_o = n - n_u - n_c
    u = rng.uniform(-0.5, 0.5, (n_u, 3)) + np.array([0.0, 1.0, 0.0])
    centres = rng.uniform(-0.4, 0.4, (3, 3)) + np.array([0.0, 1.0, 0.0])
    cl = centres[rng.integers(0, 3, n_c)] + rng.normal(0.0, 0.03, (n_c, 3))
    o = rng.uniform([-3.2, -3.2, -3.2], [3.2, 6.2, 3.2], (n_o, 3))
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.concatenate([u, cl, o])
    pos[:, 3] = 1.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 0.5, (n, 3))
    return pos, vel
