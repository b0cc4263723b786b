"""The benchmark workloads, with their sizes, as parameter sets and scenes.

  cube_drop    97,336 particles (46^3 lattice, spacing 0.5h, lower corner
               (20h, 30h, 20h)) in an 86h cube box, K = 3, 200 steps
  dam_break    1,003,520 particles (64 x 160 x 98 lattice against the x = 0
               wall, 0.5h off the wall and floor, centred in z) in the same
               box, K = 5, 300 steps
  diff_cube    cube_drop scaled to 20^3 (finite differences) or 46^3
               (timing), 60-step rollout
  batch_cubes  256 cube drops, counts log-uniform in [2,000, 64,000]
  batch_sphere 32 sphere drops, counts log-uniform in [20,000, 200,000]

Shared physics: h = 0.1, mass 1, rho0 = Poly6 density of an interior
lattice site (8078.2013), g = (0, -9.8, 0), dt = 1/120 s, CFM epsilon 100,
s_corr k = 0.1, n = 4, dq = 0.2h; damping and the wall / friction / clamp /
foam constants are the reference engine's (engine/src/Engine.cpp:22-39,
engine/shaders/Constraints.metal).  Every lattice is jittered by a seeded
uniform +-0.01h per component; the seed is 0x6D7470687973 + workload index.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi
from ._abi import PBFParams, SceneDesc

H = 0.1
SEED_BASE = 0x6D7470687973
BOX = 86 * H  # 8.6 m


def rest_density(h: float = H, spacing: float = 0.5 * H) -> float:
    return float(_abi.load().mp_lattice_rest_density(h, spacing))


def base_params(iterations: int) -> PBFParams:
    p = _abi.default_params()
    p.set(h=H, cell_size=H, rest_density=rest_density(), epsilon=100.0, gravity=(0.0, -9.8, 0.0),
          bounds_min=(0.0, 0.0, 0.0), bounds_max=(BOX, BOX, BOX), scorr_k=0.1, scorr_n=4,
          scorr_dq=0.2, solver_iterations=iterations)
    return p


def lattice(dims, origin, seed: int, spacing: float = 0.5 * H, jitter: float = 0.01 * H) -> SceneDesc:
    d = _abi.default_scene_desc()
    d.lattice = 1
    d.seed = seed
    for a in range(3):
        d.dims[a] = int(dims[a])
        d.origin[a] = float(origin[a])
    d.spacing = spacing
    d.jitter = jitter
    return d


class Workload:
    def __init__(self, name: str, params: PBFParams, scene: int, desc: SceneDesc, n: int,
                 dt: float, steps: int):
        self.name, self.params, self.scene, self.desc = name, params, scene, desc
        self.n, self.dt, self.steps = n, dt, steps

    def describe(self) -> dict:
        g = [math.ceil(BOX / H)] * 3
        return {"workload": self.name, "particles": self.n, "solver_iterations":
                int(self.params.solver_iterations), "dt": self.dt, "grid": g,
                "cells": g[0] * g[1] * g[2], "steps": self.steps}


def cube_drop(side: int = 46, iterations: int = 3, steps: int = 200) -> Workload:
    p = base_params(iterations)
    d = lattice((side, side, side), (20 * H, 30 * H, 20 * H), SEED_BASE + 0)
    return Workload("cube_drop", p, _abi.MP_SCENE_CUBE_DROP, d, side ** 3, 1.0 / 120.0, steps)


def dam_break(iterations: int = 5, steps: int = 300) -> Workload:
    p = base_params(iterations)
    nx, ny, nz = 64, 160, 98
    z0 = 0.5 * (BOX - (nz - 1) * 0.5 * H)
    d = lattice((nx, ny, nz), (0.5 * H, 0.5 * H, z0), SEED_BASE + 1)
    return Workload("dam_break", p, _abi.MP_SCENE_DAM_BREAK, d, nx * ny * nz, 1.0 / 120.0, steps)


def diff_cube(side: int = 20, steps: int = 60) -> Workload:
    w = cube_drop(side=side, iterations=3, steps=steps)
    w.name = "diff_cube"
    w.desc.seed = SEED_BASE + 2
    return w


def batch_counts(num: int, lo: int, hi: int, seed: int) -> np.ndarray:
    rng = np.random.Generator(np.random.MT19937(seed))
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=num)).astype(np.int64)


WORKLOADS = {"cube_drop": cube_drop, "dam_break": dam_break, "diff_cube": diff_cube}


class BatchWorkload:
    """Scenes of a batch: per-scene counts, parameters, dts, scene ids, descs."""

    def __init__(self, name, counts, params, dts, scenes, descs, steps, spheres=None):
        self.name, self.counts, self.params, self.dts = name, counts, params, dts
        self.scenes, self.descs, self.steps, self.spheres = scenes, descs, steps, spheres

    @property
    def n(self) -> int:
        return int(sum(self.counts))

    def describe(self) -> dict:
        return {"workload": self.name, "scenes": len(self.counts), "particles": self.n,
                "min_scene": int(min(self.counts)), "max_scene": int(max(self.counts)),
                "solver_iterations": int(self.params[0].solver_iterations), "steps": self.steps}


def batch_cubes(num: int = 256, lo: int = 2000, hi: int = 64000, steps: int = 100) -> BatchWorkload:
    """Independent cube drops: counts log-uniform in [lo, hi], cube side
    ceil(cbrt(n)) (Engine.cpp:531) at the cube-drop corner (20h, 30h, 20h) of
    the 86h box, jitter +-0.01h, per-scene dt ~ U[1/240, 1/120] and
    epsilon ~ U[50, 200], other parameters as the cube drop."""
    rng = np.random.Generator(np.random.MT19937(SEED_BASE + 3))
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), size=num)).astype(np.int64)
    dts = rng.uniform(1.0 / 240.0, 1.0 / 120.0, size=num)
    eps = rng.uniform(50.0, 200.0, size=num)
    params, descs = [], []
    for s in range(num):
        p = base_params(3)
        p.epsilon = float(eps[s])
        params.append(p)
        side = int(math.ceil(round(counts[s] ** (1.0 / 3.0), 9)))
        while side ** 3 < counts[s]:
            side += 1
        descs.append(lattice((side, side, side), (20 * H, 30 * H, 20 * H), SEED_BASE + 3 + 1000 * (s + 1)))
    return BatchWorkload("batch_cubes", [int(c) for c in counts], params, [float(d) for d in dts],
                         [_abi.MP_SCENE_CUBE_DROP] * num, descs, steps)


def batch_spheres(num: int = 32, lo: int = 20000, hi: int = 200000, steps: int = 40) -> BatchWorkload:
    """Sphere drops into pre-settled lakes: counts log-uniform in [lo, hi];
    each lake is 20h deep (40 layers at 0.5h) on a square footprint sized to
    its count, in a box whose walls hug the footprint and are 40h high; a
    kinematic sphere of radius 8h (scaled down on footprints narrower than
    2.5 x 16h) starts at height 35h over the centre with vertical speed
    v0 ~ U[0, 3] m/s (downwards).  dt = 1/120, 3 iterations."""
    rng = np.random.Generator(np.random.MT19937(SEED_BASE + 4))
    counts = np.exp(rng.uniform(math.log(lo), math.log(hi), size=num)).astype(np.int64)
    v0 = rng.uniform(0.0, 3.0, size=num)
    params, descs, spheres = [], [], []
    sp = 0.5 * H
    for s in range(num):
        layers = 40
        side = int(math.ceil(math.sqrt(counts[s] / layers)))
        width = (side - 1) * sp + 2 * 0.5 * H
        p = base_params(3)
        p.set(bounds_min=(0.0, 0.0, 0.0), bounds_max=(width, 40 * H, width))
        radius = 8 * H * min(1.0, width / (2.5 * 16 * H))
        p.sphere_radius = radius
        params.append(p)
        d = lattice((side, layers, side), (0.5 * H, 0.5 * H, 0.5 * H), SEED_BASE + 4 + 1000 * (s + 1))
        d.sphere_center[0] = d.sphere_center[2] = 0.5 * width
        d.sphere_center[1] = 35 * H
        d.sphere_velocity[1] = -float(v0[s])
        descs.append(d)
        spheres.append((0.5 * width, 35 * H, 0.5 * width, 0.0, -float(v0[s]), 0.0, radius))
    return BatchWorkload("batch_spheres", [int(c) for c in counts], params, [1.0 / 120.0] * num,
                         [_abi.MP_SCENE_SPHERE_DROP] * num, descs, steps, spheres)
