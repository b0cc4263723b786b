"""Parameter structs, reference defaults and the benchmark workloads, for the
oracle side only.

TEST INFRASTRUCTURE ONLY.  The oracle (liboracle.so) and the reference's
shaders compiled as C++ (oracle/_ref) take the parameter block laid out as
`mp_pbf_params` / `mp_scene_desc` in include/mtlphys_b200.h.  This module
declares those layouts itself, with the reference engine's default values
written out, so that the checker and the benchmark's reference arm never
import or load the product package (mtlphys_b200).  A CPU test checks that
the layouts, the defaults and the workloads below equal the product's byte
for byte.

Defaults: engine/src/Engine.cpp:22-39, 551-572 (tunables, writePBFParams),
engine/shaders/Constraints.metal:158-160, 190, 250, 297, 325, 341-347
(shader literals), engine/include/mtlphys/Engine.hpp:184 (sphere radius),
engine/shaders/Integrate.metal:29.
"""
from __future__ import annotations

import ctypes as C
import math

MP_SCENE_CUBE_DROP = 0
MP_SCENE_DAM_BREAK = 1
MP_SCENE_SPHERE_DROP = 2

H = 0.1
BOX = 86 * H  # the workloads' box, 8.6 m on a side
SEED_BASE = 0x6D7470687973


class PBFParams(C.Structure):
    """mp_pbf_params (include/mtlphys_b200.h)."""

    _fields_ = [
        ("size", C.c_uint32), ("solver_iterations", C.c_uint32), ("h", C.c_float),
        ("cell_size", C.c_float), ("rest_density", C.c_float), ("epsilon", C.c_float),
        ("damping", C.c_float), ("gravity", C.c_float * 3), ("bounds_min", C.c_float * 3),
        ("bounds_max", C.c_float * 3), ("scorr_k", C.c_float), ("scorr_n", C.c_uint32),
        ("scorr_dq", C.c_float), ("max_delta", C.c_float), ("vmax", C.c_float),
        ("wall_eps", C.c_float), ("floor_friction", C.c_float), ("wall_friction", C.c_float),
        ("foam_max_neighbors", C.c_float), ("foam_speed_lo", C.c_float), ("foam_speed_hi", C.c_float),
        ("sphere_radius", C.c_float), ("sphere_gravity", C.c_float), ("sphere_drag", C.c_float),
        ("sphere_restitution", C.c_float), ("integrate_damping", C.c_float),
        ("integrate_restitution", C.c_float), ("mouse_falloff", C.c_float),
    ]

    def copy(self) -> "PBFParams":
        return PBFParams.from_buffer_copy(self)

    def set(self, **kw) -> "PBFParams":
        for k, v in kw.items():
            cur = getattr(self, k)
            if isinstance(cur, C.Array):
                for i, x in enumerate(v):
                    cur[i] = x
            else:
                setattr(self, k, v)
        return self


class SceneDesc(C.Structure):
    """mp_scene_desc (include/mtlphys_b200.h)."""

    _fields_ = [
        ("size", C.c_uint32), ("lattice", C.c_uint32), ("seed", C.c_uint64),
        ("dims", C.c_uint32 * 3), ("origin", C.c_float * 3), ("spacing", C.c_float),
        ("jitter", C.c_float), ("sphere_center", C.c_float * 3), ("sphere_velocity", C.c_float * 3),
    ]


def as_params(p) -> PBFParams:
    """The same bytes as a PBFParams of this module (accepts the product's
    ctypes mirror too: both are the layout of mp_pbf_params)."""
    if isinstance(p, PBFParams):
        return p
    if C.sizeof(p) != C.sizeof(PBFParams):
        raise TypeError(f"{type(p).__name__} is not an mp_pbf_params")
    return PBFParams.from_buffer_copy(p)


def as_desc(d) -> SceneDesc | None:
    if d is None or isinstance(d, SceneDesc):
        return d
    if C.sizeof(d) != C.sizeof(SceneDesc):
        raise TypeError(f"{type(d).__name__} is not an mp_scene_desc")
    return SceneDesc.from_buffer_copy(d)


def default_params() -> PBFParams:
    """The reference engine's values (the product's mp_default_params)."""
    p = PBFParams()
    p.size = C.sizeof(PBFParams)
    p.set(solver_iterations=5,          # Engine.cpp:39
          h=0.10, cell_size=0.10,       # Engine.cpp:29, 25
          rest_density=8000.0,          # Engine.cpp:32
          epsilon=800.0,                # Engine.cpp:35
          damping=0.996,                # Engine.cpp:36
          gravity=(0.0, -9.81, 0.0),    # Engine.cpp:558
          bounds_min=(-3.0, -3.0, -3.0), bounds_max=(3.0, 6.0, 3.0),  # Engine.cpp:23-24
          scorr_k=1e-4, scorr_n=4, scorr_dq=0.2,  # Constraints.metal:158-160, 179
          max_delta=0.3,                # Constraints.metal:190
          vmax=1.0,                     # Constraints.metal:347
          wall_eps=1e-3,                # Constraints.metal:325
          floor_friction=0.55, wall_friction=0.97,  # Constraints.metal:341-344
          foam_max_neighbors=96.0,      # Engine.cpp:27, 806
          foam_speed_lo=1.2, foam_speed_hi=4.5,  # Constraints.metal:297
          sphere_radius=0.6,            # Engine.hpp:184
          sphere_gravity=-9.81, sphere_drag=0.998, sphere_restitution=0.4,  # Engine.cpp:694-707
          integrate_damping=0.999,      # Engine.cpp:584
          integrate_restitution=0.4,    # Integrate.metal:29
          mouse_falloff=0.4)            # Constraints.metal:250
    return p


def default_scene_desc() -> SceneDesc:
    d = SceneDesc()
    d.size = C.sizeof(SceneDesc)
    d.sphere_center[1] = 4.5  # Engine.cpp:523-525
    return d


def lattice_rest_density(h: float = H, spacing: float = 0.5 * H) -> float:
    """Poly6 density of an interior site of a cubic lattice (the particle's
    own W(0) included): sum over lattice offsets with r^2 < h^2 of
    315 / (64 pi h^9) (h^2 - r^2)^3, in FP64, offsets in z, y, x order."""
    norm = 315.0 / (64.0 * math.pi * math.pow(h, 9))
    r = int(math.ceil(h / spacing)) + 1
    rho = 0.0
    for z in range(-r, r + 1):
        for y in range(-r, r + 1):
            for x in range(-r, r + 1):
                r2 = spacing * spacing * float(x * x + y * y + z * z)
                if r2 < h * h:
                    d = h * h - r2
                    rho += norm * d * d * d
    return rho


def base_params(iterations: int) -> PBFParams:
    """The workloads' shared physics: h = 0.1, rho0 of the 0.5h lattice,
    g = (0, -9.8, 0), CFM epsilon 100, s_corr k = 0.1, n = 4, dq = 0.2h, the
    86h box."""
    p = default_params()
    return p.set(h=H, cell_size=H, rest_density=lattice_rest_density(), epsilon=100.0,
                 gravity=(0.0, -9.8, 0.0), bounds_min=(0.0, 0.0, 0.0), bounds_max=(BOX, BOX, BOX),
                 scorr_k=0.1, scorr_n=4, scorr_dq=0.2, solver_iterations=iterations)


def lattice(dims, origin, seed: int, spacing: float = 0.5 * H, jitter: float = 0.01 * H) -> SceneDesc:
    d = default_scene_desc()
    d.lattice = 1
    d.seed = seed
    for a in range(3):
        d.dims[a] = int(dims[a])
        d.origin[a] = float(origin[a])
    d.spacing = spacing
    d.jitter = jitter
    return d


class Workload:
    def __init__(self, name, params, scene, desc, n, dt, steps):
        self.name, self.params, self.scene, self.desc = name, params, scene, desc
        self.n, self.dt, self.steps = n, dt, steps

    def describe(self) -> dict:
        g = [math.ceil(BOX / H)] * 3
        return {"workload": self.name, "particles": self.n, "solver_iterations":
                int(self.params.solver_iterations), "dt": self.dt, "grid": g,
                "cells": g[0] * g[1] * g[2], "steps": self.steps}


def cube_drop(side: int = 46, iterations: int = 3, steps: int = 200) -> Workload:
    """97,336 particles (46^3 lattice at 0.5h, lower corner (20h, 30h, 20h))."""
    d = lattice((side, side, side), (20 * H, 30 * H, 20 * H), SEED_BASE + 0)
    return Workload("cube_drop", base_params(iterations), MP_SCENE_CUBE_DROP, d, side ** 3,
                    1.0 / 120.0, steps)


def dam_break(iterations: int = 5, steps: int = 300) -> Workload:
    """1,003,520 particles: a 64 x 160 x 98 lattice 0.5h off the x = 0 wall
    and the floor, centred in z."""
    nx, ny, nz = 64, 160, 98
    z0 = 0.5 * (BOX - (nz - 1) * 0.5 * H)
    d = lattice((nx, ny, nz), (0.5 * H, 0.5 * H, z0), SEED_BASE + 1)
    return Workload("dam_break", base_params(iterations), MP_SCENE_DAM_BREAK, d, nx * ny * nz,
                    1.0 / 120.0, steps)


WORKLOADS = {"cube_drop": cube_drop, "dam_break": dam_break}
