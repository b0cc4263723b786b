"""Generate the golden vectors in tests/golden/ from the reference's own
compute shaders (engine/shaders/*.metal) compiled as host C++ by
oracle/Makefile into oracle/_ref/libmtlref.so.

Run in a checkout where the reference sources are present:
    make -C oracle ref REF=<reference checkout> && python tests/golden/make_golden.py
The fixtures pin the FP64 oracle and the CUDA path to the reference's
arithmetic.  Inputs follow the reference tests (tests/test_spatial.cpp,
tests/test_pbf.cpp, tests/test_scan.cpp) and the reference engine's default
parameters (engine/src/Engine.cpp:22-39); all generators are seeded.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import params as _abi  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def f4(rows):
    return np.array(rows, np.float32)


def spatial_layouts(cs: float):
    """The reference's hand-placed spatial-hash layouts (test_spatial.cpp)."""
    s = cs * 0.99
    lattice = [[x * s, y * s, z * s, 1] for z in (-1, 0, 1) for y in (-1, 0, 1) for x in (-1, 0, 1)]
    return {
        "hash_points": f4([[0, 0, 0, 1], [2.5, 4.0, -1.5, 1], [-2.9, 5.5, 2.5, 1], [1.0, -2.0, -2.5, 1]]),
        "three_cells": f4([[0, 0, 0, 1], [0.01, 0.02, 0.01, 1], [0.03, 0.01, 0.02, 1],
                           [2, 2, 2, 1], [2.01, 2.02, 2.03, 1], [-2.5, -2.5, -2.5, 1]]),
        "isolated": f4([[0, 0, 0, 1], [1.5, 1.5, 1.5, 1], [-1.5, -1.5, -1.5, 1]]),
        "close_pair": f4([[0, 0, 0, 1], [cs * 0.5, 0, 0, 1]]),
        "lattice_099": f4(lattice),
    }


def main() -> None:
    O.ref_set_threads(1)  # sequential: the reference's atomics then give a stable order
    p = _abi.default_params()
    fx = {}

    # ---- spatial hash layouts (reference box) ----
    for name, pos in spatial_layouts(p.cell_size).items():
        h, cs, si, nc = O.ref_build_spatial_hash(p, pos)
        nz = np.nonzero(np.diff(cs))[0]
        fx[f"spatial/{name}/pos"] = pos
        fx[f"spatial/{name}/hashes"] = h
        fx[f"spatial/{name}/cell_start_total"] = np.uint32(cs[-1])
        fx[f"spatial/{name}/occupied_cells"] = nz.astype(np.uint32)
        fx[f"spatial/{name}/occupied_start"] = cs[nz]
        fx[f"spatial/{name}/sorted_index"] = si
        fx[f"spatial/{name}/neighbor_counts"] = nc

    # ---- PBF cases (test_pbf.cpp) ----
    iso = f4([[0, 1, 0, 1]])
    r = O.ref_step(p, 0.01, iso, np.zeros_like(iso))
    fx["pbf/isolated/pos"] = r["pos"]
    fx["pbf/isolated/vel"] = r["vel"]
    s = p.h * 0.4
    lam = f4([[x * s, y * s, z * s, 1] for z in (-1, 0, 1) for y in (-1, 0, 1) for x in (-1, 0, 1)]
             + [[2, 2, 2, 1]])
    r = O.ref_step(p, 1e-6, lam, np.zeros_like(lam))
    fx["pbf/lambda/pos_in"] = lam
    fx["pbf/lambda/lambda"] = r["lambda"]

    # ---- step trajectories: cube drop, dam break and sphere drop in the
    # reference box with the reference's parameters (K = 5). ----
    def trajectory(tag, scene, n, steps, keep, sphere=None, params=p, dt=1.0 / 240.0):
        pos = O.seed_scene(params, scene, n)
        vel = np.zeros_like(pos)
        sph = None if sphere is None else np.array(sphere, np.float64)
        for st in range(steps + 1):
            if st in keep:
                sin = None if sph is None else sph.copy()
                sref = None if sph is None else sph.astype(np.float32).copy()
                o = O.ref_step(params, dt, pos, vel, sref)
                k = f"traj/{tag}/{st}"
                fx[k + "/pos_in"] = pos.copy()
                fx[k + "/vel_in"] = vel.copy()
                if sin is not None:
                    fx[k + "/sphere_in"] = sin.astype(np.float32)
                    fx[k + "/sphere_out"] = sref.astype(np.float32)
                for key in ("pos", "vel", "lambda", "neighbor_counts", "foam", "hashes",
                            "sorted_index"):
                    fx[k + "/" + key] = o[key]
                fx[k + "/dt"] = np.float32(dt)
            sref = None if sph is None else sph.astype(np.float32)
            o = O.ref_step(params, dt, pos, vel, sref)
            pos, vel = o["pos"], o["vel"]
            if sph is not None:
                sph = sref.astype(np.float64)
    trajectory("cube1000", _abi.MP_SCENE_CUBE_DROP, 1000, 40, {0, 40})
    trajectory("dam2000", _abi.MP_SCENE_DAM_BREAK, 2000, 30, {30})
    # sphere resting in the lake corner: exercises the push-out
    trajectory("sphere_contact", _abi.MP_SCENE_SPHERE_DROP, 2000, 10, {0, 10},
               sphere=[-2.0, -2.5, -2.5, 0.0, 0.0, 0.0, 0.6])

    # ---- legacy integrator: 100 free-fall steps (test_integrator.cpp:47-77) ----
    pos = f4([[0, 5, 0, 1]])
    vel = np.zeros_like(pos)
    import ctypes as C
    ga = (C.c_float * 3)(0.0, -9.81, 0.0)
    lo = (C.c_float * 3)(-3, -3, -3)
    hi = (C.c_float * 3)(3, 6, 3)
    for _ in range(100):
        O.ref().ref_integrate(pos, vel, ga, C.c_float(0.01), lo, hi, C.c_float(0.999), 1)
    fx["integrate/freefall/pos"] = pos.copy()
    fx["integrate/freefall/vel"] = vel.copy()
    pos = f4([[0, -2.95, 0, 1]])
    vel = f4([[0, -10.0, 0, 0]])
    O.ref().ref_integrate(pos, vel, ga, C.c_float(0.05), lo, hi, C.c_float(0.999), 1)
    fx["integrate/bounce/pos"] = pos.copy()
    fx["integrate/bounce/vel"] = vel.copy()

    # ---- legacy integrator and mouse pulse on many particles (the reference's
    # shaders, one dispatch each), inputs inside, on and outside the box ----
    rng = np.random.default_rng(0x6D7470687973 + 17)
    n = 1024
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform([-3.5, -3.5, -3.5], [3.5, 6.5, 3.5], size=(n, 3))
    pos[:, 3] = 1.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 4.0, size=(n, 3))
    fx["integrate/many/pos_in"] = pos.copy()
    fx["integrate/many/vel_in"] = vel.copy()
    for _ in range(3):
        O.ref().ref_integrate(pos, vel, ga, C.c_float(1.0 / 60.0), lo, hi, C.c_float(0.999), n)
    fx["integrate/many/pos"] = pos.copy()
    fx["integrate/many/vel"] = vel.copy()
    origin = (C.c_float * 3)(0.5, 2.0, -6.0)
    d = np.array([0.1, -0.05, 1.0], np.float64)
    d /= np.linalg.norm(d)
    direction = (C.c_float * 3)(*[float(x) for x in d])
    force = (C.c_float * 3)(1.5, 3.0, -0.5)
    ppos = np.zeros((n, 4), np.float32)
    ppos[:, :3] = rng.uniform([-3, -3, -9], [3, 6, 3], size=(n, 3))
    ppos[:, 3] = 1.0
    pvel = np.zeros((n, 4), np.float32)
    pvel[:, :3] = rng.normal(0.0, 1.0, size=(n, 3))
    fx["mouse/pos"] = ppos.copy()
    fx["mouse/vel_in"] = pvel.copy()
    fx["mouse/ray"] = np.array([list(origin), list(direction), list(force)], np.float32)
    fx["mouse/radius"] = np.float32(1.2)
    O.ref().ref_k_mouse_pulse(pvel, ppos, origin, direction, force, C.c_float(1.2), n, n)
    fx["mouse/vel"] = pvel.copy()

    path = os.path.join(OUT, "reference_shaders.npz")
    np.savez_compressed(path, **fx)
    print(f"wrote {path}: {len(fx)} arrays, {os.path.getsize(path)} bytes")


if __name__ == "__main__":
    main()
