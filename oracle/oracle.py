"""Python binding of the CPU oracle (oracle/build/liboracle.so) and of the
reference-shader cross-check (oracle/_ref/libmtlref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg, as the checker.  The product library never
loads anything from this folder.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from .params import PBFParams, SceneDesc, as_desc, as_params

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmtlref.so")

_F = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_U = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build(with_ref: bool | None = None) -> None:
    """Compile the oracle (and the _ref cross-check when $MTLPHYS_REFERENCE
    names a reference checkout)."""
    target = ["all"] if with_ref is None else (["oracle", "ref"] if with_ref else ["oracle"])
    ref_root = os.environ.get("MTLPHYS_REFERENCE", "")
    extra = [f"REF={ref_root}"] if ref_root else []
    subprocess.run(["make", "-s", "-C", HERE, *extra, *target], check=True)


class Grid(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("cell", C.c_float), ("inv_cell", C.c_float),
                ("dims", C.c_uint32 * 3), ("cells", C.c_uint32)]


class StepOut(C.Structure):
    _fields_ = [("pos3", C.c_void_p), ("vel3", C.c_void_p), ("lam", C.c_void_p),
                ("foam", C.c_void_p), ("neighbor_counts", C.c_void_p), ("hashes", C.c_void_p),
                ("cell_start", C.c_void_p), ("sorted_index", C.c_void_p), ("pred4", C.c_void_p)]


class RefConfig(C.Structure):
    _fields_ = [("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3), ("cell", C.c_float),
                ("h", C.c_float), ("rest_density", C.c_float), ("epsilon", C.c_float),
                ("damping", C.c_float), ("gravity", C.c_float * 3), ("iterations", C.c_uint32),
                ("max_neighbors", C.c_uint32), ("sphere", C.c_uint32),
                ("sphere_center", C.c_float * 3), ("sphere_velocity", C.c_float * 3),
                ("sphere_radius", C.c_float)]


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        L = C.CDLL(ORACLE_SO)
        L.or_make_grid.argtypes = [C.POINTER(PBFParams), C.POINTER(Grid)]
        L.or_hash_f32.argtypes = [_F, C.c_uint32, C.POINTER(Grid), _U]
        L.or_hash_f32.restype = None
        L.or_exclusive_scan_u32.argtypes = [_U, _U, C.c_uint32]
        L.or_exclusive_scan_u32.restype = None
        L.or_counting_sort.argtypes = [_U, C.c_uint32, C.c_uint32, _U, _U]
        L.or_counting_sort.restype = None
        L.or_count_neighbors_f32.argtypes = [_F, C.c_uint32, C.POINTER(Grid), C.c_float, _U, _U, _U]
        L.or_count_neighbors_f32.restype = None
        L.or_predict_f32.argtypes = [_F, _F, C.c_uint32, C.POINTER(C.c_float), C.c_float, _F]
        L.or_predict_f32.restype = None
        L.or_seed_scene.argtypes = [C.POINTER(PBFParams), C.c_uint32, C.POINTER(SceneDesc),
                                    C.c_uint32, _F]
        L.or_sphere_advance.argtypes = [C.POINTER(PBFParams), C.c_double, _D]
        L.or_sphere_advance.restype = None
        L.or_integrate_f32.argtypes = [C.POINTER(PBFParams), C.c_float, C.c_uint32, _F, _F]
        L.or_integrate_f32.restype = None
        L.or_mouse_pulse_f32.argtypes = [C.POINTER(PBFParams), C.POINTER(C.c_float), C.POINTER(C.c_float),
                                         C.POINTER(C.c_float), C.c_float, C.c_uint32, _F, _F]
        L.or_mouse_pulse_f32.restype = None
        L.or_step.argtypes = [C.POINTER(PBFParams), C.c_float, C.c_uint32, _F, _F, C.c_void_p,
                              C.POINTER(StepOut)]
        L.or_step_f64.argtypes = [C.POINTER(PBFParams), C.c_double, C.c_uint32, _D, _D, C.c_void_p]
        L.or_plant_fault.argtypes = [C.c_int]
        L.or_plant_fault.restype = None
        L.or_set_threads.argtypes = [C.c_int]
        L.or_set_threads.restype = None
        L.or_get_threads.restype = C.c_int
        _lib = L
    return _lib


def has_ref() -> bool:
    return os.path.exists(REF_SO)


def ref() -> C.CDLL:
    """The reference's shaders compiled as C++ (built only where the
    reference sources are present)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = C.CDLL(REF_SO)
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_set_threads.restype = None
        L.ref_threads.restype = C.c_int
        L.ref_grid.argtypes = [C.POINTER(RefConfig), _U]
        L.ref_grid.restype = C.c_uint32
        L.ref_build_spatial_hash.argtypes = [C.POINTER(RefConfig), C.c_uint32, _F, _U, _U, _U, _F, _U]
        L.ref_build_spatial_hash.restype = None
        L.ref_step.argtypes = [C.POINTER(RefConfig), C.c_float, C.c_uint32, _F, _F, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p]
        L.ref_step.restype = None
        L.ref_integrate.argtypes = [_F, _F, C.POINTER(C.c_float), C.c_float, C.POINTER(C.c_float),
                                    C.POINTER(C.c_float), C.c_float, C.c_uint32]
        L.ref_integrate.restype = None
        L.ref_k_mouse_pulse.argtypes = [_F, _F, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                        C.POINTER(C.c_float), C.c_float, C.c_uint32, C.c_uint32]
        L.ref_k_mouse_pulse.restype = None
        _ref = L
    return _ref


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f4(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    assert a.ndim == 2 and a.shape[1] == 4
    return a


# ---- oracle -------------------------------------------------------------------

def grid(p: PBFParams) -> Grid:
    g = Grid()
    rc = lib().or_make_grid(C.byref(as_params(p)), C.byref(g))
    if rc != 0:
        raise ValueError("invalid grid parameters")
    return g


def hash_f32(p: PBFParams, pos4) -> np.ndarray:
    pos4 = _f4(pos4)
    out = np.empty(len(pos4), np.uint32)
    lib().or_hash_f32(pos4, len(pos4), C.byref(grid(p)), out)
    return out


def exclusive_scan(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.uint32)
    out = np.empty_like(x)
    lib().or_exclusive_scan_u32(x, out, len(x))
    return out


def build_spatial_hash(p: PBFParams, pos4):
    """hashes, cell_start, sorted_index, neighbor_counts of pos4 (stable)."""
    pos4 = _f4(pos4)
    g = grid(p)
    n = len(pos4)
    hashes = np.empty(n, np.uint32)
    lib().or_hash_f32(pos4, n, C.byref(g), hashes)
    cs = np.empty(g.cells + 1, np.uint32)
    si = np.empty(n, np.uint32)
    lib().or_counting_sort(hashes, n, g.cells, cs, si)
    nc = np.empty(n, np.uint32)
    h2 = np.float32(p.h) * np.float32(p.h)
    lib().or_count_neighbors_f32(pos4, n, C.byref(g), C.c_float(h2), cs, si, nc)
    return hashes, cs, si, nc


def predict_f32(p: PBFParams, pos4, vel4, dt: float) -> np.ndarray:
    pos4, vel4 = _f4(pos4), _f4(vel4)
    out = np.empty_like(pos4)
    lib().or_predict_f32(pos4, vel4, len(pos4), p.gravity, C.c_float(dt), out)
    return out


def seed_scene(p: PBFParams, scene: int, n: int, desc: SceneDesc | None = None) -> np.ndarray:
    out = np.empty((n, 4), np.float32)
    rc = lib().or_seed_scene(C.byref(as_params(p)), scene, C.byref(as_desc(desc)) if desc is not None else None, n, out)
    if rc != 0:
        raise ValueError(f"or_seed_scene failed ({rc})")
    return out


def step(p: PBFParams, dt: float, pos4, vel4, sphere=None) -> dict:
    """One FP64 oracle step from an FP32 state.  `sphere`: 7 doubles
    (center, velocity, radius) or None; advanced in place."""
    pos4, vel4 = _f4(pos4), _f4(vel4)
    n = len(pos4)
    g = grid(p)
    o = {
        "pos": np.empty((n, 3)), "vel": np.empty((n, 3)), "lambda": np.empty(n),
        "foam": np.empty(n), "neighbor_counts": np.empty(n, np.uint32),
        "hashes": np.empty(n, np.uint32), "cell_start": np.empty(g.cells + 1, np.uint32),
        "sorted_index": np.empty(n, np.uint32), "pred4": np.empty((n, 4), np.float32),
    }
    so = StepOut(_ptr(o["pos"]), _ptr(o["vel"]), _ptr(o["lambda"]), _ptr(o["foam"]),
                 _ptr(o["neighbor_counts"]), _ptr(o["hashes"]), _ptr(o["cell_start"]),
                 _ptr(o["sorted_index"]), _ptr(o["pred4"]))
    sph = None
    if sphere is not None:
        sph = np.ascontiguousarray(sphere, dtype=np.float64)
        assert sph.shape == (7,)
    rc = lib().or_step(C.byref(as_params(p)), C.c_float(dt), n, pos4, vel4, _ptr(sph), C.byref(so))
    if rc != 0:
        raise ValueError(f"or_step failed ({rc})")
    if sphere is not None:
        sphere[:] = sph
    return o


def integrate_f32(p: PBFParams, dt: float, pos4, vel4):
    """Engine::integrate in FP32; returns new (pos4, vel4) arrays."""
    pos4, vel4 = _f4(pos4).copy(), _f4(vel4).copy()
    lib().or_integrate_f32(C.byref(as_params(p)), C.c_float(dt), len(pos4), pos4, vel4)
    return pos4, vel4


def mouse_pulse_f32(p: PBFParams, origin, direction, force, radius: float, pos4, vel4):
    """Engine::applyMousePulse in FP32; returns the new velocities."""
    vel4 = _f4(vel4).copy()
    v3 = lambda a: (C.c_float * 3)(*[float(x) for x in a])
    lib().or_mouse_pulse_f32(C.byref(as_params(p)), v3(origin), v3(direction), v3(force), C.c_float(radius),
                             len(vel4), _f4(pos4), vel4)
    return vel4


def step_f64(p: PBFParams, dt: float, pos3, vel3, sphere=None) -> None:
    """One FP64 oracle step on an FP64 state (n x 3 arrays, in place)."""
    assert pos3.dtype == np.float64 and pos3.flags.c_contiguous
    assert vel3.dtype == np.float64 and vel3.flags.c_contiguous
    sph = None if sphere is None else sphere
    rc = lib().or_step_f64(C.byref(as_params(p)), C.c_double(dt), len(pos3), pos3, vel3, _ptr(sph))
    if rc != 0:
        raise ValueError(f"or_step_f64 failed ({rc})")


class planted_fault:
    """Context manager: the oracle's step runs with deliberate mistake
    `which` (see or_plant_fault), so a test can show a check rejects it."""

    def __init__(self, which: int):
        self.which = which

    def __enter__(self):
        lib().or_plant_fault(self.which)
        return self

    def __exit__(self, *exc):
        lib().or_plant_fault(0)


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def threads() -> int:
    return lib().or_get_threads()


# ---- reference shaders compiled as C++ -------------------------------------------

def ref_config(p: PBFParams, sphere=None) -> RefConfig:
    c = RefConfig()
    for a in range(3):
        c.bounds_min[a] = p.bounds_min[a]
        c.bounds_max[a] = p.bounds_max[a]
        c.gravity[a] = p.gravity[a]
    c.cell = p.cell_size
    c.h = p.h
    c.rest_density = p.rest_density
    c.epsilon = p.epsilon
    c.damping = p.damping
    c.iterations = p.solver_iterations
    c.max_neighbors = int(p.foam_max_neighbors)
    if sphere is not None:
        c.sphere = 1
        for a in range(3):
            c.sphere_center[a] = sphere[a]
            c.sphere_velocity[a] = sphere[3 + a]
        c.sphere_radius = sphere[6]
    return c


def ref_build_spatial_hash(p: PBFParams, pos4):
    pos4 = _f4(pos4)
    c = ref_config(p)
    dims = np.empty(3, np.uint32)
    cells = ref().ref_grid(C.byref(c), dims)
    n = len(pos4)
    hashes = np.empty(n, np.uint32)
    cs = np.empty(cells + 1, np.uint32)
    si = np.empty(n, np.uint32)
    sp = np.empty((n, 4), np.float32)
    nc = np.empty(n, np.uint32)
    ref().ref_build_spatial_hash(C.byref(c), n, pos4, hashes, cs, si, sp, nc)
    return hashes, cs, si, nc


def ref_step(p: PBFParams, dt: float, pos4, vel4, sphere=None) -> dict:
    """One step of the reference's own shader code (FP32).  Returns the new
    state and diagnostics; `sphere` (7 floats) is advanced in place."""
    pos = _f4(pos4).copy()
    vel = _f4(vel4).copy()
    c = ref_config(p, sphere)
    dims = np.empty(3, np.uint32)
    cells = ref().ref_grid(C.byref(c), dims)
    n = len(pos)
    o = {"prev": np.empty((n, 4), np.float32), "lambda": np.empty(n, np.float32),
         "neighbor_counts": np.empty(n, np.uint32), "foam": np.empty(n, np.float32),
         "hashes": np.empty(n, np.uint32), "cell_start": np.empty(cells + 1, np.uint32),
         "sorted_index": np.empty(n, np.uint32)}
    ref().ref_step(C.byref(c), C.c_float(dt), n, pos, vel, _ptr(o["prev"]), _ptr(o["lambda"]),
                   _ptr(o["neighbor_counts"]), _ptr(o["foam"]), _ptr(o["hashes"]),
                   _ptr(o["cell_start"]), _ptr(o["sorted_index"]))
    o["pos"] = pos
    o["vel"] = vel
    if sphere is not None:
        for a in range(3):
            sphere[a] = c.sphere_center[a]
            sphere[3 + a] = c.sphere_velocity[a]
    return o


def ref_set_threads(n: int) -> None:
    ref().ref_set_threads(n)
