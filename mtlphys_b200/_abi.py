"""ctypes mirror of include/mtlphys_b200.h (structs, constants, prototypes).

The product library is ``mtlphys_b200/libmtlphys_b200.so`` (CUDA kernels for
sm_100a behind a C ABI).  ``load()`` opens it and fails loudly when it is
missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

MP_OK = 0
MP_ERR_INVALID_ARGUMENT = 1
MP_ERR_OUT_OF_MEMORY = 2
MP_ERR_CUDA = 3
MP_ERR_DEVICE = 4
MP_ERR_SPIN_LIMIT = 5
MP_ERR_UNSUPPORTED = 6

MP_DEVERR_SPIN_LIMIT = 0x1
MP_DEVERR_NAN = 0x2
MP_DEVERR_INDEX = 0x4

MP_SCENE_CUBE_DROP = 0
MP_SCENE_DAM_BREAK = 1
MP_SCENE_SPHERE_DROP = 2

MP_SCENE_GRADS = 8
MP_GRAD_SCORR_K = 0
MP_GRAD_CENTER = 1
MP_GRAD_VELOCITY = 4
MP_GRAD_RADIUS = 7

MP_RENDER_BOX = 1
MP_RENDER_SPHERE = 2
MP_RENDER_FOAM = 4
MP_RENDER_BUF_COLOR = 0
MP_RENDER_BUF_DEPTH = 1
MP_RENDER_BUF_SMOOTHED = 2
MP_RENDER_BUF_THICKNESS = 3
MP_RENDER_BUF_NDC_DEPTH = 4

MP_BUF_POSITIONS = 0
MP_BUF_VELOCITIES = 1
MP_BUF_PREV_POSITIONS = 2
MP_BUF_CELL_HASHES = 3
MP_BUF_CELL_START = 4
MP_BUF_SORTED_INDEX = 5
MP_BUF_NEIGHBOR_COUNTS = 6
MP_BUF_LAMBDAS = 7
MP_BUF_FOAM = 8
MP_BUF_SORTED_POSITIONS = 9
MP_BUF_COUNT = 10

# (element width in 32-bit words, numpy dtype) per buffer
BUF_LAYOUT = {
    MP_BUF_POSITIONS: (4, "float32"),
    MP_BUF_VELOCITIES: (4, "float32"),
    MP_BUF_PREV_POSITIONS: (4, "float32"),
    MP_BUF_CELL_HASHES: (1, "uint32"),
    MP_BUF_CELL_START: (1, "uint32"),
    MP_BUF_SORTED_INDEX: (1, "uint32"),
    MP_BUF_NEIGHBOR_COUNTS: (1, "uint32"),
    MP_BUF_LAMBDAS: (1, "float32"),
    MP_BUF_FOAM: (1, "float32"),
    MP_BUF_SORTED_POSITIONS: (4, "float32"),
}


class PBFParams(C.Structure):
    """mp_pbf_params."""

    _fields_ = [
        ("size", C.c_uint32),
        ("solver_iterations", C.c_uint32),
        ("h", C.c_float),
        ("cell_size", C.c_float),
        ("rest_density", C.c_float),
        ("epsilon", C.c_float),
        ("damping", C.c_float),
        ("gravity", C.c_float * 3),
        ("bounds_min", C.c_float * 3),
        ("bounds_max", C.c_float * 3),
        ("scorr_k", C.c_float),
        ("scorr_n", C.c_uint32),
        ("scorr_dq", C.c_float),
        ("max_delta", C.c_float),
        ("vmax", C.c_float),
        ("wall_eps", C.c_float),
        ("floor_friction", C.c_float),
        ("wall_friction", C.c_float),
        ("foam_max_neighbors", C.c_float),
        ("foam_speed_lo", C.c_float),
        ("foam_speed_hi", C.c_float),
        ("sphere_radius", C.c_float),
        ("sphere_gravity", C.c_float),
        ("sphere_drag", C.c_float),
        ("sphere_restitution", C.c_float),
        ("integrate_damping", C.c_float),
        ("integrate_restitution", C.c_float),
        ("mouse_falloff", C.c_float),
    ]

    def copy(self) -> "PBFParams":
        out = PBFParams()
        C.memmove(C.byref(out), C.byref(self), C.sizeof(PBFParams))
        return out

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
    """mp_scene_desc."""

    _fields_ = [
        ("size", C.c_uint32),
        ("lattice", C.c_uint32),
        ("seed", C.c_uint64),
        ("dims", C.c_uint32 * 3),
        ("origin", C.c_float * 3),
        ("spacing", C.c_float),
        ("jitter", C.c_float),
        ("sphere_center", C.c_float * 3),
        ("sphere_velocity", C.c_float * 3),
    ]


class KernelTime(C.Structure):
    """mp_kernel_time."""

    _fields_ = [("name", C.c_char * 32), ("launches", C.c_uint32), ("ms", C.c_double)]


class RenderParams(C.Structure):
    """mp_render_params."""

    _fields_ = [("size", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("flags", C.c_uint32),
                ("eye", C.c_float * 3), ("target", C.c_float * 3), ("fov_y", C.c_float),
                ("z_near", C.c_float), ("z_far", C.c_float), ("particle_radius", C.c_float),
                ("foam_radius_scale", C.c_float)]


class BatchTuning(C.Structure):
    """mp_batch_tuning."""

    _fields_ = [("block", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("ms_per_step", C.c_float)]


_VP = C.c_void_p
_U32 = C.c_uint32
_INT = C.c_int
_SZ = C.c_size_t

# name -> (restype, argtypes)
PROTOTYPES = {
    "mp_last_error": (C.c_char_p, []),
    "mp_abi_version": (_U32, []),
    "mp_default_params": (_INT, [C.POINTER(PBFParams)]),
    "mp_default_scene_desc": (_INT, [C.POINTER(SceneDesc)]),
    "mp_lattice_rest_density": (C.c_double, [C.c_double, C.c_double]),
    "mp_engine_create": (_INT, [_INT, C.POINTER(_VP)]),
    "mp_engine_destroy": (_INT, [_VP]),
    "mp_engine_set_params": (_INT, [_VP, C.POINTER(PBFParams)]),
    "mp_engine_get_params": (_INT, [_VP, C.POINTER(PBFParams)]),
    "mp_engine_reset": (_INT, [_VP, _U32]),
    "mp_engine_reset_scene": (_INT, [_VP, _U32, _U32, C.POINTER(SceneDesc)]),
    "mp_engine_step": (_INT, [_VP, C.c_float, _VP]),
    "mp_engine_build_spatial_hash": (_INT, [_VP, _VP]),
    "mp_engine_set_graph_mode": (_INT, [_VP, _INT]),
    "mp_engine_set_profiling": (_INT, [_VP, _INT]),
    "mp_engine_kernel_times": (_INT, [_VP, C.POINTER(KernelTime), _U32, C.POINTER(_U32)]),
    "mp_step_launch_count": (_U32, [_U32]),
    "mp_engine_particle_count": (_U32, [_VP]),
    "mp_engine_total_cells": (_U32, [_VP]),
    "mp_engine_cell_size": (C.c_float, [_VP]),
    "mp_engine_current_scene": (_U32, [_VP]),
    "mp_engine_grid_dims": (_INT, [_VP, C.POINTER(_U32)]),
    "mp_engine_buffer": (_INT, [_VP, _U32, C.POINTER(_VP), C.POINTER(_SZ)]),
    "mp_engine_upload": (_INT, [_VP, _U32, _VP, _SZ, _VP]),
    "mp_engine_download": (_INT, [_VP, _U32, _VP, _SZ, _VP]),
    "mp_engine_set_sphere": (_INT, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float]),
    "mp_engine_get_sphere": (_INT, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]),
    "mp_engine_check_errors": (_INT, [_VP, C.POINTER(_U32)]),
    "mp_engine_integrate": (_INT, [_VP, C.c_float, _VP]),
    "mp_engine_apply_mouse_pulse": (_INT, [_VP, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                           C.POINTER(C.c_float), C.c_float, _VP]),
    "mp_engine_synchronize": (_INT, [_VP]),
    "mp_batch_create": (_INT, [_INT, C.POINTER(_VP)]),
    "mp_batch_destroy": (_INT, [_VP]),
    "mp_batch_reset": (_INT, [_VP, _U32, C.POINTER(_U32), C.POINTER(_U32), C.POINTER(PBFParams),
                              C.POINTER(SceneDesc), C.POINTER(C.c_float)]),
    "mp_batch_set_dts": (_INT, [_VP, C.POINTER(C.c_float)]),
    "mp_batch_step": (_INT, [_VP, _VP]),
    "mp_batch_set_mode": (_INT, [_VP, _INT]),
    "mp_batch_set_graph_mode": (_INT, [_VP, _INT]),
    "mp_batch_set_launch": (_INT, [_VP, _U32, _U32]),
    "mp_batch_get_launch": (_INT, [_VP, C.POINTER(_U32), C.POINTER(_U32)]),
    "mp_batch_autotune": (_INT, [_VP, _U32, C.POINTER(BatchTuning)]),
    "mp_batch_scene_count": (_U32, [_VP]),
    "mp_batch_particle_count": (_U32, [_VP]),
    "mp_batch_scene_range": (_INT, [_VP, _U32, C.POINTER(_U32), C.POINTER(_U32)]),
    "mp_batch_buffer": (_INT, [_VP, _U32, C.POINTER(_VP), C.POINTER(_SZ)]),
    "mp_batch_upload": (_INT, [_VP, _U32, _VP, _SZ, _VP]),
    "mp_batch_download": (_INT, [_VP, _U32, _VP, _SZ, _VP]),
    "mp_batch_set_sphere": (_INT, [_VP, _U32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float]),
    "mp_batch_get_sphere": (_INT, [_VP, _U32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                   C.POINTER(C.c_float)]),
    "mp_batch_check_errors": (_INT, [_VP, C.POINTER(_U32)]),
    "mp_batch_set_params": (_INT, [_VP, _U32, C.POINTER(PBFParams)]),
    "mp_batch_get_params": (_INT, [_VP, _U32, C.POINTER(PBFParams)]),
    "mp_batch_rollout_forward": (_INT, [_VP, _U32, _U32, _VP]),
    "mp_batch_rollout_backward": (_INT, [_VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "mp_batch_rollout_launch_count": (_U32, [_VP, _U32]),
    "mp_default_render_params": (_INT, [C.POINTER(RenderParams)]),
    "mp_render_camera": (_INT, [C.POINTER(RenderParams), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mp_engine_render": (_INT, [_VP, C.POINTER(RenderParams), _VP, _VP]),
    "mp_engine_render_buffer": (_INT, [_VP, _U32, C.POINTER(_VP), C.POINTER(_SZ)]),
    "mp_engine_snapshot_size": (_SZ, [_VP]),
    "mp_engine_snapshot": (_INT, [_VP, _VP, _SZ]),
    "mp_engine_restore": (_INT, [_VP, _VP, _SZ]),
    "mp_batch_snapshot_size": (_SZ, [_VP]),
    "mp_batch_snapshot": (_INT, [_VP, _VP, _SZ]),
    "mp_batch_restore": (_INT, [_VP, _VP, _SZ]),
    "mp_exclusive_scan_scratch_bytes": (_SZ, [_U32]),
    "mp_exclusive_scan": (_INT, [_VP, _VP, _U32, _VP, _SZ, _VP]),
    "mp_exclusive_scan_noalloc": (_INT, [_VP, _VP, _U32, _VP]),
    "mp_exclusive_scan_status": (_INT, [_VP, _VP]),
    "mp_debug_exclusive_scan_from_ticket": (_INT, [_VP, _VP, _U32, _VP, _SZ, C.c_uint64, _VP]),
    "mp_set_spin_limit": (_INT, [_U32]),
    "mp_set_device_allocator": (_INT, [_VP, _VP, _VP]),
    "mp_batch_debug_barrier_extra": (_INT, [_VP, _U32]),
}

# mp_device_alloc_fn / mp_device_free_fn
DEVICE_ALLOC_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_void_p), C.c_size_t, C.c_int, C.c_void_p)
DEVICE_FREE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_void_p)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmtlphys_b200.so")

_lib = None


class MPError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where} failed with status {code}: {msg}")
        self.code = code


def load() -> C.CDLL:
    """Open the product library (built by ``__graft_entry__.build()``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()'); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code: int, where: str) -> None:
    if code != MP_OK:
        msg = load().mp_last_error().decode(errors="replace")
        raise MPError(code, where, msg)


def default_params() -> PBFParams:
    p = PBFParams()
    check(load().mp_default_params(C.byref(p)), "mp_default_params")
    return p


def default_render_params(**kw) -> RenderParams:
    rp = RenderParams()
    check(load().mp_default_render_params(C.byref(rp)), "mp_default_render_params")
    for k, v in kw.items():
        cur = getattr(rp, k)
        if isinstance(cur, C.Array):
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(rp, k, v)
    return rp


def render_camera(rp: RenderParams):
    """(view, proj) of a render as row-major 4x4 float32 numpy matrices."""
    import numpy as np

    v, p = (C.c_float * 16)(), (C.c_float * 16)()
    check(load().mp_render_camera(C.byref(rp), v, p), "mp_render_camera")
    return (np.array(v[:], np.float32).reshape(4, 4).T.copy(), np.array(p[:], np.float32).reshape(4, 4).T.copy())


def default_scene_desc() -> SceneDesc:
    d = SceneDesc()
    check(load().mp_default_scene_desc(C.byref(d)), "mp_default_scene_desc")
    return d
