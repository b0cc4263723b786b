"""B200-native Position-Based Fluids engine.

The simulation step of the reference engine (rakdcolon/mtlphys,
engine/src/Engine.cpp:685-811) as hand-written sm_100a CUDA kernels behind a
C ABI (include/mtlphys_b200.h); this package is the Python surface over that
ABI.  There is no CPU fallback: importing ``Engine`` needs the built
``libmtlphys_b200.so``.
"""
from ._abi import (MP_SCENE_CUBE_DROP, MP_SCENE_DAM_BREAK, MP_SCENE_SPHERE_DROP, MPError,
                   PBFParams, SceneDesc, default_params, default_scene_desc, load)
from .engine import Engine, exclusive_scan

__all__ = [
    "Engine", "PBFParams", "SceneDesc", "MPError", "default_params", "default_scene_desc",
    "exclusive_scan", "load", "MP_SCENE_CUBE_DROP", "MP_SCENE_DAM_BREAK", "MP_SCENE_SPHERE_DROP",
]
