"""State snapshots of an Engine or a Batch: the byte layout written by
mp_engine_snapshot / mp_batch_snapshot (mtlphys_b200/csrc/snapshot.h), read
and written here without a GPU.

  header   64 bytes: b"MTLPSNAP", version, kind (0 engine, 1 batch), scene
           count, particle count, sizes of the embedded structs
  scenes   one record per scene: mp_pbf_params, mp_scene_desc, scene id,
           particle count, dt (batch scenes), sphere center/velocity/radius
  arrays   positions then velocities, float4 per particle, original order

``Engine.save(path)`` / ``Engine.load(path)`` and the same on ``Batch`` go
through the C ABI; ``read``/``write`` here let tools inspect or build
snapshots (for instance to start a batch from states saved by engines).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._abi import PBFParams, SceneDesc

MAGIC = b"MTLPSNAP"
VERSION = 1
KIND_ENGINE, KIND_BATCH = 0, 1


class Header(C.Structure):
    _fields_ = [("magic", C.c_char * 8), ("version", C.c_uint32), ("kind", C.c_uint32),
                ("nscenes", C.c_uint32), ("particles", C.c_uint32), ("params_size", C.c_uint32),
                ("scene_size", C.c_uint32), ("desc_size", C.c_uint32), ("reserved", C.c_uint32 * 7)]


class SceneRecord(C.Structure):
    _fields_ = [("params", PBFParams), ("desc", SceneDesc), ("scene_id", C.c_uint32),
                ("count", C.c_uint32), ("dt", C.c_float), ("sphere", C.c_float * 7)]


@dataclass
class Snapshot:
    kind: int
    scenes: list = field(default_factory=list)  # SceneRecord per scene
    positions: np.ndarray | None = None          # (N, 4) float32
    velocities: np.ndarray | None = None         # (N, 4) float32

    @property
    def particles(self) -> int:
        return 0 if self.positions is None else len(self.positions)


def from_bytes(data: bytes) -> Snapshot:
    data = bytes(data)
    if len(data) < C.sizeof(Header):
        raise ValueError("snapshot shorter than its header")
    h = Header.from_buffer_copy(data[:C.sizeof(Header)])
    if h.magic != MAGIC:
        raise ValueError("not a snapshot (bad magic)")
    if h.version != VERSION:
        raise ValueError(f"unsupported snapshot version {h.version}")
    if (h.params_size, h.scene_size, h.desc_size) != (C.sizeof(PBFParams), C.sizeof(SceneRecord),
                                                      C.sizeof(SceneDesc)):
        raise ValueError("snapshot written by an incompatible build (struct sizes differ)")
    off = C.sizeof(Header)
    need = off + h.nscenes * C.sizeof(SceneRecord) + 32 * h.particles
    if len(data) < need:
        raise ValueError("snapshot truncated")
    scenes = []
    for _ in range(h.nscenes):
        scenes.append(SceneRecord.from_buffer_copy(data[off:off + C.sizeof(SceneRecord)]))
        off += C.sizeof(SceneRecord)
    n = h.particles
    pos = np.frombuffer(data, np.float32, 4 * n, off).reshape(n, 4).copy()
    vel = np.frombuffer(data, np.float32, 4 * n, off + 16 * n).reshape(n, 4).copy()
    if sum(s.count for s in scenes) != n:
        raise ValueError("snapshot particle counts disagree")
    return Snapshot(h.kind, scenes, pos, vel)


def to_bytes(snap: Snapshot) -> bytes:
    n = snap.particles
    h = Header()
    h.magic = MAGIC
    h.version = VERSION
    h.kind = snap.kind
    h.nscenes = len(snap.scenes)
    h.particles = n
    h.params_size = C.sizeof(PBFParams)
    h.scene_size = C.sizeof(SceneRecord)
    h.desc_size = C.sizeof(SceneDesc)
    parts = [bytes(h)] + [bytes(s) for s in snap.scenes]
    parts.append(np.ascontiguousarray(snap.positions, np.float32).reshape(n, 4).tobytes())
    parts.append(np.ascontiguousarray(snap.velocities, np.float32).reshape(n, 4).tobytes())
    return b"".join(parts)


def read(path: str) -> Snapshot:
    with open(path, "rb") as f:
        return from_bytes(f.read())


def write(path: str, snap: Snapshot) -> None:
    with open(path, "wb") as f:
        f.write(to_bytes(snap))
