"""Python surface of the multi-scene batch (mp_batch_* of the C ABI).

Many independent scenes, each with its own particle count, parameters, dt
and seeding, advance together: one persistent cooperative launch per step
(optionally replayed as a CUDA graph), or, in serial mode, the same kernel
launched scene by scene.  Scene s owns the particle range ``scene_range(s)``
of the batch's buffers and gets exactly the results a single-scene
``Engine`` would give it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import BUF_LAYOUT, MP_BUF_POSITIONS, MP_BUF_VELOCITIES, PBFParams, SceneDesc, check
from .engine import _CudaArray, stream_handle


class Batch:
    def __init__(self, device: int = 0):
        self._lib = _abi.load()
        h = C.c_void_p()
        check(self._lib.mp_batch_create(int(device), C.byref(h)), "mp_batch_create")
        self._h = h
        self.device = int(device)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mp_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset(self, counts, params, dts, scenes=None, descs=None) -> None:
        """counts[s] particles per scene; params: one PBFParams per scene (or
        one for all); dts: per-scene time steps; scenes: MP_SCENE_* ids;
        descs: SceneDesc per scene (None: reference placement)."""
        n = len(counts)
        if isinstance(params, PBFParams):
            params = [params] * n
        cnt = (C.c_uint32 * n)(*[int(x) for x in counts])
        prm = (PBFParams * n)(*params)
        dt = (C.c_float * n)(*[float(x) for x in dts])
        sid = (C.c_uint32 * n)(*[int(x) for x in scenes]) if scenes is not None else None
        dsc = (SceneDesc * n)(*descs) if descs is not None else None
        check(self._lib.mp_batch_reset(self._h, n, cnt, sid, prm, dsc, dt), "mp_batch_reset")

    def set_dts(self, dts) -> None:
        n = self.scene_count()
        check(self._lib.mp_batch_set_dts(self._h, (C.c_float * n)(*dts)), "mp_batch_set_dts")

    def step(self, stream=None) -> None:
        check(self._lib.mp_batch_step(self._h, stream_handle(stream)), "mp_batch_step")

    def set_serial(self, serial: bool) -> None:
        check(self._lib.mp_batch_set_mode(self._h, 1 if serial else 0), "mp_batch_set_mode")

    def set_graph_mode(self, enable: bool) -> None:
        check(self._lib.mp_batch_set_graph_mode(self._h, 1 if enable else 0), "mp_batch_set_graph_mode")

    def set_launch(self, block: int, blocks_per_sm: int = 0) -> None:
        check(self._lib.mp_batch_set_launch(self._h, block, blocks_per_sm), "mp_batch_set_launch")

    def launch(self) -> tuple[int, int]:
        b, g = C.c_uint32(), C.c_uint32()
        check(self._lib.mp_batch_get_launch(self._h, C.byref(b), C.byref(g)), "mp_batch_get_launch")
        return b.value, g.value

    def autotune(self, steps: int = 3) -> dict:
        t = _abi.BatchTuning()
        check(self._lib.mp_batch_autotune(self._h, steps, C.byref(t)), "mp_batch_autotune")
        return {"block": t.block, "blocks_per_sm": t.blocks_per_sm, "ms_per_step": t.ms_per_step}

    def scene_count(self) -> int:
        return int(self._lib.mp_batch_scene_count(self._h))

    def particle_count(self) -> int:
        return int(self._lib.mp_batch_particle_count(self._h))

    def scene_range(self, s: int) -> tuple[int, int]:
        f, c = C.c_uint32(), C.c_uint32()
        check(self._lib.mp_batch_scene_range(self._h, s, C.byref(f), C.byref(c)), "mp_batch_scene_range")
        return f.value, c.value

    def read(self, which: int, count: int | None = None) -> np.ndarray:
        width, dtype = BUF_LAYOUT[which]
        if count is None:
            p = C.c_void_p()
            nb = C.c_size_t()
            check(self._lib.mp_batch_buffer(self._h, which, C.byref(p), C.byref(nb)), "mp_batch_buffer")
            count = nb.value // (4 * width)
        out = np.empty((count, width) if width > 1 else (count,), dtype=dtype)
        check(self._lib.mp_batch_download(self._h, which, out.ctypes.data_as(C.c_void_p), count, None),
              "mp_batch_download")
        return out

    def write(self, which: int, data) -> None:
        width, dtype = BUF_LAYOUT[which]
        arr = np.ascontiguousarray(data, dtype=dtype)
        check(self._lib.mp_batch_upload(self._h, which, arr.ctypes.data_as(C.c_void_p), arr.shape[0],
                                        None), "mp_batch_upload")
        self._lib.mp_batch_check_errors(self._h, None)  # waits: the host array may go away

    def positions(self) -> np.ndarray:
        return self.read(MP_BUF_POSITIONS)

    def velocities(self) -> np.ndarray:
        return self.read(MP_BUF_VELOCITIES)

    def sphere(self, s: int) -> np.ndarray:
        c = (C.c_float * 3)()
        v = (C.c_float * 3)()
        r = C.c_float()
        check(self._lib.mp_batch_get_sphere(self._h, s, c, v, C.byref(r)), "mp_batch_get_sphere")
        return np.array([c[0], c[1], c[2], v[0], v[1], v[2], r.value], np.float32)

    def set_sphere(self, s: int, center, velocity, radius: float) -> None:
        check(self._lib.mp_batch_set_sphere(self._h, s, (C.c_float * 3)(*center),
                                            (C.c_float * 3)(*velocity), C.c_float(radius)),
              "mp_batch_set_sphere")

    def check_errors(self) -> int:
        bits = C.c_uint32()
        check(self._lib.mp_batch_check_errors(self._h, C.byref(bits)), "mp_batch_check_errors")
        return bits.value

    # ---- state snapshots ----
    def snapshot_bytes(self) -> bytes:
        """The engine state as a snapshot byte string (waits for queued work)."""
        size = int(self._lib.mp_batch_snapshot_size(self._h))
        buf = (C.c_char * size)()
        check(self._lib.mp_batch_snapshot(self._h, buf, size), "mp_batch_snapshot")
        return bytes(buf)

    def restore_bytes(self, data: bytes) -> None:
        """Re-create the state saved in a snapshot byte string."""
        buf = C.create_string_buffer(bytes(data), len(data))
        check(self._lib.mp_batch_restore(self._h, buf, len(data)), "mp_batch_restore")

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(self.snapshot_bytes())

    def load(self, path: str) -> None:
        with open(path, "rb") as f:
            self.restore_bytes(f.read())

    def params(self, s: int) -> PBFParams:
        p = PBFParams()
        check(self._lib.mp_batch_get_params(self._h, s, C.byref(p)), "mp_batch_get_params")
        return p

    def set_params(self, s: int, p: PBFParams) -> None:
        check(self._lib.mp_batch_set_params(self._h, s, C.byref(p)), "mp_batch_set_params")

    def buffer(self, which: int) -> tuple[int, int]:
        p = C.c_void_p()
        nb = C.c_size_t()
        check(self._lib.mp_batch_buffer(self._h, which, C.byref(p), C.byref(nb)), "mp_batch_buffer")
        return int(p.value or 0), int(nb.value)

    def tensor(self, which: int):
        """Zero-copy torch view of buffer `which` (all scenes' particles)."""
        import torch

        width, dtype = BUF_LAYOUT[which]
        ptr, _ = self.buffer(which)
        count = self.particle_count()
        shape = (count, width) if width > 1 else (count,)
        typestr = "<f4" if dtype == "float32" else "<i4"
        return torch.as_tensor(_CudaArray(ptr, shape, typestr, self), device=f"cuda:{self.device}")

    # ---- differentiable rollouts ----

    def rollout_forward(self, steps: int, checkpoint_every: int = 10, stream=None) -> None:
        """Advance `steps` steps keeping a checkpoint every `checkpoint_every`."""
        check(self._lib.mp_batch_rollout_forward(self._h, int(steps), int(checkpoint_every),
                                                 stream_handle(stream)), "mp_batch_rollout_forward")

    def rollout_backward(self, dpos=None, dvel=None, stream=None):
        """Adjoint of the last rollout_forward.  dpos, dvel: dL/d(final
        positions, velocities) as (N, 4) float32 CUDA tensors (or None).
        Returns (dL/dpos0, dL/dvel0, per-scene grads (S, MP_SCENE_GRADS) float64)."""
        import torch

        n, S = self.particle_count(), self.scene_count()
        dev = torch.device("cuda", self.device)
        out_p = torch.empty((n, 4), dtype=torch.float32, device=dev)
        out_v = torch.empty((n, 4), dtype=torch.float32, device=dev)
        out_s = torch.empty((S, _abi.MP_SCENE_GRADS), dtype=torch.float64, device=dev)

        def ptr(t):
            if t is None:
                return None
            assert t.is_cuda and t.dtype == torch.float32 and t.shape == (n, 4) and t.is_contiguous()
            return C.c_void_p(t.data_ptr())

        check(self._lib.mp_batch_rollout_backward(self._h, ptr(dpos), ptr(dvel), C.c_void_p(out_p.data_ptr()),
                                                  C.c_void_p(out_v.data_ptr()), C.c_void_p(out_s.data_ptr()),
                                                  stream_handle(stream)), "mp_batch_rollout_backward")
        return out_p, out_v, out_s

    def rollout_launch_count(self, steps: int) -> int:
        return int(self._lib.mp_batch_rollout_launch_count(self._h, int(steps)))
