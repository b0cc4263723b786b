"""Python surface of the B200 PBF engine over its C ABI.

``Engine`` mirrors the reference's ``mtlphys::Engine``
(engine/include/mtlphys/Engine.hpp:27-190) and its Obj-C++ bridge
(app/bridge/EngineBridge.h:10-33): ``reset(n[, scene])``, ``step(dt)``,
``build_spatial_hash()``, ``particle_count()``, ``total_cells()``,
``cell_size()``, ``current_scene()`` and the diagnostic buffer accessors.
Where the reference takes an ``MTL::CommandBuffer`` this takes an optional
CUDA stream (``torch.cuda.Stream``, a raw ``cudaStream_t`` int, or None for
the legacy default stream); work is asynchronous on it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (BUF_LAYOUT, MP_BUF_CELL_HASHES, MP_BUF_CELL_START, MP_BUF_FOAM,
                   MP_BUF_LAMBDAS, MP_BUF_NEIGHBOR_COUNTS, MP_BUF_POSITIONS,
                   MP_BUF_PREV_POSITIONS, MP_BUF_SORTED_INDEX, MP_BUF_SORTED_POSITIONS,
                   MP_BUF_VELOCITIES, PBFParams, SceneDesc, check)


def stream_handle(stream) -> C.c_void_p:
    """cudaStream_t of `stream` (torch stream, int handle or None)."""
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    handle = getattr(stream, "cuda_stream", None)
    if handle is None:
        raise TypeError(f"not a CUDA stream: {stream!r}")
    return C.c_void_p(handle)


class _CudaArray:
    """Minimal __cuda_array_interface__ holder for zero-copy torch views."""

    def __init__(self, ptr: int, shape, typestr: str, owner):
        self.__cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": typestr, "data": (ptr, False), "version": 2,
            "strides": None,
        }
        self._owner = owner


class Engine:
    kSceneCubeDrop = _abi.MP_SCENE_CUBE_DROP
    kSceneDamBreak = _abi.MP_SCENE_DAM_BREAK
    kSceneSphereDrop = _abi.MP_SCENE_SPHERE_DROP

    def __init__(self, device: int = 0, params: PBFParams | None = None):
        """Engine(device): binds the GPU and seeds 200K cube-drop particles
        (Engine.cpp:97-102).  `params` are applied before that reset."""
        self._lib = _abi.load()
        h = C.c_void_p()
        check(self._lib.mp_engine_create(int(device), C.byref(h)), "mp_engine_create")
        self._h = h
        self.device = int(device)
        if params is not None:
            self.set_params(params)
            self.reset(200_000, self.kSceneCubeDrop)

    # ---- lifetime ----------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mp_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- parameters / scenes ---------------------------------------------------
    def params(self) -> PBFParams:
        p = PBFParams()
        check(self._lib.mp_engine_get_params(self._h, C.byref(p)), "mp_engine_get_params")
        return p

    def set_params(self, p: PBFParams) -> None:
        check(self._lib.mp_engine_set_params(self._h, C.byref(p)), "mp_engine_set_params")

    def reset(self, n: int, scene: int | None = None, desc: SceneDesc | None = None) -> None:
        """reset(particleCount[, sceneIdx]) (Engine.cpp:125-134)."""
        if scene is None and desc is None:
            check(self._lib.mp_engine_reset(self._h, int(n)), "mp_engine_reset")
            return
        if scene is None:
            scene = self.current_scene()
        check(self._lib.mp_engine_reset_scene(self._h, int(n), int(scene),
                                              C.byref(desc) if desc is not None else None),
              "mp_engine_reset_scene")

    # ---- simulation ----------------------------------------------------------------
    def step(self, dt: float, stream=None) -> None:
        check(self._lib.mp_engine_step(self._h, C.c_float(dt), stream_handle(stream)),
              "mp_engine_step")

    def build_spatial_hash(self, stream=None) -> None:
        check(self._lib.mp_engine_build_spatial_hash(self._h, stream_handle(stream)),
              "mp_engine_build_spatial_hash")

    def set_graph_mode(self, enable: bool) -> None:
        check(self._lib.mp_engine_set_graph_mode(self._h, 1 if enable else 0),
              "mp_engine_set_graph_mode")

    def set_profiling(self, enable: bool) -> None:
        check(self._lib.mp_engine_set_profiling(self._h, 1 if enable else 0),
              "mp_engine_set_profiling")

    def kernel_times(self) -> dict:
        """{kernel: (launches, total ms)} since the last call (profiling on)."""
        cap = 64
        arr = (_abi.KernelTime * cap)()
        cnt = C.c_uint32()
        check(self._lib.mp_engine_kernel_times(self._h, arr, cap, C.byref(cnt)),
              "mp_engine_kernel_times")
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].ms))
                for i in range(min(cnt.value, cap))}

    def synchronize(self) -> None:
        check(self._lib.mp_engine_synchronize(self._h), "mp_engine_synchronize")

    def check_errors(self) -> int:
        """Wait, then raise if a kernel set the device error word."""
        bits = C.c_uint32()
        check(self._lib.mp_engine_check_errors(self._h, C.byref(bits)), "mp_engine_check_errors")
        return bits.value

    def error_bits(self) -> int:
        """Wait and return (and clear) the device error word without raising."""
        bits = C.c_uint32()
        self._lib.mp_engine_check_errors(self._h, C.byref(bits))
        return bits.value

    # ---- queries ---------------------------------------------------------------------
    def particle_count(self) -> int:
        return int(self._lib.mp_engine_particle_count(self._h))

    def total_cells(self) -> int:
        return int(self._lib.mp_engine_total_cells(self._h))

    def cell_size(self) -> float:
        return float(self._lib.mp_engine_cell_size(self._h))

    def current_scene(self) -> int:
        return int(self._lib.mp_engine_current_scene(self._h))

    def grid_dims(self) -> tuple[int, int, int]:
        d = (C.c_uint32 * 3)()
        check(self._lib.mp_engine_grid_dims(self._h, d), "mp_engine_grid_dims")
        return (d[0], d[1], d[2])

    # ---- buffers ---------------------------------------------------------------------
    def buffer(self, which: int) -> tuple[int, int]:
        """(device pointer, bytes) of buffer `which` (MP_BUF_*), borrowed."""
        p = C.c_void_p()
        n = C.c_size_t()
        check(self._lib.mp_engine_buffer(self._h, int(which), C.byref(p), C.byref(n)),
              "mp_engine_buffer")
        return int(p.value or 0), int(n.value)

    def _count(self, which: int) -> int:
        width, _ = BUF_LAYOUT[which]
        _, nbytes = self.buffer(which)
        return nbytes // (4 * width)

    def read(self, which: int, count: int | None = None, stream=None) -> np.ndarray:
        width, dtype = BUF_LAYOUT[which]
        if count is None:
            count = self._count(which)
        out = np.empty((count, width) if width > 1 else (count,), dtype=dtype)
        check(self._lib.mp_engine_download(self._h, int(which), out.ctypes.data_as(C.c_void_p),
                                           count, stream_handle(stream)), "mp_engine_download")
        return out

    def write(self, which: int, data, stream=None) -> None:
        width, dtype = BUF_LAYOUT[which]
        arr = np.ascontiguousarray(data, dtype=dtype)
        count = arr.shape[0] if arr.ndim else 0
        if width > 1 and (arr.ndim != 2 or arr.shape[1] != width):
            raise ValueError(f"buffer {which} takes ({count}, {width}) arrays")
        check(self._lib.mp_engine_upload(self._h, int(which), arr.ctypes.data_as(C.c_void_p), count,
                                         stream_handle(stream)), "mp_engine_upload")
        # pageable host memory: the copy has been staged when upload returns
        self._keepalive = arr

    def tensor(self, which: int):
        """Zero-copy torch view of buffer `which` on the engine's device."""
        import torch

        width, dtype = BUF_LAYOUT[which]
        ptr, nbytes = self.buffer(which)
        count = nbytes // (4 * width)
        shape = (count, width) if width > 1 else (count,)
        typestr = "<f4" if dtype == "float32" else "<u4"
        if dtype == "uint32":
            t = torch.as_tensor(_CudaArray(ptr, shape, "<i4", self), device=f"cuda:{self.device}")
            return t
        return torch.as_tensor(_CudaArray(ptr, shape, typestr, self), device=f"cuda:{self.device}")

    # reference accessor names (Engine.hpp:83-90)
    def positions(self) -> np.ndarray:
        return self.read(MP_BUF_POSITIONS)

    def velocities(self) -> np.ndarray:
        return self.read(MP_BUF_VELOCITIES)

    def prev_positions(self) -> np.ndarray:
        return self.read(MP_BUF_PREV_POSITIONS)

    def cell_hashes(self) -> np.ndarray:
        return self.read(MP_BUF_CELL_HASHES)

    def cell_start(self) -> np.ndarray:
        return self.read(MP_BUF_CELL_START)

    def sorted_index(self) -> np.ndarray:
        return self.read(MP_BUF_SORTED_INDEX)

    def neighbor_counts(self) -> np.ndarray:
        return self.read(MP_BUF_NEIGHBOR_COUNTS)

    def lambdas(self) -> np.ndarray:
        return self.read(MP_BUF_LAMBDAS)

    def foam(self) -> np.ndarray:
        return self.read(MP_BUF_FOAM)

    def sorted_positions(self) -> np.ndarray:
        return self.read(MP_BUF_SORTED_POSITIONS)

    def set_positions(self, pos4) -> None:
        self.write(MP_BUF_POSITIONS, pos4)

    def set_velocities(self, vel4) -> None:
        self.write(MP_BUF_VELOCITIES, vel4)

    # ---- sphere (scene 2) ------------------------------------------------------------
    def sphere(self) -> np.ndarray:
        c = (C.c_float * 3)()
        v = (C.c_float * 3)()
        r = C.c_float()
        check(self._lib.mp_engine_get_sphere(self._h, c, v, C.byref(r)), "mp_engine_get_sphere")
        return np.array([c[0], c[1], c[2], v[0], v[1], v[2], r.value], np.float32)

    def integrate(self, dt: float, stream=None) -> None:
        """Engine::integrate: the legacy semi-implicit Euler step with box bounds."""
        check(self._lib.mp_engine_integrate(self._h, C.c_float(dt), stream_handle(stream)),
              "mp_engine_integrate")

    def apply_mouse_pulse(self, ray_origin, ray_dir, force, radius: float, stream=None) -> None:
        """Engine::applyMousePulse: add force * exp(-r^2 / (R^2 falloff)) to the
        velocities of particles within `radius` of the ray (ray_dir normalized)."""
        v3 = lambda a: (C.c_float * 3)(*[float(x) for x in a])
        check(self._lib.mp_engine_apply_mouse_pulse(self._h, v3(ray_origin), v3(ray_dir), v3(force),
                                                    C.c_float(radius), stream_handle(stream)),
              "mp_engine_apply_mouse_pulse")

    # ---- headless rendering ----
    def render(self, params=None, stream=None, **kw):
        """Engine::render into a device image: (H, W, 4) float32 torch tensor
        of linear RGBA in [0, 1], y = 0 on the top row.  params: a
        RenderParams (default: _abi.default_render_params(**kw))."""
        import torch

        rp = params if params is not None else _abi.default_render_params(**kw)
        out = torch.empty((rp.height, rp.width, 4), dtype=torch.float32, device=f"cuda:{self.device}")
        check(self._lib.mp_engine_render(self._h, C.byref(rp), C.c_void_p(out.data_ptr()),
                                         stream_handle(stream)), "mp_engine_render")
        return out

    def render_buffer(self, which: int):
        """Zero-copy torch view of an image buffer of the last render (MP_RENDER_BUF_*)."""
        import torch

        p, nb = C.c_void_p(), C.c_size_t()
        check(self._lib.mp_engine_render_buffer(self._h, which, C.byref(p), C.byref(nb)),
              "mp_engine_render_buffer")
        shape = (nb.value // 16, 4) if which == _abi.MP_RENDER_BUF_COLOR else (nb.value // 4,)
        typestr = "<u4" if which == _abi.MP_RENDER_BUF_DEPTH else "<f4"
        t = torch.as_tensor(_CudaArray(int(p.value), shape, "<f4" if typestr == "<f4" else "<i4", self),
                            device=f"cuda:{self.device}")
        return t.view(torch.float32) if which == _abi.MP_RENDER_BUF_DEPTH else t

    # ---- state snapshots ----
    def snapshot_bytes(self) -> bytes:
        """The engine state as a snapshot byte string (waits for queued work)."""
        size = int(self._lib.mp_engine_snapshot_size(self._h))
        buf = (C.c_char * size)()
        check(self._lib.mp_engine_snapshot(self._h, buf, size), "mp_engine_snapshot")
        return bytes(buf)

    def restore_bytes(self, data: bytes) -> None:
        """Re-create the state saved in a snapshot byte string."""
        buf = C.create_string_buffer(bytes(data), len(data))
        check(self._lib.mp_engine_restore(self._h, buf, len(data)), "mp_engine_restore")

    def save(self, path: str) -> None:
        with open(path, "wb") as f:
            f.write(self.snapshot_bytes())

    def load(self, path: str) -> None:
        with open(path, "rb") as f:
            self.restore_bytes(f.read())

    def set_sphere(self, center, velocity, radius: float) -> None:
        c = (C.c_float * 3)(*center)
        v = (C.c_float * 3)(*velocity)
        check(self._lib.mp_engine_set_sphere(self._h, c, v, C.c_float(radius)),
              "mp_engine_set_sphere")


def exclusive_scan(inp, out=None, stream=None):
    """runExclusiveScan (Engine.cpp:843-882) on torch uint32/int32 CUDA
    tensors through mp_exclusive_scan; scratch comes from torch's allocator."""
    import torch

    lib = _abi.load()
    n = inp.numel()
    if out is None:
        out = torch.empty_like(inp)
    nbytes = lib.mp_exclusive_scan_scratch_bytes(n)
    scratch = torch.empty(max(int(nbytes), 8), dtype=torch.uint8, device=inp.device)
    if stream is None:
        stream = torch.cuda.current_stream(inp.device)
    check(lib.mp_exclusive_scan(C.c_void_p(inp.data_ptr()), C.c_void_p(out.data_ptr()), n,
                                C.c_void_p(scratch.data_ptr()), C.c_size_t(scratch.numel()),
                                stream_handle(stream)), "mp_exclusive_scan")
    return out
