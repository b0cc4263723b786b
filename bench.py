"""PBF step benchmark on B200 (one JSON line on stdout from rank 0).

Workload (default): the 1,003,520-particle dam break in an 86h cube box
(636,056 hash cells), 5 solver iterations, dt = 1/120 s, seeded jittered
lattice (synthetic; see mtlphys_b200/configs.py).  A "step" is one full PBF
step: predict, spatial hash, K x (lambda, delta), scatter-back, finalize,
foam.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value          ms per 1M-particle step for the whole job: device time (CUDA
               events on the engine's stream, L2 flushed between timed steps,
               max over ranks) / (K * N).  N > 1 runs N independent replicas
               (a single scene does not shard: no data-path collective).
e2e            the same metric through the C ABI with the state in pinned
               host memory: every step uploads positions + velocities, steps,
               and downloads them; the timed region's K steps again from its
               start state, so e2e - value is the cost of the copies.
roofline       the dominant kernel's algorithmic bytes per launch / its mean
               CUDA-event duration, against the measured HBM copy bandwidth.
three_iterations  the same scene stepped with 3 solver iterations (the
               step an HBM-fraction target is usually quoted for): ms per
               step and the whole step's algorithmic bytes / time / peak.
cpu_baseline   the FP64 oracle (OpenMP on the host cores) on a bounded
               sample of the same workload (rank 0, N = 1).
--impl reference  the reference's own compute shaders compiled as C++
               (oracle/_ref; OpenMP on all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PBF step ms @1M (%HBM peak); batched vs serial scenes/s; adjoint/fwd ratio"
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 256 << 20


# ---- algorithmic bytes (reference dataflow, each array element read or written
# once per reference kernel that touches it) --------------------------------------
def kernel_bytes(n: int, c: int) -> dict:
    """Bytes per launch of each kernel of this engine, as the sum of the
    reference kernels it replaces (predict 64N, hash 20N, count 4N+8C, zero
    8C, scan 16C, scatter 8N+12C, gather 36N, countNeighbors 40N+4C, lambda
    28N+4C, delta 36N+4C, scatter-back 36N, finalize 64N, foam 24N)."""
    return {
        "predict_hash": 88 * n + 8 * c,
        "scan": 24 * c,
        "scatter": 8 * n + 12 * c,
        "sort_gather": 36 * n,
        "long_segments": 0,
        "lambda_count": 68 * n + 8 * c,
        "lambda": 28 * n + 4 * c,
        "delta": 36 * n + 4 * c,
        "delta_finalize": 160 * n + 4 * c,
    }


def step_bytes(n: int, c: int, k: int) -> int:
    return (296 + 64 * k) * n + (48 + 8 * k) * c


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---- clocks ------------------------------------------------------------------------
REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]


class ClockSampler:
    """SM clock and clock-event reasons of one GPU, sampled every few
    milliseconds through NVML by a thread while the timed region runs (a
    1M-particle timed region lasts tens of milliseconds, so nvidia-smi's
    200 ms loop would see at most one sample); nvidia-smi is the fallback."""

    PERIOD_S = 0.004

    def __init__(self, gpu_uuid: str):
        self.uuid = gpu_uuid
        self.samples: list[tuple[float, float, set]] = []
        self.source = None
        self._stop = threading.Event()
        self._thread = None
        self._proc = None

    def _nvml_loop(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((sm, mx, {k for k, b in bits.items() if r & b}))
            except Exception:
                pass
            self._stop.wait(self.PERIOD_S)

    def _smi_loop(self):
        for line in self._proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm, mx = float(parts[0]), float(parts[1])
            except ValueError:
                continue
            self.samples.append((sm, mx, {k for k, v in zip(REASONS, parts[4:8])
                                          if v.lower().startswith("active")}))

    def __enter__(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByUUID(self.uuid)
            self._thread = threading.Thread(target=self._nvml_loop, args=(nv, h), daemon=True)
            self.source = "nvml"
        except Exception:
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            try:
                self._proc = subprocess.Popen(
                    ["nvidia-smi", "-i", self.uuid, f"--query-gpu={q}", "--format=csv,noheader,nounits",
                     "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._thread = threading.Thread(target=self._smi_loop, daemon=True)
                self.source = "nvidia-smi"
            except Exception:
                self._thread = None
        if self._thread is not None:
            self._thread.start()
            t0 = time.perf_counter()  # the first sample lands before the timed region
            while not self.samples and time.perf_counter() - t0 < 2.0:
                time.sleep(0.001)
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=5)

    def summary(self) -> dict:
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": self.source}
        reasons = set().union(*(r for _, _, r in self.samples))
        return {"sm_mhz": statistics.median(s for s, _, _ in self.samples),
                "sm_max_mhz": max(m for _, m, _ in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": self.source}


# ---- distributed plumbing ----------------------------------------------------------
def dist_setup(n_gpus: int):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def gpu_uuid(local: int) -> str:
    import torch

    try:
        u = str(torch.cuda.get_device_properties(local).uuid)
        return u if u.startswith("GPU-") else f"GPU-{u}"
    except Exception:
        return str(local)


# ---- our arm -------------------------------------------------------------------------
def run_ours(args, world, rank, local) -> dict | None:
    import ctypes as C

    import numpy as np
    import torch

    from mtlphys_b200 import Engine, _abi, configs

    w = configs.WORKLOADS[args.workload]()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    e = Engine(local)
    e.set_params(w.params)
    e.reset(w.n, w.scene, w.desc)
    n, k_it = w.n, int(w.params.solver_iterations)
    cells = e.total_cells()
    e.set_graph_mode(True)

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.zero_()

    for _ in range(args.warmup):
        e.step(w.dt, stream)
    stream.synchronize()
    if e.check_errors():
        raise RuntimeError("device error during warm-up")
    # the timed region's start state, in pinned host memory: the end-to-end
    # leg below uploads it and replays the same steps through the C ABI
    lib = _abi.load()
    sh = C.c_void_p(stream.cuda_stream)
    h_pos = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    h_vel = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    _abi.check(lib.mp_engine_download(e._h, _abi.MP_BUF_POSITIONS, C.c_void_p(h_pos.data_ptr()), n, sh), "download")
    _abi.check(lib.mp_engine_download(e._h, _abi.MP_BUF_VELOCITIES, C.c_void_p(h_vel.data_ptr()), n, sh), "download")
    stream.synchronize()
    start_state = (h_pos.numpy().copy(), h_vel.numpy().copy())  # for the CPU baseline

    # ---- timed region: K steps, L2 flushed between steps (outside the events)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    with ClockSampler(gpu_uuid(local)) as clk:
        for i in range(args.steps):
            flush_l2()
            starts[i].record(stream)
            e.step(w.dt, stream)
            ends[i].record(stream)
        torch.cuda.synchronize(dev)
    dist_barrier(world)
    total_ms = sum(s.elapsed_time(t) for s, t in zip(starts, ends))
    e.check_errors()
    timed_final = e.positions()  # the end-to-end leg must arrive at the same state
    total_ms = dist_max(total_ms, world)
    ms_per_step = total_ms / args.steps
    value = total_ms / (args.steps * world)

    # ---- hot L2: the timed region's steps again from its start state, back to
    # back without the flush (for reference only: value - hot is the flush's cost)
    _abi.check(lib.mp_engine_upload(e._h, _abi.MP_BUF_POSITIONS, C.c_void_p(h_pos.data_ptr()), n, sh), "upload")
    _abi.check(lib.mp_engine_upload(e._h, _abi.MP_BUF_VELOCITIES, C.c_void_p(h_vel.data_ptr()), n, sh), "upload")
    stream.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        e.step(w.dt, stream)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    hot_ms = ev0.elapsed_time(ev1) / args.steps

    # ---- per-kernel timing (CUDA events around every launch, captured with
    # the step as event nodes of its graph, so no host launch gaps; L2 flushed)
    e.set_graph_mode(True)
    e.set_profiling(True)
    e.kernel_times()
    # from the timed region's start state, so the kernels see the same steps
    _abi.check(lib.mp_engine_upload(e._h, _abi.MP_BUF_POSITIONS, C.c_void_p(h_pos.data_ptr()), n, sh), "upload")
    _abi.check(lib.mp_engine_upload(e._h, _abi.MP_BUF_VELOCITIES, C.c_void_p(h_vel.data_ptr()), n, sh), "upload")
    stream.synchronize()
    prof_steps = max(3, min(args.steps, 10))
    for _ in range(prof_steps):
        flush_l2()
        e.step(w.dt, stream)
    times = e.kernel_times()
    e.set_profiling(False)
    kb = kernel_bytes(n, cells)
    kernels = {}
    for name, (launches, ms) in times.items():
        avg = ms / max(1, launches)
        gbs = kb.get(name, 0) / (avg * 1e-3) / 1e9 if avg > 0 else 0.0
        kernels[name] = {"launches_per_step": launches / prof_steps, "ms": round(avg, 5),
                         "algorithmic_bytes": kb.get(name, 0), "GB/s": round(gbs, 1)}
    dominant = max(kernels, key=lambda k: kernels[k]["ms"] * kernels[k]["launches_per_step"])
    peak, peak_kind = measured_hbm_peak()
    dk = kernels[dominant]
    traffic = read_traffic(dominant)
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": dk["GB/s"], "peak": peak,
                "unit": "GB/s", "frac": round(dk["GB/s"] / peak, 4), "traffic": traffic,
                "peak_source": peak_kind,
                "step_frac": round(step_bytes(n, cells, k_it) / (ms_per_step * 1e-3) / 1e9 / peak, 4)}

    # ---- end to end through the C ABI with host (pinned) buffers: the timed
    # region's K steps again from its start state (the state is positions and
    # velocities; the first upload restores it), so e2e - value is the copies
    e.set_graph_mode(True)
    e2e_steps = args.steps

    def e2e_step():
        _abi.check(lib.mp_engine_upload(e._h, _abi.MP_BUF_POSITIONS, C.c_void_p(h_pos.data_ptr()), n, sh), "upload")
        _abi.check(lib.mp_engine_upload(e._h, _abi.MP_BUF_VELOCITIES, C.c_void_p(h_vel.data_ptr()), n, sh), "upload")
        _abi.check(lib.mp_engine_step(e._h, C.c_float(w.dt), sh), "step")
        _abi.check(lib.mp_engine_download(e._h, _abi.MP_BUF_POSITIONS, C.c_void_p(h_pos.data_ptr()), n, sh), "download")
        _abi.check(lib.mp_engine_download(e._h, _abi.MP_BUF_VELOCITIES, C.c_void_p(h_vel.data_ptr()), n, sh), "download")

    # graph re-captured (the profiling leg ran without it) outside the timed
    # steps: one step, then the start state again
    e.step(w.dt, stream)
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    e2e_ms = 0.0
    for _ in range(e2e_steps):
        flush_l2()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        e2e_step()
        s1.record(stream)
        s1.synchronize()
        e2e_ms += s0.elapsed_time(s1)
    e.check_errors()
    e2e_ms = dist_max(e2e_ms, world)
    e2e_value = e2e_ms / (e2e_steps * world)
    e2e_same = bool((h_pos.numpy() == timed_final).all())
    e.close()

    # ---- the same scene at 3 solver iterations (the step the HBM target is stated for)
    w3 = configs.WORKLOADS[args.workload]()
    w3.params.solver_iterations = 3
    e3 = Engine(local)
    e3.set_params(w3.params)
    e3.reset(w3.n, w3.scene, w3.desc)
    e3.set_graph_mode(True)
    for _ in range(args.warmup):
        e3.step(w3.dt, stream)
    dist_barrier(world)
    torch.cuda.synchronize(dev)
    k3_ms = 0.0
    for _ in range(args.steps):
        flush_l2()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        e3.step(w3.dt, stream)
        s1.record(stream)
        s1.synchronize()
        k3_ms += s0.elapsed_time(s1)
    e3.check_errors()
    e3.close()
    k3_ms = dist_max(k3_ms, world) / args.steps
    three = {"solver_iterations": 3, "ms_per_step": round(k3_ms, 5),
             "algorithmic_bytes": step_bytes(n, cells, 3),
             "step_frac": round(step_bytes(n, cells, 3) / (k3_ms * 1e-3) / 1e9 / peak, 4),
             "l2": "flushed between timed steps"}

    batched = None if args.no_batch else run_batched(args, world, rank, local, stream, flush_l2)
    adjoint = None if args.no_adjoint else run_adjoint(args, world, rank, local, stream)

    if rank != 0:
        return None
    line = {
        "metric": METRIC, "value": round(value, 5), "unit": "ms/step", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic: seeded jittered lattice ({w.name}), no dataset",
        "config": bench_config(w, world), "mode": "CUDA graph replay of the step",
        "ms_per_step_hot_l2": round(hot_ms, 5),
        "steps_per_s": round(1000.0 / ms_per_step, 2),
        "particle_steps_per_s": round(n * world * 1000.0 / ms_per_step, 1),
        "roofline": roofline, "kernels": kernels,
        "kernels_timing": "CUDA events as event nodes of the step's graph, L2 flushed before each step",
        "three_iterations": three,
        "e2e": {"value": round(e2e_value, 5), "unit": "ms/step", "h2d_bytes_per_step": 32 * n,
                "d2h_bytes_per_step": 32 * n, "steps": e2e_steps,
                "start": "the timed region's start state: the same steps as value",
                "same_final_state": e2e_same},
        "gpu_launches": int(lib.mp_step_launch_count(k_it)) * args.steps
                        + int(lib.mp_step_launch_count(3)) * args.steps,
        "clocks": clk.summary(),
    }
    if batched is not None:
        line["batched"] = batched
        line["gpu_launches"] += batched["launches_timed"]
    if adjoint is not None:
        line["adjoint"] = adjoint
        line["gpu_launches"] += adjoint.pop("launches_timed")
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, args, start_state, args.warmup)
    return line


def run_adjoint(args, world, rank, local, stream) -> dict:
    """Cost of the gradient relative to the forward rollout it differentiates:
    backward ms (the recomputation of every 10-step segment with the steps
    recorded, and the adjoint kernels) / forward ms (the rollout with its
    checkpoints), both CUDA-event timed on the engine's stream, max over
    ranks.  Workloads: the 97,336-particle differentiable cube drop (60
    steps; loss = mean squared distance to the final positions of a seeded
    run with initial velocities N(0, 0.5 m/s); gradients w.r.t. every initial
    velocity and s_corr k) at the benchmark parameters and at the
    well-conditioned ones the gradient checks use; and the 32-scene batched
    sphere drop (40 steps, all scenes in one launch per step; gradients
    w.r.t. every scene's sphere state and radius)."""
    import torch

    from mtlphys_b200 import _abi, configs
    from mtlphys_b200.batch import Batch
    from mtlphys_b200.ensemble import shard_workload

    reps = max(1, min(3, args.steps))
    out = {}
    launches = 0

    def time_rollout(b, steps, every, pos0, vel0, target, reset=None):
        nonlocal launches
        n = b.particle_count()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        fwd = bwd = 0.0
        for r in range(reps + 1):  # the first repetition warms up
            if reset is not None:
                reset()
            with torch.cuda.stream(stream):
                b.tensor(_abi.MP_BUF_POSITIONS).copy_(pos0)
                b.tensor(_abi.MP_BUF_VELOCITIES).copy_(vel0)
            dist_barrier(world)
            torch.cuda.synchronize()
            ev[0].record(stream)
            b.rollout_forward(steps, every, stream)
            ev[1].record(stream)
            with torch.cuda.stream(stream):  # dL/dx(T) of the mean squared distance
                g = (b.tensor(_abi.MP_BUF_POSITIONS) - target) * (2.0 / max(n, 1))
                g[:, 3] = 0.0
            ev[2].record(stream)
            b.rollout_backward(g, None, stream)
            ev[3].record(stream)
            torch.cuda.synchronize()
            if r > 0:
                fwd += ev[0].elapsed_time(ev[1])
                bwd += ev[2].elapsed_time(ev[3])
                launches += steps + b.rollout_launch_count(steps)
        if b.check_errors():
            raise RuntimeError("device error in the adjoint leg")
        fwd = dist_max(fwd / reps, world)
        bwd = dist_max(bwd / reps, world)
        return {"forward_ms": round(fwd, 3), "backward_ms": round(bwd, 3), "ratio": round(bwd / fwd, 3)}

    def target_of(b, steps, pos0, vel_t):
        with torch.cuda.stream(stream):
            b.tensor(_abi.MP_BUF_POSITIONS).copy_(pos0)
            b.tensor(_abi.MP_BUF_VELOCITIES).copy_(vel_t)
        for _ in range(steps):
            b.step(stream)
        torch.cuda.synchronize()
        return b.tensor(_abi.MP_BUF_POSITIONS).clone()

    dev = torch.device("cuda", local)
    gen = torch.Generator(device=dev)
    for label, k, cfm in (("benchmark_params", None, None), ("conditioned", 1e-4, 1e5)):
        w = configs.diff_cube(side=46, steps=60)
        if k is not None:
            w.params.scorr_k = k
            w.params.epsilon = cfm
        b = Batch(local)
        b.reset([w.n], [w.params], [w.dt], [w.scene], [w.desc])
        b.set_graph_mode(True)
        pos0 = b.tensor(_abi.MP_BUF_POSITIONS).clone()
        gen.manual_seed(configs.SEED_BASE + 2)
        vel_t = torch.zeros((w.n, 4), device=dev)
        vel_t[:, :3] = torch.randn((w.n, 3), device=dev, generator=gen) * 0.5
        target = target_of(b, w.steps, pos0, vel_t)
        t = time_rollout(b, w.steps, 10, pos0, torch.zeros_like(vel_t), target)
        out[label] = {"workload": "diff_cube", "particles": w.n, "steps": w.steps, "checkpoint_every": 10,
                      "scorr_k": float(w.params.scorr_k), "epsilon": float(w.params.epsilon), **t}
        b.close()
    full = configs.batch_spheres()
    ws, _ = shard_workload(full, rank, world)
    b = Batch(local)
    b.reset(ws.counts, ws.params, ws.dts, ws.scenes, ws.descs)
    b.set_graph_mode(True)
    pos0 = b.tensor(_abi.MP_BUF_POSITIONS).clone()
    zero = torch.zeros_like(pos0)
    target = target_of(b, ws.steps, pos0, zero)  # spheres from their seeded starts
    def spheres_start():  # the optimised run: each sphere's initial speed halved
        for s, sph in enumerate(ws.spheres):
            b.set_sphere(s, sph[:3], (sph[3], 0.5 * sph[4], sph[5]), sph[6])

    t = time_rollout(b, ws.steps, 10, pos0, zero, target, spheres_start)
    out["batched_sphere_drop"] = {"workload": "batch_spheres", "scenes": len(full.counts),
                                  "particles": full.n, "steps": ws.steps, "checkpoint_every": 10, **t}
    b.close()
    out["what"] = ("backward (recompute of each checkpointed segment with the steps recorded + adjoint "
                   "kernels) / forward rollout with checkpoints")
    out["launches_timed"] = launches
    return out


def run_batched(args, world, rank, local, stream, flush_l2) -> dict:
    """The batched ensemble (256 cube drops, 2,000-64,000 particles each,
    log-uniform): scenes x steps / s with every scene advanced by one
    persistent launch per step (CUDA graph, autotuned launch shape) against
    the same kernel launched scene by scene (CUDA graph, its own autotuned
    shape), from the same start state; the two final states must be
    bit-identical.  With N ranks the scenes are bin-packed over the ranks by
    particle count and the time is the max over ranks."""
    import numpy as np
    import torch

    from mtlphys_b200 import configs
    from mtlphys_b200.batch import Batch
    from mtlphys_b200.ensemble import shard_workload

    full = configs.batch_cubes()
    w, _ = shard_workload(full, rank, world)
    steps = max(3, min(args.steps, args.batch_steps))
    b = Batch(local)
    res, finals = {}, {}
    for mode in ("batched", "serial"):
        b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        b.set_serial(mode == "serial")
        b.set_graph_mode(False)
        tune = b.autotune(steps=2)
        b.set_graph_mode(True)
        for _ in range(args.warmup):
            b.step(stream)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        dist_barrier(world)
        torch.cuda.synchronize()
        for i in range(steps):
            flush_l2()
            starts[i].record(stream)
            b.step(stream)
            ends[i].record(stream)
        torch.cuda.synchronize()
        dist_barrier(world)
        if b.check_errors():
            raise RuntimeError(f"device error in the {mode} batch run")
        ms = dist_max(sum(s.elapsed_time(t) for s, t in zip(starts, ends)) / steps, world)
        finals[mode] = (b.positions(), b.velocities())
        launches = 1 if mode == "batched" else sum(1 for c in w.counts if c > 0)
        res[mode] = {"ms_per_step": round(ms, 4),
                     "scenes_per_s": round(len(full.counts) * 1000.0 / ms, 1),
                     "launch": {"block": tune["block"], "blocks_per_sm": tune["blocks_per_sm"]},
                     "launches_per_step": launches}
    ranges = [b.scene_range(s) for s in range(len(w.counts))]
    b.close()

    # the single-scene engine (the multi-kernel step: 5 + 2K launches in a
    # CUDA graph), one engine per scene, stepped one scene after another
    from mtlphys_b200 import Engine

    engines = []
    for s in range(len(w.counts)):
        e = Engine(local)
        e.set_params(w.params[s])
        e.reset(w.counts[s], w.scenes[s], w.descs[s])
        e.set_graph_mode(True)
        engines.append(e)
    for _ in range(args.warmup):
        for s, e in enumerate(engines):
            e.step(w.dts[s], stream)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    dist_barrier(world)
    torch.cuda.synchronize()
    for i in range(steps):
        flush_l2()
        starts[i].record(stream)
        for s, e in enumerate(engines):
            e.step(w.dts[s], stream)
        ends[i].record(stream)
    torch.cuda.synchronize()
    dist_barrier(world)
    ms = dist_max(sum(s.elapsed_time(t) for s, t in zip(starts, ends)) / steps, world)
    same_engine = True
    for s, e in enumerate(engines):
        f, n = ranges[s]
        same_engine &= bool(np.array_equal(e.positions(), finals["batched"][0][f:f + n]))
        e.close()
    k_it = int(w.params[0].solver_iterations) if w.params else 0
    per_scene = 5 + 2 * k_it
    res["engines"] = {"ms_per_step": round(ms, 4), "scenes_per_s": round(len(full.counts) * 1000.0 / ms, 1),
                      "launches_per_step": per_scene * sum(1 for c in w.counts if c > 0),
                      "what": "one single-scene engine per scene (multi-kernel step in a CUDA graph), "
                              "stepped one after another"}

    same = all(np.array_equal(x, y) for x, y in zip(finals["batched"], finals["serial"]))
    return {"workload": full.describe(), "steps": steps, "warmup": args.warmup,
            "batched": res["batched"], "serial": res["serial"], "engines": res["engines"],
            "speedup": round(res["serial"]["ms_per_step"] / res["batched"]["ms_per_step"], 3),
            "speedup_vs_engines": round(res["engines"]["ms_per_step"] / res["batched"]["ms_per_step"], 3),
            "bit_identical": bool(dist_max(0.0 if same else 1.0, world) == 0.0),
            "bit_identical_engines": bool(dist_max(0.0 if same_engine else 1.0, world) == 0.0),
            "l2": "flushed between timed steps", "mode": "CUDA graph replay",
            "launches_timed": steps * (res["batched"]["launches_per_step"] + res["serial"]["launches_per_step"]
                                       + res["engines"]["launches_per_step"])}


def read_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel:
                    return int(float(parts[1]))
    except OSError:
        pass
    return None


def cpu_baseline(w, args, start, first_step) -> dict:
    """The FP64 oracle on the host cores, a bounded sample of the workload:
    the first of the timed region's steps, from its start state."""
    import numpy as np

    from oracle import oracle as O

    pos, vel = start
    O.set_threads(0)
    steps = 0
    t0 = time.perf_counter()
    while steps < args.cpu_steps and (time.perf_counter() - t0) < args.cpu_budget_s:
        o = O.step(w.params, w.dt, pos, vel)
        pos = np.concatenate([o["pos"], np.ones((w.n, 1))], axis=1).astype(np.float32)
        vel = np.concatenate([o["vel"], np.zeros((w.n, 1))], axis=1).astype(np.float32)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": round(dt * 1000.0 / steps, 2), "unit": "ms/step", "cores": O.threads(),
            "kind": "port",
            "sample": f"steps {first_step}-{first_step + steps - 1} of the {w.name} workload ({w.n} particles; "
                      f"the first {steps} timed steps, from their start state), FP64 oracle"}


# ---- reference arm ----------------------------------------------------------------------
L2_NOTE = "flushed between timed steps (256 MiB write outside the timed region)"


def bench_config(w, world: int) -> dict:
    """The `config` both arms print: the workload with its sizes, how the work
    is spread, and how caches are flushed between timed steps."""
    return {**w.describe(), "parallelism": "replicas" if world > 1 else "single", "l2": L2_NOTE}


def run_reference(args, world, rank) -> dict | None:
    """The reference's own CPU implementation of the step on the host cores:
    its compute shaders (engine/shaders/*.metal) compiled as C++ into
    oracle/_ref and dispatched in Engine::step order (engine/src/Engine.cpp:
    685-811), OpenMP over all host cores; the FP64 oracle port where _ref was
    not built.  Same workload, warm-up and timed steps as our arm; nothing of
    the product package is imported or loaded (the workload comes from
    oracle/params.py, which a CPU test pins to the product's).  The shaders
    hard-code s_corr k = 1e-4 (Constraints.metal:158); the config says so."""
    if rank != 0:
        return None
    import numpy as np

    from oracle import oracle as O
    from oracle import params as OP

    w = OP.WORKLOADS[args.workload]()
    cores = os.cpu_count() or 1
    pos = O.seed_scene(w.params, w.scene, w.n, w.desc)
    vel = np.zeros_like(pos)
    config = bench_config(w, world)
    if O.has_ref():
        kind = "reference"
        O.ref_set_threads(cores)
        config["scorr_k"] = 1e-4

        def step(pos, vel):
            o = O.ref_step(w.params, w.dt, pos, vel)
            return o["pos"], o["vel"]
        what = ("the reference's compute shaders (engine/shaders/*.metal) compiled as C++, "
                "dispatched in Engine::step order; s_corr k is the shaders' hard-coded 1e-4")
    else:
        kind = "port"
        O.set_threads(cores)

        def step(pos, vel):
            o = O.step(w.params, w.dt, pos, vel)
            return (np.concatenate([o["pos"], np.ones((w.n, 1))], axis=1).astype(np.float32),
                    np.concatenate([o["vel"], np.zeros((w.n, 1))], axis=1).astype(np.float32))
        what = "FP64 oracle port (the reference's shaders were not compiled here)"
    flush = np.empty(L2_FLUSH_BYTES, np.uint8)
    for _ in range(args.warmup):
        pos, vel = step(pos, vel)
    total = 0.0
    for i in range(args.steps):
        flush.fill(i & 0xFF)  # evict the host caches, outside the timed region
        t0 = time.perf_counter()
        pos, vel = step(pos, vel)
        total += time.perf_counter() - t0
    ms = total * 1000.0 / args.steps
    return {
        "metric": METRIC, "value": round(ms, 3), "unit": "ms/step", "impl": "reference",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": f"synthetic: seeded jittered lattice ({w.name}), no dataset",
        "config": config,
        "cpu_baseline": {"value": round(ms, 3), "unit": "ms/step", "cores": cores, "kind": kind,
                         "sample": f"{args.steps} whole steps of {w.name} ({w.n} particles) after "
                                   f"{args.warmup} warm-up steps: {what}"},
        "e2e": {"value": round(ms, 3), "unit": "ms/step", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


# ---- fixed short runs for profilers ---------------------------------------------------
def run_profile(which: str) -> str:
    """One workload run once, a short fixed sequence of launches for a
    profiler to capture: `step` (1M dam break, 3 steps), `batch` (256 cube
    drops, 3 batched steps), `adjoint` (97K cube, 20-step rollout + gradient),
    `adjoint_spheres` (32 sphere drops, 10-step rollout + gradient; `_small`:
    4 of them, for captures that save and restore device memory),
    `render` (1M dam break, 3 frames at 1280x720).  Returns one line with its
    CUDA-event time; not a benchmark value."""
    import torch

    from mtlphys_b200 import Engine, _abi, configs
    from mtlphys_b200.batch import Batch

    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    if which == "step":
        w = configs.dam_break()
        e = Engine(0)
        e.set_params(w.params)
        e.reset(w.n, w.scene, w.desc)
        ms = timed(lambda: [e.step(w.dt, stream) for _ in range(3)])
        e.check_errors()
        return f"step: 3 steps of {w.n} particles in {ms:.3f} ms"
    if which == "batch":
        w = configs.batch_cubes()
        b = Batch(0)
        b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        ms = timed(lambda: [b.step(stream) for _ in range(3)])
        b.check_errors()
        return f"batch: 3 steps of {len(w.counts)} scenes ({w.n} particles) in {ms:.3f} ms"
    if which == "adjoint":
        w = configs.diff_cube(side=46, steps=20)
        b = Batch(0)
        b.reset([w.n], [w.params], [w.dt], [w.scene], [w.desc])
        g = torch.zeros((w.n, 4), device="cuda")
        g[:, 1] = 1.0 / w.n

        def go():
            b.rollout_forward(w.steps, 10, stream)
            b.rollout_backward(g, None, stream)

        ms = timed(go)
        b.check_errors()
        return f"adjoint: {w.steps}-step rollout + gradient of {w.n} particles in {ms:.3f} ms"
    if which in ("adjoint_spheres", "adjoint_spheres_small"):
        w = configs.batch_spheres(num=32 if which == "adjoint_spheres" else 4, steps=10)
        b = Batch(0)
        b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        g = torch.zeros((w.n, 4), device="cuda")
        g[:, 1] = 1.0 / w.n

        def go():
            b.rollout_forward(w.steps, 10, stream)
            b.rollout_backward(g, None, stream)

        ms = timed(go)
        b.check_errors()
        return (f"{which}: {w.steps}-step rollout + gradient of {len(w.counts)} scenes "
                f"({w.n} particles) in {ms:.3f} ms")
    if which == "render":
        w = configs.dam_break()
        e = Engine(0)
        e.set_params(w.params)
        e.reset(w.n, w.scene, w.desc)
        for _ in range(20):
            e.step(w.dt, stream)
        rp = _abi.default_render_params(width=1280, height=720)
        rp.eye[:] = [14.0, 8.0, 15.0]
        rp.target[:] = [4.3, 2.0, 4.3]
        ms = timed(lambda: [e.render(rp, stream) for _ in range(3)])
        return f"render: 3 frames of {w.n} particles at 1280x720 in {ms:.3f} ms"
    raise SystemExit(f"unknown profile workload {which!r}: step, batch, adjoint or render")


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["dam_break", "cube_drop"], default="dam_break")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=15)
    ap.add_argument("--cpu-budget-s", type=float, default=60.0)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-ensemble leg")
    ap.add_argument("--batch-steps", type=int, default=10, help="timed steps of the batched leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost leg")
    ap.add_argument("--profile", choices=["step", "batch", "adjoint", "adjoint_spheres", "adjoint_spheres_small", "render"],
                    help="run one fixed short workload for a profiler and exit (no bench line)")
    args = ap.parse_args()
    if args.profile:
        print(run_profile(args.profile), flush=True)
        return
    if args.warmup < 3 and args.impl == "ours":
        ap.error("--warmup must be >= 3")

    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, world, rank)
    else:
        world, rank, local = dist_setup(args.gpus)
        line = run_ours(args, world, rank, local)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
