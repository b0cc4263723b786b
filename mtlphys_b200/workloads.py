"""Run one workload of the engine once, for profilers and quick checks:

    python -m mtlphys_b200.workloads step      # 1M dam break, 3 steps
    python -m mtlphys_b200.workloads batch     # 256 cube drops, 3 batched steps
    python -m mtlphys_b200.workloads adjoint   # 97K cube, 20-step rollout + gradient
    python -m mtlphys_b200.workloads render    # 1M dam break, 3 frames at 1280x720

Each prints one line with its CUDA-event time.  The benchmark proper is
bench.py; this exists so that a profiler can capture a short, fixed
sequence of launches.
"""
from __future__ import annotations

import sys


def _time(fn, stream):
    import torch

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run(which: str) -> str:
    import torch

    from . import Engine, _abi, configs
    from .batch import Batch

    stream = torch.cuda.current_stream()
    if which == "step":
        w = configs.dam_break()
        e = Engine(0)
        e.set_params(w.params)
        e.reset(w.n, w.scene, w.desc)
        ms = _time(lambda: [e.step(w.dt, stream) for _ in range(3)], stream)
        e.check_errors()
        return f"step: 3 steps of {w.n} particles in {ms:.3f} ms"
    if which == "batch":
        w = configs.batch_cubes()
        b = Batch(0)
        b.reset(w.counts, w.params, w.dts, w.scenes, w.descs)
        ms = _time(lambda: [b.step(stream) for _ in range(3)], stream)
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

        ms = _time(go, stream)
        b.check_errors()
        return f"adjoint: {w.steps}-step rollout + gradient of {w.n} particles in {ms:.3f} ms"
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
        ms = _time(lambda: [e.render(rp, stream) for _ in range(3)], stream)
        return f"render: 3 frames of {w.n} particles at 1280x720 in {ms:.3f} ms"
    raise SystemExit(f"unknown workload {which!r}: step, batch, adjoint or render")


if __name__ == "__main__":
    print(run(sys.argv[1] if len(sys.argv) > 1 else "step"), flush=True)
