"""Differentiable PBF rollouts for torch.

``Rollout`` is a ``torch.autograd.Function`` over the batch engine's C ABI:
its forward pass loads the initial state and the differentiable parameters
into a ``Batch`` and calls ``mp_batch_rollout_forward`` (the same steps as
``Batch.step``, with a checkpoint every ``checkpoint_every`` steps); its
backward pass calls ``mp_batch_rollout_backward``, which recomputes each
segment between checkpoints with the steps recorded and runs the adjoint
kernels over it in reverse.  The neighbour topology and the clamp states of
every step are held fixed.  Gradients flow to the initial positions and
velocities of every particle, each scene's s_corr strength k, and each
scene's initial sphere center, velocity and radius.  Scalar reductions (the
per-scene parameter gradients) are FP64 on the GPU; everything else is FP32.
"""
from __future__ import annotations

import torch

from . import _abi
from ._abi import MP_BUF_POSITIONS, MP_BUF_VELOCITIES


class Rollout(torch.autograd.Function):
    """(pos_T, vel_T) = rollout(pos0, vel0, scorr_k, sphere_center, sphere_velocity, sphere_radius).

    pos0, vel0: (N, 4) float32 CUDA tensors (w ignored) for all scenes'
    particles in batch order; scorr_k: (S,) per-scene s_corr k; the sphere
    tensors ((S, 3), (S, 3), (S,)) or None when no scene is a sphere drop."""

    @staticmethod
    def forward(ctx, batch, steps: int, checkpoint_every: int, pos0, vel0, scorr_k, sphere_center,
                sphere_velocity, sphere_radius):
        stream = torch.cuda.current_stream(pos0.device)
        batch.tensor(MP_BUF_POSITIONS).copy_(pos0)
        batch.tensor(MP_BUF_VELOCITIES).copy_(vel0)
        S = batch.scene_count()
        if scorr_k is not None:
            ks = scorr_k.detach().double().cpu().tolist()
            for s in range(S):
                p = batch.params(s)
                if p.scorr_k != ks[s]:
                    p.scorr_k = ks[s]
                    batch.set_params(s, p)
        if sphere_center is not None:
            cs = sphere_center.detach().double().cpu().tolist()
            vs = sphere_velocity.detach().double().cpu().tolist()
            rs = sphere_radius.detach().double().cpu().tolist()
            for s in range(S):
                batch.set_sphere(s, cs[s], vs[s], rs[s])
        batch.rollout_forward(steps, checkpoint_every, stream)
        ctx.batch = batch
        ctx.k_like = None if scorr_k is None else (scorr_k.dtype, scorr_k.device)
        ctx.sph_like = None if sphere_center is None else (sphere_center.dtype, sphere_center.device)
        return batch.tensor(MP_BUF_POSITIONS).clone(), batch.tensor(MP_BUF_VELOCITIES).clone()

    @staticmethod
    def backward(ctx, gpos, gvel):
        stream = torch.cuda.current_stream()
        prep = lambda g: None if g is None else g.to(torch.float32).contiguous()
        dpos0, dvel0, dscene = ctx.batch.rollout_backward(prep(gpos), prep(gvel), stream)
        dk = dc = dv = dr = None
        if ctx.k_like is not None:
            dtype, device = ctx.k_like
            dk = dscene[:, _abi.MP_GRAD_SCORR_K].to(device=device, dtype=dtype)
        if ctx.sph_like is not None:
            dtype, device = ctx.sph_like
            part = lambda a, b: dscene[:, a:b].to(device=device, dtype=dtype)
            dc = part(_abi.MP_GRAD_CENTER, _abi.MP_GRAD_CENTER + 3)
            dv = part(_abi.MP_GRAD_VELOCITY, _abi.MP_GRAD_VELOCITY + 3)
            dr = dscene[:, _abi.MP_GRAD_RADIUS].to(device=device, dtype=dtype)
        return None, None, None, dpos0, dvel0, dk, dc, dv, dr


def rollout(batch, steps: int, pos0, vel0, scorr_k=None, sphere=None, checkpoint_every: int = 10):
    """Differentiable rollout of every scene of `batch`.  sphere: None or a
    (center (S, 3), velocity (S, 3), radius (S,)) tuple.  Returns the final
    positions and velocities, (N, 4) each."""
    c, v, r = sphere if sphere is not None else (None, None, None)
    return Rollout.apply(batch, int(steps), int(checkpoint_every), pos0, vel0, scorr_k, c, v, r)
