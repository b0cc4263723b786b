"""Sharding a batch of independent scenes over the ranks of a job.

A single PBF scene does not shard (a domain split would need halo exchanges
of width h twice per solver iteration), but a batch of independent scenes
does: every rank advances its own subset in one persistent launch per step,
with no data-path collective.  The only exchange is of per-scene scalars
(losses, parameter gradients) at the end of a rollout, gathered in FP64.
"""
from __future__ import annotations

import heapq


def partition_scenes(counts, world: int) -> list[list[int]]:
    """Greedy longest-processing-time bin-packing of scenes over `world` ranks
    by particle count: scenes in decreasing count (ties by index) go to the
    rank with the fewest particles so far (ties by rank).  Deterministic, so
    every rank computes the same partition without communicating.  Each
    rank's list is in increasing scene index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(counts)), key=lambda s: (-int(counts[s]), s))
    heap = [(0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for s in order:
        load, r = heapq.heappop(heap)
        shards[r].append(s)
        heapq.heappush(heap, (load + int(counts[s]), r))
    return [sorted(x) for x in shards]


def shard_workload(w, rank: int, world: int):
    """The scenes of batch workload `w` that rank `rank` advances, as a new
    workload of the same kind, plus their indices in `w`."""
    idx = partition_scenes(w.counts, world)[rank]
    pick = lambda xs: None if xs is None else [xs[i] for i in idx]
    sub = type(w)(w.name, pick(w.counts), pick(w.params), pick(w.dts), pick(w.scenes), pick(w.descs),
                  w.steps, pick(w.spheres))
    return sub, idx


def gather_scene_scalars(values, idx, nscenes: int, world: int):
    """All-gather per-scene FP64 scalars (one value per scene this rank owns,
    scene indices `idx`) into a length-`nscenes` list on every rank.  Uses
    the default process group (NCCL on GPUs, gloo on CPU) when one is
    initialised, a single rank included; without one, world must be 1."""
    import torch
    import torch.distributed as dist

    out = [0.0] * nscenes
    if world == 1 and not (dist.is_available() and dist.is_initialized()):
        for i, v in zip(idx, values):
            out[i] = float(v)
        return out

    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    local = torch.zeros(nscenes, dtype=torch.float64, device=dev)
    mask = torch.zeros(nscenes, dtype=torch.float64, device=dev)
    for i, v in zip(idx, values):
        local[i] = float(v)
        mask[i] = 1.0
    parts = [torch.empty_like(local) for _ in range(world)]
    masks = [torch.empty_like(mask) for _ in range(world)]
    dist.all_gather(parts, local)
    dist.all_gather(masks, mask)
    for p, m in zip(parts, masks):
        pm, mm = p.cpu().tolist(), m.cpu().tolist()
        for s in range(nscenes):
            if mm[s]:
                out[s] = pm[s]
    return out
