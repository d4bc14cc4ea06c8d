"""Ensembles of independent boxes across GPUs (one process per GPU).

Boxes never interact, so sharding an ensemble needs no data-path collective:
each rank owns a subset of the boxes, steps them in its own context (one
persistent set of launches over all its boxes), and only the per-box
diagnostics travel, as a host-side gather at the end.

Boxes are assigned by longest-processing-time-first on the expected pair work
of a box (particles x mean neighbours): boxes sorted by cost, each given to the
least-loaded rank (ties to the lower rank), which is deterministic and within
4/3 of the optimal makespan.
"""
from __future__ import annotations

import heapq

import numpy as np

from . import abi


def lpt_partition(costs, world):
    """Rank of every box: greedy longest-processing-time on `costs`."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda b: (-costs[b], b))
    heap = [(0.0, r) for r in range(world)]
    owner = np.zeros(len(costs), dtype=np.int64)
    for b in order:
        load, r = heapq.heappop(heap)
        owner[b] = r
        heapq.heappush(heap, (load + costs[b], r))
    return owner


def shard(workload, rank, world, neighbours_per_particle=57.0):
    """The sub-ensemble of `rank`: its boxes renumbered 0..k-1, their particles,
    and the global ids of its boxes."""
    s = workload.species[abi.SPECIES_DEFAULT]
    nbox = len(workload.boxes)
    counts = np.bincount(s.box_id, minlength=nbox)
    owner = lpt_partition(counts * neighbours_per_particle, world)
    mine = np.flatnonzero(owner == rank)
    remap = -np.ones(nbox, dtype=np.int64)
    remap[mine] = np.arange(len(mine))
    sel = np.isin(s.box_id, mine)
    sub = abi.Species(int(sel.sum()))
    for c in abi.COLUMNS:
        setattr(sub, c, np.ascontiguousarray(getattr(s, c)[..., sel]))
    sub.box_id = np.ascontiguousarray(remap[s.box_id[sel]].astype(np.int32))
    return [workload.boxes[b] for b in mine], sub, mine


def gather_diagnostics(local, box_ids, nbox, group=None):
    """Per-box diagnostics of every rank, in global box order, on rank 0 (host gather)."""
    import torch.distributed as dist
    payload = list(zip([int(b) for b in box_ids], local))
    if not dist.is_available() or not dist.is_initialized():
        merged = payload
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, payload, group=group)
        merged = [x for p in parts for x in p]
    out = [None] * nbox
    for b, d in merged:
        out[b] = d
    return out


def run_shard(workload, rank, world, steps, device=0, make_context=None):
    """Step this rank's boxes `steps` times; returns (box ids, per-box diagnostics)."""
    boxes, sub, mine = shard(workload, rank, world)
    if len(mine) == 0:
        return mine, []
    if make_context is None:
        import spearhed_b200 as sb
        params = workload.params
        params.device = device
        ctx = sb.Context(params, boxes)
    else:
        ctx = make_context(workload.params, boxes)
    ctx.set_species(abi.SPECIES_DEFAULT, sub)
    ctx.step(steps)
    diags = ctx.ensemble_reduce(len(boxes))
    ctx.close()
    return mine, diags
