"""Batches over several GPUs: one process per GPU, complexes sharded by size.

A single reduction does not shard (one pivot table, arbitrary column
dependencies), but independent complexes do.  Every rank takes a share of the
complexes - assigned largest first to the rank with the fewest columns so far,
the same assignment on every rank, with no communication - reduces its share
as one batch on its own GPU, and the results are gathered on the host of one
rank.  Nothing crosses between GPUs on the data path; the only collective is
the final gather of host arrays over torch.distributed (gloo or nccl object
collectives).
"""
from __future__ import annotations

import heapq

import numpy as np


def local_device() -> int:
    """This process's GPU under one process per GPU: LOCAL_RANK (set by torchrun),
    else the current CUDA device once CUDA is initialised, else 0."""
    import os

    if "LOCAL_RANK" in os.environ:
        return int(os.environ["LOCAL_RANK"])
    try:
        import torch

        if torch.cuda.is_available() and torch.cuda.is_initialized():
            return torch.cuda.current_device()
    except ImportError:
        pass
    return 0


def shard(ncols, world: int) -> list:
    """Complex indices of each rank (largest complexes first, to the least loaded rank)."""
    order = sorted(range(len(ncols)), key=lambda i: (-int(ncols[i]), i))
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(ncols[i]), r))
    return [sorted(p) for p in parts]


def _reduce_local(mats, params, device):
    from .engine import Engine

    if not mats:
        return []
    with Engine(device) as e:
        e.load_batch(mats)
        e.reduce(params)
        return e.batch_results()


def reduce_batch(mats, params, group=None, device: int | None = None, dst: int = 0, reduce_fn=None):
    """Reduces `mats` (the same list on every rank) across the ranks of `group`.

    Returns [(pairs, essentials)] in input order on rank `dst`, None elsewhere.
    reduce_fn(local_mats, params, device) replaces the single-GPU batch reduction
    (the default runs the engine on `device`).  `device` defaults to this
    process's GPU (see local_device); with the nccl backend, call
    torch.cuda.set_device(local_rank) first, as the object gather needs it.
    """
    import torch.distributed as dist

    device = local_device() if device is None else device

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = shard([m.ncols for m in mats], world)
    mine = parts[rank]
    res = (reduce_fn or _reduce_local)([mats[i] for i in mine], params, device)
    payload = [(i, np.asarray(p), np.asarray(e)) for i, (p, e) in zip(mine, res)]
    gathered = [None] * world if rank == dst else None
    dist.gather_object(payload, gathered, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * len(mats)
    for part in gathered:
        for i, p, e in part:
            out[i] = (p, e)
    return out


def _size_of(req) -> int:
    """Work estimate of a point-cloud or field request: its vertex count."""
    kind, data = req[0], req[1]
    return int(np.asarray(data).shape[0]) if kind == "rips" else int(np.asarray(data).size)


def _reduce_built_local(reqs, params, device):
    from .engine import Engine

    out = []
    if not reqs:
        return out
    with Engine(device) as e:
        for req in reqs:
            if req[0] == "rips":
                e.load_rips(req[1], req[2], req[3])
            else:
                e.load_lowerstar(req[1], req[2])
            e.reduce(params)
            out.append((e.pairs(), e.essentials()))
    return out


def reduce_requests(reqs, params, group=None, device: int | None = None, dst: int = 0, reduce_fn=None):
    """Point clouds and fields across the ranks of `group`: each rank builds (on its GPU) and
    reduces its share.  reqs: ("rips", points [npts, D], radius, maxdim) or ("lowerstar",
    field [gz, gy, gx], maxdim), the same list on every rank.  Returns [(pairs, essentials)]
    in input order on rank `dst` (indices of the built matrices), None elsewhere;
    reduce_fn(local_reqs, params, device) replaces the single-GPU loop.  `device`
    defaults to this process's GPU, as for reduce_batch."""
    import torch.distributed as dist

    device = local_device() if device is None else device

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = shard([_size_of(r) for r in reqs], world)
    mine = parts[rank]
    res = (reduce_fn or _reduce_built_local)([reqs[i] for i in mine], params, device)
    payload = [(i, np.asarray(p), np.asarray(e)) for i, (p, e) in zip(mine, res)]
    gathered = [None] * world if rank == dst else None
    dist.gather_object(payload, gathered, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * len(reqs)
    for part in gathered:
        for i, p, e in part:
            out[i] = (p, e)
    return out

