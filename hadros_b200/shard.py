"""Multi-GPU sharding of image work: one process per GPU, no data-path
collective.

Pixels and cameras are independent, so a scan over N GPUs is a partition of
its work items: whole cameras for scans of many cameras (longest-first
greedy balance by pixel count), or contiguous pixel ranges of one image.
Each rank traces its share with its own context; results meet on rank 0
only at the end (``gather_to_root``), and the only other collective is the
timing reduction (``max_over_ranks``).  The tracer is a parameter, so the
partition and gather logic is exercised on CPU with the gloo backend.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence

import numpy as np


def partition_cameras(costs: Sequence[float], world: int) -> list[list[int]]:
    """Longest-processing-time-first: cameras sorted by cost, each given to the
    least loaded rank.  Returns the camera indices of every rank, each list in
    ascending camera order."""
    if world <= 0:
        raise ValueError("world must be positive")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts: list[list[int]] = [[] for _ in range(world)]
    for idx in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        parts[r].append(idx)
        heapq.heappush(heap, (load + float(costs[idx]), r))
    return [sorted(p) for p in parts]


def pixel_range(n_pixels: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [start, stop) of an image's pixels for `rank`."""
    base, extra = divmod(n_pixels, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather_to_root(obj, dist, rank: int, world: int):
    """List of every rank's object on rank 0 (None elsewhere)."""
    if dist is None or world == 1:
        return [obj]
    out = [None] * world if rank == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def init_from_env(backend: str | None = None, timeout_s: int = 1800):
    """(dist, rank, world, local_rank) of a torchrun launch; (None, 0, 1, 0)
    without one.  backend None: nccl when CUDA is available, else gloo."""
    import os
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank, local = int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return None, 0, 1, 0
    import datetime

    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return dist, rank, world, local


def max_over_ranks(x: float, dist, device=None) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_scan(cams: Sequence, trace: Callable[[list], list], dist=None, rank: int = 0,
             world: int = 1, costs: Sequence[float] | None = None) -> list | None:
    """Trace `cams` (or any work items) across ranks: this rank runs its
    partition with `trace(list_of_items) -> list_of_results`; rank 0 returns
    the results in item order, other ranks return None.  Items are balanced
    by `costs` (default: the cameras' pixel counts)."""
    if costs is None:
        costs = [float(c.nx) * float(c.ny) for c in cams]
    parts = partition_cameras(costs, world)
    mine = parts[rank]
    local = trace([cams[i] for i in mine]) if mine else []
    gathered = gather_to_root(list(zip(mine, local)), dist, rank, world)
    if rank != 0:
        return None
    res: list = [None] * len(cams)
    for part in gathered:
        for i, r in part:
            res[i] = r
    return res


def run_image_sharded(p, trace_pixels: Callable[[object, np.ndarray], dict], dist=None,
                      rank: int = 0, world: int = 1) -> dict | None:
    """One image split into contiguous pixel ranges; `trace_pixels(p, ids)`
    traces a pixel list.  Rank 0 returns the whole image (pixel order)."""
    P = int(p.nx) * int(p.ny)
    a, b = pixel_range(P, rank, world)
    local = trace_pixels(p, np.arange(a, b, dtype=np.int32)) if b > a else {}
    gathered = gather_to_root((a, b, local), dist, rank, world)
    if rank != 0:
        return None
    keys = next((set(g[2]) for g in gathered if g[2]), set())
    out = {}
    for k in keys:
        parts = [g[2][k] for g in sorted(gathered, key=lambda g: g[0]) if g[2]]
        out[k] = np.concatenate(parts, axis=0)
    return out
