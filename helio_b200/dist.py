"""Multi-GPU plumbing for the visibility path: one process per GPU.

Views (and serving requests) are independent units, so the path shards without any
collective on the data path: each rank owns a subset of the views (balanced by
estimated cost, shard_views) of a scene that every rank holds resident, and culls
them in one batch of its own. The only collectives are
timing and result bookkeeping on the host side (max over ranks of a step time,
gathers of per-rank counts), which run on whatever backend the process group has
(NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env_rank() -> tuple[int, int, int]:
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def init(backend: str | None = None, timeout_s: int = 120) -> tuple[int, int]:
    """Initialises the default process group from torchrun's environment (no-op for one rank)."""
    rank, world, local = env_rank()
    if world > 1 and not dist.is_initialized():
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world


def shard_by_cost(costs: list[float], world: int) -> list[list[int]]:
    """Longest-processing-time assignment of unit indices to `world` ranks.
    Deterministic: ties break on the unit index, then on the rank index."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += costs[i]
    return [sorted(x) for x in out]


def assign_online(costs: list[float], world: int) -> list[int]:
    """Owner rank of each unit of a stream, in arrival order: the rank with the least
    cost assigned so far (ties to the lower rank). Units are not reordered, so a
    rank's units keep their arrival order; every rank computes the same owners."""
    loads = [0.0] * world
    owner = []
    for c in costs:
        r = min(range(world), key=lambda k: (loads[k], k))
        owner.append(r)
        loads[r] += c
    return owner


def view_cost(width: int, height: int, lod0_meshlets: int) -> float:
    """Cost estimate of one view: Hi-Z bytes plus the scene's object / meshlet test work."""
    return 8.0 * width * height + 4.0 * lod0_meshlets


def shard_views(views: list, lod0_meshlets: int, world: int, rank: int) -> list[int]:
    """Indices of the views that `rank` culls: the cost-balanced share (shard_by_cost
    over view_cost) of a view set whose scene every rank holds resident. Every rank
    computes the same partition, so no exchange is needed."""
    costs = [view_cost(v.width, v.height, lod0_meshlets) for v in views]
    return shard_by_cost(costs, world)[rank]


def gather_objects(obj, device=None) -> list:
    """Every rank's `obj`, in rank order (a list of one element for one rank)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [obj]
    parts: list = [None] * dist.get_world_size()
    dist.all_gather_object(parts, obj)
    return parts


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank number (step time) over all ranks."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: int, device=None) -> int:
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return int(value)
    t = torch.tensor([int(value)], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def sum_parity(summary: dict | None, device=None) -> dict | None:
    """Merges per-rank parity summaries (counts summed, mismatched fields merged, the
    slowest rank's check time) so that rank 0 reports the whole job's check."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return summary
    parts: list = [None] * dist.get_world_size()
    dist.all_gather_object(parts, summary)
    parts = [p for p in parts if p]
    if not parts:
        return None
    out = dict(parts[0])
    for k in ("views", "mismatches", "marginal_decisions", "marginal_meshlets", "marginal_objects", "meshlet_tests",
              "visible_meshlets"):
        out[k] = sum(int(p.get(k, 0)) for p in parts)
    fields: dict = {}
    for p in parts:
        for f, n in p.get("mismatched_fields", {}).items():
            fields[f] = fields.get(f, 0) + n
    out["mismatched_fields"] = fields
    out["seconds"] = max(float(p.get("seconds", 0.0)) for p in parts)
    out["ranks"] = len(parts)
    return out
