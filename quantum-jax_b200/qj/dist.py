"""One process per GPU (launched by torchrun): rank plumbing for replicas and
box-sharded ensembles.  The step itself has no data-path collective: a single
box runs as replicas, and independent boxes are split across ranks; only the
timing (max over ranks) and optional diagnostics cross ranks."""

from __future__ import annotations

import datetime
import math
import os

import torch


def rank_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", device=None, timeout_s=120):
    """Join the process group when WORLD_SIZE > 1 (a short timeout, so ranks
    that wait on a missing peer end with an error); returns the
    torch.distributed module or None for a single process."""
    _, world, _ = rank_env()
    if world <= 1:
        return None
    import torch.distributed as dist

    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl" and device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """Maximum of a scalar over all ranks (the job's time is its slowest rank)."""
    if dist is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_box_records(records, dist=None):
    """End-of-run gather of per-box scalar diagnostics.  records: this rank's
    list of dicts, each with an integer "box" (the box's index in the whole
    ensemble).  Every rank gets all ranks' records ordered by box; a box
    reported by two ranks is an error (the partition gives each box to one
    rank).  One all_gather_object, after the timed region."""
    mine = [dict(r) for r in records]
    if dist is None:
        parts = [mine]
    else:
        parts = [None] * dist.get_world_size()
        dist.all_gather_object(parts, mine)
    out = sorted((r for p in parts for r in p), key=lambda r: r["box"])
    boxes = [r["box"] for r in out]
    if len(set(boxes)) != len(boxes):
        raise ValueError("gather_box_records: a box was reported by more than one rank")
    return out


def box_cost(n_cells: int) -> float:
    """Relative cost of one box step: C log C (FFT-dominated)."""
    return n_cells * math.log2(max(n_cells, 2))


def partition_boxes(costs, world: int):
    """Greedy longest-processing-time assignment of boxes to ranks: boxes in
    decreasing cost (ties by index), each to the least-loaded rank (ties by
    rank).  Deterministic, so every rank computes the same split.  Returns a
    list of box-index lists, one per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
