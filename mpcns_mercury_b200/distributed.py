"""Requests and ensemble members across the ranks of a multi-GPU job (one
process per GPU, torch.distributed for the plumbing).

Solves are independent, so the data path has no collective: each rank
admits and runs its own partition of one request stream (or of one
ensemble), and only the statistics meet, once, at the end — the cell
updates are summed, the makespan is the slowest rank's, and the latency
percentiles are taken over every rank's requests together.
"""
from __future__ import annotations

import numpy as np


def partition(work, world: int):
    """Indices of `work` (per-item costs) for each rank: longest first onto
    the least loaded rank (ties to the lower rank), each rank's indices in
    their original order.  Deterministic, so every rank computes the same
    partition from the same stream."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for q in sorted(range(len(work)), key=lambda i: (-float(work[i]), i)):
        r = min(range(world), key=lambda x: (load[x], x))
        parts[r].append(q)
        load[r] += float(work[q])
    return [sorted(p) for p in parts]


def gather_latencies(latencies):
    """Every rank's request latencies, concatenated in rank order (identity
    on one process)."""
    import torch

    dist = torch.distributed
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(latencies)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(latencies))
    return [v for part in out for v in part]


def aggregate(stats, latencies):
    """Job-wide serving statistics from each rank's own: cell updates summed,
    makespan the slowest rank's, p50/p99 over all requests."""
    import torch

    lat = gather_latencies(latencies)
    dist = torch.distributed
    work, span = float(stats["cell_updates"]), float(stats["makespan_s"])
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        t = torch.tensor([work, span], dtype=torch.float64)
        w = t.clone()
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
        m = t.clone()
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        work, span = float(w[0]), float(m[1])
    arr = np.asarray(lat, dtype=np.float64)
    return {"requests": len(lat), "cell_updates": work, "makespan_s": span,
            "mcell_updates_per_s": work / span / 1e6 if span > 0 else float("nan"),
            "latency_p50_s": float(np.percentile(arr, 50)) if len(arr) else float("nan"),
            "latency_p99_s": float(np.percentile(arr, 99)) if len(arr) else float("nan")}
