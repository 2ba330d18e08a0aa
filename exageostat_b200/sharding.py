"""Sharding independent fields across GPUs (one process per GPU).

A single field's factorisation is one dependent DAG and stays on one GPU
(replicas only).  A batch of independent regional fields shards naturally:
fields go to ranks by longest-processing-time-first on their N^3 cost, every
rank evaluates its own fields with no inter-GPU traffic on the data path, and
one gather at the end hands every rank the full vector of log-likelihoods.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(costs, nranks: int):
    """Greedy LPT: fields in decreasing cost, each to the least-loaded rank.
    Returns a list of index lists (one per rank, each sorted)."""
    heap = [(0.0, r) for r in range(nranks)]
    parts = [[] for _ in range(nranks)]
    for i in sorted(range(len(costs)), key=lambda i: -costs[i]):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def sharded_batch_loglik(sizes, thetas, evaluate, group=None):
    """Evaluates every field's log-likelihood across the ranks of ``group``.

    ``evaluate(indices, thetas_subset) -> array`` computes this rank's fields
    (on the GPU: a ``Batch`` over those fields).  Returns the full vector on
    every rank.  Uses torch.distributed (gloo or nccl) for the final gather
    only."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    sizes = np.asarray(sizes)
    thetas = np.asarray(thetas, dtype=np.float64)
    parts = lpt_partition(sizes.astype(np.float64) ** 3, world)
    mine = parts[rank]
    local = np.asarray(evaluate(mine, thetas[mine]), dtype=np.float64) if mine else np.zeros(0)
    if world == 1:
        return local
    width = max(len(p) for p in parts)
    backend = dist.get_backend(group)
    device = "cuda" if backend == "nccl" else "cpu"
    buf = torch.full((width,), float("nan"), dtype=torch.float64, device=device)
    buf[: len(local)] = torch.from_numpy(local).to(device)
    gathered = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    out = np.empty(len(sizes))
    for r, p in enumerate(parts):
        out[p] = gathered[r][: len(p)].cpu().numpy()
    return out
