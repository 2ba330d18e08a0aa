"""Sharding independent fields across GPUs (one process per GPU).

A single field's factorisation is one dependent DAG and stays on one GPU
(replicas only).  A batch of independent regional fields shards naturally:
fields go to ranks by longest-processing-time-first on their N^3 cost, every
rank evaluates its own fields with no inter-GPU traffic on the data path, and
one gather at the end hands every rank the full vectors of log-likelihoods
(and gradients).
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


def _world(group):
    import torch.distributed as dist

    if not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def _gather_rows(local, parts, ncols, group):
    """All-gathers every rank's (len(part), ncols) block into the full
    (nfields, ncols) array, on every rank."""
    import torch
    import torch.distributed as dist

    world, _ = _world(group)
    width = max(len(p) for p in parts)
    device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    buf = torch.full((width, ncols), float("nan"), dtype=torch.float64, device=device)
    if len(local):
        buf[: len(local)] = torch.from_numpy(np.asarray(local, dtype=np.float64).reshape(len(local), ncols)).to(device)
    gathered = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(gathered, buf, group=group)
    out = np.empty((sum(len(p) for p in parts), ncols))
    for r, p in enumerate(parts):
        out[p] = gathered[r][: len(p)].cpu().numpy()
    return out


def sharded_batch_loglik(sizes, thetas, evaluate, group=None, grad=False):
    """Evaluates every field's log-likelihood (and, with grad, its gradient)
    across the ranks of ``group``.

    ``evaluate(indices, thetas_subset)`` computes this rank's fields and
    returns the log-likelihoods, or (log-likelihoods, gradients) with grad.
    Returns the full vector (and the full gradient array) on every rank.
    Uses torch.distributed (gloo or nccl) for the final gather only."""
    world, rank = _world(group)
    sizes = np.asarray(sizes)
    thetas = np.asarray(thetas, dtype=np.float64)
    nparams = thetas.shape[1]
    parts = lpt_partition(sizes.astype(np.float64) ** 3, world)
    mine = parts[rank]
    if mine:
        res = evaluate(mine, thetas[mine])
        ll, g = (res if grad else (res, None))
        ll = np.asarray(ll, dtype=np.float64)
        g = None if g is None else np.asarray(g, dtype=np.float64).reshape(len(mine), nparams)
    else:
        ll, g = np.zeros(0), np.zeros((0, nparams))
    if world == 1:
        return (ll, g) if grad else ll
    cols = 1 + (nparams if grad else 0)
    local = np.concatenate([ll.reshape(-1, 1)] + ([g] if grad else []), axis=1) if len(mine) else np.zeros((0, cols))
    full = _gather_rows(local, parts, cols, group)
    return (full[:, 0], full[:, 1:]) if grad else full[:, 0]


class ShardedBatch:
    """This rank's share (LPT on N^3) of a batch of independent fields as one
    ``exageostat_b200.Batch``; ``loglik`` evaluates it and gathers every
    field's log-likelihood (and gradient) onto every rank."""

    def __init__(self, xs, ys, zs, kernel: int = 0, metric: int = 0, ts: int = 256, group=None):
        from . import Batch

        world, rank = _world(group)
        self.group = group
        self.sizes = np.array([len(x) for x in xs])
        self.parts = lpt_partition(self.sizes.astype(np.float64) ** 3, world)
        self.mine = self.parts[rank]
        self.batch = Batch([xs[i] for i in self.mine], [ys[i] for i in self.mine], [zs[i] for i in self.mine],
                           kernel=kernel, metric=metric, ts=ts) if self.mine else None

    def loglik(self, thetas, grad: bool = False):
        def evaluate(idx, th):
            return self.batch.loglik(th, grad=grad)

        return sharded_batch_loglik(self.sizes, thetas, evaluate, group=self.group, grad=grad)

    def close(self):
        if self.batch is not None:
            self.batch.close()
            self.batch = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
