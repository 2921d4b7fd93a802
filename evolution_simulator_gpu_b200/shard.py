"""One generation over several GPUs.

Creatures are independent, so a generation splits into contiguous ranges of
the packed order, one per rank, balanced by each creature's predicted cost;
every rank runs its range on its own GPU with no exchange during the trials,
and the results are gathered to every rank at the end (an all-gather of the
76-byte records). The reference spreads work over devices the same way,
through independent engines (src/scheduler.rs:290-372).

The cost model is the arithmetic of one substep of a body of N nodes and M
muscles: about 75 M + 40 (N - 1) + 36 N + 110 (N - 2) operations.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

from .api import RESULT_DTYPE, WavePack


def predicted_cost(wave: WavePack) -> np.ndarray:
    n = (wave.heads[:, 0] & 255).astype(np.float64)
    m = wave.heads[:, 1].astype(np.float64)
    return 75.0 * m + 40.0 * (n - 1.0) + 36.0 * n + 110.0 * np.maximum(n - 2.0, 0.0)


def plan(cost: np.ndarray, world_size: int) -> np.ndarray:
    """Boundaries b[0..world_size] of contiguous ranges with about equal total
    cost: rank r runs creatures [b[r], b[r+1])."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    total = np.concatenate([[0.0], np.cumsum(cost, dtype=np.float64)])
    targets = total[-1] * np.arange(world_size + 1) / world_size
    b = np.searchsorted(total, targets, side="left").astype(np.int64)
    b[0], b[-1] = 0, len(cost)
    return np.maximum.accumulate(b)


def evaluate_sharded(evaluate: Callable[[WavePack], np.ndarray], wave: WavePack, rank: int, world_size: int,
                     group=None, device=None) -> np.ndarray:
    """Results of every creature of `wave` (packed order) on every rank; this
    rank evaluates its range with `evaluate` (a WavePack -> results
    function, such as Engine.run's first result)."""
    b = plan(predicted_cost(wave), world_size)
    mine = evaluate(wave.take(np.arange(b[rank], b[rank + 1]))) if b[rank + 1] > b[rank] else \
        np.zeros(0, RESULT_DTYPE)
    if world_size == 1:
        return mine
    import torch
    import torch.distributed as dist
    longest = int(np.max(np.diff(b)))
    words = RESULT_DTYPE.itemsize // 4
    local = np.zeros((longest, words), np.int32)
    local[:len(mine)] = np.ascontiguousarray(mine).view(np.int32).reshape(-1, words)
    t = torch.from_numpy(local)
    if device is not None:
        t = t.to(device)
    parts = [torch.empty_like(t) for _ in range(world_size)]
    dist.all_gather(parts, t, group=group)
    out = np.zeros(len(wave), RESULT_DTYPE)
    for r in range(world_size):
        k = int(b[r + 1] - b[r])
        out[b[r]:b[r + 1]] = parts[r].cpu().numpy()[:k].reshape(-1).view(RESULT_DTYPE)
    return out


def global_top_k(values: np.ndarray, ids: np.ndarray, k: int, world_size: int = 1, group=None, device=None):
    """The k largest `values` over all ranks with their `ids` (ties: the
    smaller id first), the same on every rank: each rank's own top k, an
    all-gather of k (value, id) pairs a rank, and one selection. Values that
    are not finite rank last."""
    v = np.where(np.isfinite(values), np.asarray(values, np.float64), -np.inf)
    ids = np.asarray(ids, np.int64)
    order = np.lexsort((ids, -v))[:k]
    v, ids = v[order], ids[order]
    if world_size == 1:
        return v, ids
    import torch
    import torch.distributed as dist
    pad = k - len(v)
    v = np.concatenate([v, np.full(pad, -np.inf)])
    ids = np.concatenate([ids, np.full(pad, np.iinfo(np.int64).max, np.int64)])
    tv, ti = torch.from_numpy(v), torch.from_numpy(ids)
    if device is not None:
        tv, ti = tv.to(device), ti.to(device)
    pv = [torch.empty_like(tv) for _ in range(world_size)]
    pi = [torch.empty_like(ti) for _ in range(world_size)]
    dist.all_gather(pv, tv, group=group)
    dist.all_gather(pi, ti, group=group)
    v = np.concatenate([p.cpu().numpy() for p in pv])
    ids = np.concatenate([p.cpu().numpy() for p in pi])
    order = np.lexsort((ids, -v))[:k]
    keep = ids[order] != np.iinfo(np.int64).max
    return v[order][keep], ids[order][keep]


def all_sum(values, world_size: int = 1, group=None, device=None) -> np.ndarray:
    """Element-wise sum of a few float64 values over the ranks."""
    x = np.asarray(values, np.float64)
    if world_size == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(x.copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, group=group)
    return t.cpu().numpy()
