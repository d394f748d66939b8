"""Permutation tests sharded over GPUs (one process per GPU).

The refits of a permutation test are independent instances sharing X, so
they shard with no data-path collective: every rank holds a replica of X,
runs the batched engine on its slice of the permutations, and the ranks
exchange only the per-permutation metric rows (a few KB) at the end. The
p-value follows R/main.R:2702-2718, (b + 1) / (B + 1).
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def shard(count: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous [start, stop) slice of `count` items for `rank`."""
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def pvalues(observed: np.ndarray, permuted: np.ndarray, lower_tail=False):
    """Per-column permutation p-values over the finite permuted rows."""
    observed = np.asarray(observed, dtype=np.float64)
    permuted = np.asarray(permuted, dtype=np.float64)
    out = np.full(observed.shape, np.nan)
    for j in range(observed.size):
        col = permuted[:, j]
        valid = np.isfinite(col)
        done = int(valid.sum())
        if not done or not np.isfinite(observed[j]):
            continue
        if lower_tail:
            extreme = int(np.sum(col[valid] <= observed[j]))
        else:
            extreme = int(np.sum(col[valid] >= observed[j]))
        out[j] = (extreme + 1) / (done + 1)
    return out


def _gather(rows: np.ndarray, world: int, group=None) -> np.ndarray:
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(np.ascontiguousarray(rows, dtype=np.float64))
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([t.shape[0]], dtype=torch.int64), group=group)
    width = t.shape[1]
    cap = int(max(s.item() for s in sizes))
    padded = torch.zeros((cap, width), dtype=torch.float64)
    padded[: t.shape[0]] = t
    bufs = [torch.zeros((cap, width), dtype=torch.float64) for _ in range(world)]
    dist.all_gather(bufs, padded, group=group)
    return np.concatenate([b[: int(s.item())].numpy() for b, s in zip(bufs, sizes)])


def permutation_test(X, Y, folds, permutations, prefixes, *, world=1, rank=0,
                     metric="q2", compute: Callable | None = None, group=None,
                     **kwargs):
    """Observed CV metric path and permutation p-values, permutations sharded
    over `world` ranks. `compute(X, Y, folds, perms, prefixes, metric=...)`
    returns a (len(perms) + 1) x prefixes metric array (row 0 observed); it
    defaults to the batched CUDA engine."""
    if compute is None:
        from .api import cv_permutation

        def compute(x, y, f, p, pre, metric="q2", **kw):
            return cv_permutation(x, y, f, p, pre, metric=metric, **kw)["metrics"]
    perms = np.asarray(permutations)
    start, stop = shard(perms.shape[0], world, rank)
    local = np.asarray(compute(X, Y, folds, perms[start:stop], prefixes,
                               metric=metric, **kwargs))
    observed = local[0]
    permuted = local[1:]
    if world > 1:
        permuted = _gather(permuted, world, group)
    lower = metric == "rmsd"
    return observed, permuted, pvalues(observed, permuted, lower_tail=lower)
