"""Subset sharding across ranks (one process per GPU).

Subsets are independent in every batched call (the reference runs them under `parfor`,
func_quadtree/LocalICGNQuadtree.m:116), so a call shards by contiguous ranges of subsets,
balanced by an expected cost per subset (window area; iterations are unknown beforehand).
Each rank solves its range on its own GPU; the per-subset results (~64 B each) are then
all-gathered so every rank holds the full arrays the host-side filters and fills of the
reference driver need.  The gather is the only collective; there is none inside the
data path.
"""
from __future__ import annotations

import numpy as np


def partition(n: int, world: int, cost=None):
    """Contiguous [start, stop) ranges of n subsets for `world` ranks with near-equal
    total cost (cost: per-subset weights, default uniform)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if cost is None:
        bounds = np.linspace(0, n, world + 1).round().astype(int)
    else:
        c = np.concatenate([[0.0], np.cumsum(np.asarray(cost, dtype=np.float64))])  # c[k] = cost of [0, k)
        targets = c[-1] * np.arange(1, world) / world
        hi = np.clip(np.searchsorted(c, targets, side="left"), 1, max(n, 1))
        lo = hi - 1
        cut = np.where(np.abs(c[lo] - targets) <= np.abs(c[np.minimum(hi, n)] - targets), lo, hi)
        bounds = np.concatenate([[0], np.minimum(cut, n), [n]]).astype(int)
        bounds = np.maximum.accumulate(bounds)
    return [(int(bounds[r]), int(bounds[r + 1])) for r in range(world)]


# per-subset widths of the arrays a local IC-GN call returns (MATLAB layouts)
ICGN_FIELDS = {"U": 2, "F": 4, "H": 21, "conv": 1}


def _slice_rows(arr, start, stop, width):
    a = np.asarray(arr)
    if width == 21:  # n x 21
        return a[start:stop]
    return a.reshape(-1, width)[start:stop].reshape(-1) if width > 1 else a[start:stop]


def sharded_local_icgn(solve, coords, U0, group=None, cost=None):
    """Run `solve(coords_part, U0_part) -> dict(U, F, H, conv)` on this rank's range of
    subsets and all-gather the results.  With no process group the call is local."""
    coords = np.asarray(coords, dtype=np.float64)
    n = coords.shape[0]
    import torch.distributed as dist

    if group is None and not (dist.is_available() and dist.is_initialized()):
        return solve(coords, np.asarray(U0, dtype=np.float64))
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition(n, world, cost)
    s, e = parts[rank]
    U0 = np.asarray(U0, dtype=np.float64)
    mine = solve(coords[s:e], U0[2 * s:2 * e])
    gathered = [None] * world
    dist.all_gather_object(gathered, {k: np.asarray(mine[k]) for k in ICGN_FIELDS}, group=group)
    out = {}
    for k, width in ICGN_FIELDS.items():
        pieces = [g[k] for g in gathered]
        out[k] = np.concatenate(pieces, axis=0)
    return out
