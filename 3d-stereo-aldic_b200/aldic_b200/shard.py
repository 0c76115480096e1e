"""Subset sharding across ranks (one process per GPU).

Subsets are independent in every batched call (the reference runs them under `parfor`,
func_quadtree/LocalICGNQuadtree.m:116), so a call shards by contiguous ranges of subsets,
balanced by an expected cost per subset (window area times the expected iteration count: the
previous frame's codes where a sequence has them, else uniform).  Each rank solves its range
on its own GPU into device tensors; the per-subset results (U, F and the code: 7 FP64 values,
56 B per subset; the 21 Hessian entries on request) are packed into one tensor per rank and
all-gathered with `torch.distributed.all_gather` (NCCL over NVLink for CUDA tensors, gloo for
CPU ones), so every rank holds the full arrays the host-side filters and fills of the
reference driver need.  The gather is the only collective; there is none inside the data
path.
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


def icgn_cost(winsize, conv=None, n=None):
    """Expected cost per subset: (w + 1)^2 pixels times the iterations the previous solve took
    (its codes; 100 for failures), or times 1 without one."""
    w = np.asarray(winsize, dtype=np.float64)
    area = (w + 1.0) ** 2
    if conv is None:
        return np.broadcast_to(area, (n,)).astype(np.float64) if area.ndim == 0 else area
    c = np.asarray(conv)
    it = np.where((c > 0) & (c <= 100), c, 100).astype(np.float64)
    return area * it


# per-subset widths of the arrays a local IC-GN call returns (MATLAB layouts)
ICGN_FIELDS = {"U": 2, "F": 4, "conv": 1, "H": 21}


def pack(results, fields, n, torch, device):
    """One (n, sum of widths) FP64 tensor of the per-subset results (numpy arrays or tensors,
    MATLAB layouts: U 2n interleaved, F 4n, conv n, H n x 21)."""
    cols = []
    for k in fields:
        v = results[k]
        t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v))
        t = t.to(device=device, dtype=torch.float64)
        if k == "H" and t.dim() == 1:  # flat n x 21 column-major (a device output buffer)
            t = t.reshape(21, n).t()
        cols.append(t.reshape(n, ICGN_FIELDS[k]))
    return torch.cat(cols, 1) if cols else torch.empty((n, 0), dtype=torch.float64, device=device)


def unpack(packed, fields, torch):
    """The inverse of pack: a dict of tensors in MATLAB layouts (conv as int32)."""
    out, c = {}, 0
    for k in fields:
        w = ICGN_FIELDS[k]
        v = packed[:, c:c + w]
        c += w
        out[k] = v.reshape(-1).to(torch.int32) if k == "conv" else (v.contiguous() if k == "H" else v.reshape(-1))
    return out


def gather_rows(mine, parts, group=None):
    """All-gather the row blocks of a partition: `mine` is this rank's (stop - start, m)
    tensor; returns the (n, m) tensor of all ranks' rows in subset order.  Blocks are padded
    to the largest, so every rank sends the same size (one all_gather call)."""
    import torch
    import torch.distributed as dist

    rows = max(e - s for s, e in parts)
    m = mine.shape[1]
    buf = torch.zeros((rows, m), dtype=mine.dtype, device=mine.device)
    buf[:mine.shape[0]] = mine
    blocks = [torch.empty_like(buf) for _ in parts]
    dist.all_gather(blocks, buf, group=group)
    return torch.cat([b[:e - s] for b, (s, e) in zip(blocks, parts)], 0)


def sharded_local_icgn(solve, coords, U0, group=None, cost=None, fields=("U", "F", "conv"), device=None):
    """Run `solve(coords_part, U0_part) -> dict(U, F, conv[, H])` on this rank's range of
    subsets and all-gather the results as one packed FP64 tensor per rank (on `device`: the
    rank's CUDA device under NCCL, the CPU under gloo).  Returns a dict of tensors on that
    device.  With no process group the call is local."""
    import torch
    import torch.distributed as dist

    coords = np.asarray(coords, dtype=np.float64)
    U0 = np.asarray(U0, dtype=np.float64)
    n = coords.shape[0]
    if group is None and not (dist.is_available() and dist.is_initialized()):
        res = solve(coords, U0)
        return unpack(pack(res, fields, n, torch, device or "cpu"), fields, torch)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = partition(n, world, cost)
    s, e = parts[rank]
    mine = pack(solve(coords[s:e], U0[2 * s:2 * e]), fields, e - s, torch, device)
    return unpack(gather_rows(mine, parts, group), fields, torch)
