"""Sharding one volume across GPUs (one process per GPU, torch.distributed).

Voxels are independent (the reference's ThreadedLoop relies on the same,
core/algo/threaded_loop.h:324-362), so each rank deconvolves a contiguous
z-slab of the volume chosen to balance the number of masked voxels, with no
exchange during the solve.  The only collective is the final gather of the
FOD slabs to rank 0, after every rank has finished.
"""
from __future__ import annotations

import numpy as np


def slab_bounds(mask: np.ndarray | None, dims, world: int):
    """Voxel-index ranges [start, end) per rank, cut at z-slice boundaries
    (layout [z][y][x]) so that each holds about the same number of masked
    voxels.  Every voxel belongs to exactly one range."""
    nx, ny, nz = dims
    plane = nx * ny
    if mask is None:
        per_z = np.full(nz, plane, np.int64)
    else:
        per_z = np.asarray(mask, bool).reshape(nz, plane).sum(axis=1).astype(np.int64)
    cum = np.concatenate([[0], np.cumsum(per_z)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        z = int(np.searchsorted(cum, target, side="left"))
        z = min(max(z, cuts[-1]), nz)
        cuts.append(z)
    cuts.append(nz)
    return [(cuts[r] * plane, cuts[r + 1] * plane) for r in range(world)]


def dwi2fod_distributed(dwi: np.ndarray, mask: np.ndarray | None, dims, nsh: int, solve, group=None):
    """Deconvolve this rank's slab with ``solve(dwi_slab, mask_slab) -> fod
    [n][nsh] float32`` and gather the full FOD on rank 0 (None elsewhere)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    bounds = slab_bounds(mask, dims, world)
    a, b = bounds[rank]
    fod = np.asarray(solve(dwi[a:b], None if mask is None else mask[a:b]), np.float32).reshape(b - a, nsh)
    # pad every slab to the longest for a fixed-size gather
    longest = max(e - s for s, e in bounds)
    buf = torch.zeros((longest, nsh), dtype=torch.float32)
    buf[:b - a] = torch.from_numpy(fod)
    backend = dist.get_backend(group)
    if backend == "nccl":
        buf = buf.cuda()
    gathered = [torch.empty_like(buf) for _ in range(world)] if rank == 0 else None
    dist.gather(buf, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = np.zeros((dwi.shape[0], nsh), np.float32)
    for r, (s, e) in enumerate(bounds):
        out[s:e] = gathered[r][:e - s].cpu().numpy()
    return out
