"""Splitting one analysis over several GPUs (one process per GPU).

Every grid point is independent once the observations are replicated, which
is how the reference decomposes the analysis over MPI ranks: each rank owns
``nij1`` columns of the grid (letkf/run/src/common_mpi.f90:314, scatter at
:103) and receives every observation (MPI_ALLREDUCE / BCAST,
common_obs.f90:140, common_io.f90:1217-1223).  Here:

* ``partition_columns`` cuts the columns, in their grid order (latitude
  bands, so each rank's search boxes overlap and share L2), into contiguous
  ranges of nearly equal cost, the cost of a column being the sum over its
  levels of a per-point model fed by the nobsl histogram;
* ``broadcast_obs`` replicates the observation arrays from one rank with
  ``torch.distributed.broadcast`` (NCCL over NVLink on GPUs, gloo on CPU);
* ``column_slice`` gives a rank's grid and state, which go unchanged through
  the same analysis entry point (its ``nij1`` is the local column count, as
  in the reference);
* ``gather_columns`` reassembles the analysis on one rank when the output is
  needed in one place.

No collective runs during the analysis itself.
"""
from __future__ import annotations

import numpy as np
import torch

GRID_1D = ("lon1", "lat1", "ri1", "rj1", "dlon1", "dlat1", "phi1")


def point_cost(nobsl, k: int):
    """Relative cost of analysing a point with nobsl local observations:
    selection ~ nobsl, Gram ~ k^2 nobsl, eigensolve ~ k^3 when nobsl > 0."""
    n = np.asarray(nobsl, dtype=np.float64)
    return 1.0 + 0.05 * n + (k * k * n + 10.0 * k ** 3 * (n > 0)) / 2e4


def partition_columns(col_cost, nranks: int) -> list:
    """Contiguous column ranges [start, stop) with nearly equal total cost
    (greedy split of the cost prefix sum at multiples of total/nranks)."""
    c = np.asarray(col_cost, dtype=np.float64)
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    pre = np.concatenate([[0.0], np.cumsum(c)])
    tot = pre[-1]
    cuts = [0]
    for r in range(1, nranks):
        cut = int(np.searchsorted(pre, tot * r / nranks, side="left"))
        cuts.append(min(max(cut, cuts[-1]), c.size))
    cuts.append(c.size)
    return [(cuts[r], cuts[r + 1]) for r in range(nranks)]


def column_slice(grid: dict, fcst3d, fcst2d, start: int, stop: int):
    """A rank's grid (every [nij1] and [nlev][nij1] array cut to its columns)
    and forecast blocks [nv3d][nmem][nlev][ncol], [nv2d][nmem][ncol]."""
    g = {k: (v[..., start:stop] if k == "depth1" else v[start:stop]).contiguous() for k, v in grid.items()}
    return g, fcst3d[..., start:stop].contiguous(), fcst2d[..., start:stop].contiguous()


def broadcast_obs(obs: dict | None, src: int = 0, group=None, device=None) -> dict:
    """Replicate the observation arrays of rank `src` on every rank."""
    import torch.distributed as dist
    rank = dist.get_rank(group)
    meta = [None]
    if rank == src:
        meta = [{k: (tuple(v.shape), v.dtype) for k, v in obs.items()}]
    dist.broadcast_object_list(meta, src=src, group=group)
    out = {}
    for k, (shape, dtype) in meta[0].items():
        if rank == src:
            t = obs[k].contiguous()
            if device is not None:
                t = t.to(device)
        else:
            t = torch.empty(shape, dtype=dtype, device=device)
        dist.broadcast(t, src=src, group=group)
        out[k] = t
    return out


def gather_columns(a3, a2, parts: list, dst: int = 0, group=None):
    """Concatenate every rank's [..., ncol] analysis blocks on rank `dst`
    (None elsewhere).  Ranks pad to the largest part for the collective."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    width = max(b - a for a, b in parts)
    out = []
    for x in (a3, a2):
        pad = torch.zeros(*x.shape[:-1], width, dtype=x.dtype, device=x.device)
        pad[..., : x.shape[-1]] = x
        bufs = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(bufs, pad, group=group)
        out.append(torch.cat([bufs[r][..., : parts[r][1] - parts[r][0]] for r in range(world)], dim=-1)
                   if rank == dst else None)
    return out[0], out[1]
