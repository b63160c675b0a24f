"""Multi-GPU batching of signature work: one process per GPU.

Streams are independent, so a batch shards across ranks with no collective
on the data path: every rank takes a contiguous slice of streams, balanced by
total number of increments (so ranks finish together under uneven lengths),
and computes it with its own persistent launch.  The only collective is the
optional all-gather of the results when every rank needs the whole output
(NCCL over NVLink on GPUs; any torch.distributed backend works, which is how
the plumbing is tested with gloo on CPU).
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import signatures as S


def shard_bounds(offsets, world: int):
    """Contiguous stream ranges [lo, hi) per rank, balanced by total length.

    Rank r takes the streams whose increment rows start before the r-th
    quantile of all rows; every rank gets a (possibly empty) range and the
    ranges tile [0, n_streams).
    """
    off = np.asarray(offsets, dtype=np.int64)
    n = off.shape[0] - 1
    total = int(off[-1])
    bounds = []
    lo = 0
    for r in range(world):
        if r == world - 1:
            hi = n
        else:
            target = total * (r + 1) / world
            # first stream whose midpoint passes the target starts the next shard
            mids = (off[:-1] + off[1:]) / 2.0
            hi = int(np.searchsorted(mids, target, side="left"))
            hi = max(lo, min(hi, n))
        bounds.append((lo, hi))
        lo = hi
    return bounds


def _local_rows(increments, offsets, lo, hi):
    off = np.asarray(offsets, dtype=np.int64)
    local_off = off[lo:hi + 1] - off[lo]
    rows = increments[int(off[lo]):int(off[hi])]
    return rows, local_off


def sharded_signatures(increments, offsets, width: int, depth: int, mode: str = "f32c",
                       group=None, gather: bool = True, compute=None, device=None):
    """Signatures of a batch sharded over the ranks of `group`.

    ``increments``: this rank's view of the whole batch (host array or tensor
    with all rows; only the rank's slice is used).  ``compute(rows,
    local_offsets)`` returns the slice's signatures as a tensor ``[m, T]``; by
    default the GPU signature kernel on ``device``.  With ``gather`` the full
    ``[n_streams, T]`` result is returned on every rank (one all-gather),
    otherwise ``(lo, hi, local_result)``.
    """
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    bounds = shard_bounds(offsets, world)
    lo, hi = bounds[rank]
    rows, local_off = _local_rows(increments, offsets, lo, hi)
    T = S.tensor_size(width, depth)
    if compute is None:
        dev = torch.device(device or "cuda")
        dt = torch.float64 if mode == "f64" else torch.float32
        x = torch.as_tensor(np.asarray(rows)).to(dev, dt).contiguous()
        plan = S.SignaturePlan(local_off, width, depth, mode, device=dev)
        local = plan.run(x) if plan.n_streams else torch.zeros((0, T), dtype=dt, device=dev)
    else:
        local = compute(rows, local_off)
    if not gather or world == 1:
        return (lo, hi, local) if not gather else local
    # all-gather with padding to the largest shard
    m = max(h - l for l, h in bounds)
    pad = torch.zeros((m, T), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([parts[r][:h - l] for r, (l, h) in enumerate(bounds)])
