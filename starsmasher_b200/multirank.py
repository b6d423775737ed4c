"""Multi-rank host logic: which rows / sets each rank computes, and the
gather of results.  One process per GPU, ``torch.distributed`` for the
plumbing (NCCL on GPUs, gloo on CPU).

Reference behaviour restated:
  * row split of the GPU path across gravity ranks, main.f:283-295:
    gravstride = (n-1)/ngravprocs + 1; rank r computes rows
    [r*gravstride, min((r+1)*gravstride, n)) against all n sources;
  * results gathered to every rank (the reference gathers grpot to rank 0
    with mpi_gatherv, balAV3.f:423-434, and allreduces accelerations,
    balAV3.f:478-483; here each rank's rows are all-gathered);
  * independent particle sets (batches) are sharded whole, longest first by
    pair count, with no data exchange before the gather.

The per-rank computation is a callable, so the same logic runs with the GPU
library (``gpu_compute``) or, in the CPU tests, with any other evaluator.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np

# compute(x, y, z, m, range2, i_begin, ni) -> (ax, ay, az, pot) for rows [i_begin, i_begin+ni)
RowCompute = Callable[[np.ndarray, np.ndarray, np.ndarray, np.ndarray, np.ndarray, int, int],
                      Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]]


def gpu_row_range(n: int, nranks: int, rank: int) -> Tuple[int, int]:
    """0-based [lo, hi) rows of ``rank`` (main.f:283-295)."""
    stride = (n - 1) // nranks + 1 if n > 0 else 0
    lo = min(stride * rank, n)
    return lo, min(lo + stride, n)


def shard_sets(sizes: Sequence[int], nranks: int) -> List[List[int]]:
    """Longest-processing-time assignment of sets (cost N^2) to ranks."""
    order = sorted(range(len(sizes)), key=lambda s: -int(sizes[s]) ** 2)
    load = [0] * nranks
    out: List[List[int]] = [[] for _ in range(nranks)]
    for s in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(s)
        load[r] += int(sizes[s]) ** 2
    return [sorted(v) for v in out]


def _allgather_rows(group, rank: int, nranks: int, n: int, lo: int, part: np.ndarray):
    import torch
    import torch.distributed as dist
    stride = (n - 1) // nranks + 1 if n > 0 else 0
    buf = torch.zeros((4, stride), dtype=torch.float64)
    buf[:, : part.shape[1]] = torch.from_numpy(part)
    bufs = [torch.zeros_like(buf) for _ in range(nranks)]
    dist.all_gather(bufs, buf, group=group)
    full = np.zeros((4, n))
    for r in range(nranks):
        a, b = gpu_row_range(n, nranks, r)
        full[:, a:b] = bufs[r].numpy()[:, : b - a]
    return full


def forces_row_split(compute: RowCompute, x, y, z, m, range2, group=None):
    """Every rank computes its row slice of one set against all sources and
    receives the full result (ax, ay, az, pot)."""
    import torch.distributed as dist
    nranks = dist.get_world_size(group)
    rank = dist.get_rank(group)
    n = len(x)
    lo, hi = gpu_row_range(n, nranks, rank)
    ax, ay, az, pot = compute(x, y, z, m, range2, lo, hi - lo)
    part = np.stack([np.asarray(a)[lo:hi] if len(a) == n else np.asarray(a)
                     for a in (ax, ay, az, pot)])
    return tuple(_allgather_rows(group, rank, nranks, n, lo, part))


def forces_set_shard(compute: RowCompute, offsets, x, y, z, m, range2, group=None):
    """Batches: whole sets per rank (LPT by N^2), all results gathered."""
    import torch
    import torch.distributed as dist
    nranks = dist.get_world_size(group)
    rank = dist.get_rank(group)
    offsets = np.asarray(offsets)
    sizes = np.diff(offsets)
    mine = shard_sets(sizes, nranks)[rank]
    n = int(offsets[-1])
    local = np.zeros((4, n))
    owned = np.zeros(n)
    for s in mine:
        a, b = int(offsets[s]), int(offsets[s + 1])
        res = compute(x[a:b], y[a:b], z[a:b], m[a:b], range2[a:b], 0, b - a)
        for q in range(4):
            local[q, a:b] = np.asarray(res[q])[: b - a]
        owned[a:b] = 1.0
    t = torch.from_numpy(np.vstack([local, owned[None, :]]))
    dist.all_reduce(t, group=group)  # each row is owned by exactly one rank
    t = t.numpy()
    assert np.all(t[4] == 1.0)
    return tuple(t[q].copy() for q in range(4))


def gpu_compute(ctx, nkernel: int = 0, precision: str = "f32split") -> RowCompute:
    """Per-rank computation with the GPU library (host arrays)."""
    def f(x, y, z, m, range2, i_begin, ni):
        return ctx.forces(x, y, z, m, range2, nkernel, precision, i_begin, ni)
    return f
