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
    pair count, with no data exchange before the gather;
  * device-resident form (``forces_row_split_device``): every rank holds the
    positions of its own rows (as after the reference's integrator step), the
    five source arrays are all-gathered on the device (NCCL over NVLink), each
    rank evaluates its rows against all n sources, and the row slices are
    all-gathered again; no reduction is needed.

Collective buffers live on the process group's device: the current CUDA
device under NCCL, host memory under gloo.  The per-rank computation is a
callable, so the same logic runs with the GPU library (``gpu_compute``,
``gpu_compute_device``) or, in the CPU tests, with any other evaluator.
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


def comm_device(group=None):
    """Where collective buffers must live for ``group``: NCCL takes CUDA
    tensors (the current device), gloo host tensors."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def allgather_rows(part, n: int, group=None):
    """All-gather row slices: ``part`` is a (k, hi - lo) tensor holding this
    rank's rows [lo, hi) of gpu_row_range; returns the (k, n) tensor on
    ``part``'s device.  Slices are padded to the common stride (all_gather
    wants equal sizes) and unpadded on arrival."""
    import torch
    import torch.distributed as dist
    nranks = dist.get_world_size(group)
    stride = (n - 1) // nranks + 1 if n > 0 else 0
    buf = part.new_zeros((part.shape[0], stride))
    buf[:, : part.shape[1]] = part
    bufs = [torch.empty_like(buf) for _ in range(nranks)]
    dist.all_gather(bufs, buf, group=group)
    full = part.new_empty((part.shape[0], n))
    for r in range(nranks):
        a, b = gpu_row_range(n, nranks, r)
        full[:, a:b] = bufs[r][:, : b - a]
    return full


def _allgather_rows(group, rank: int, nranks: int, n: int, lo: int, part: np.ndarray):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(part)).to(comm_device(group))
    return allgather_rows(t, n, group).cpu().numpy()


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
    """Batches: whole sets per rank (LPT by N^2), all results gathered.  Each
    rank packs the rows of its own sets, in set order, into a (4, k) block;
    the blocks are all-gathered (padded to the largest) and unpacked with the
    set assignment every rank knows, so no rank sends rows it does not own."""
    import torch
    import torch.distributed as dist
    nranks = dist.get_world_size(group)
    rank = dist.get_rank(group)
    offsets = np.asarray(offsets)
    sizes = np.diff(offsets)
    shards = shard_sets(sizes, nranks)
    n = int(offsets[-1])
    counts = [int(sum(int(sizes[s]) for s in shards[r])) for r in range(nranks)]
    width = max(1, max(counts))
    block = np.zeros((4, width))
    col = 0
    for s in shards[rank]:
        a, b = int(offsets[s]), int(offsets[s + 1])
        res = compute(x[a:b], y[a:b], z[a:b], m[a:b], range2[a:b], 0, b - a)
        for q in range(4):
            block[q, col:col + b - a] = np.asarray(res[q])[: b - a]
        col += b - a
    dev = comm_device(group)
    t = torch.from_numpy(block).to(dev)
    bufs = [torch.empty_like(t) for _ in range(nranks)]
    dist.all_gather(bufs, t, group=group)
    out = np.zeros((4, n))
    for r in range(nranks):
        got = bufs[r].cpu().numpy()
        col = 0
        for s in shards[r]:
            a, b = int(offsets[s]), int(offsets[s + 1])
            out[:, a:b] = got[:, col:col + b - a]
            col += b - a
    return tuple(out[q].copy() for q in range(4))


def gpu_compute(ctx, nkernel: int = 0, precision: str = "f32split") -> RowCompute:
    """Per-rank computation with the GPU library (host arrays)."""
    def f(x, y, z, m, range2, i_begin, ni):
        return ctx.forces(x, y, z, m, range2, nkernel, precision, i_begin, ni)
    return f


# compute(src, i_begin, ni, out): src a (5, n) tensor of x, y, z, m, range2;
# fills rows [i_begin, i_begin + ni) of the (4, n) tensor out (ax, ay, az, pot)
DeviceRowCompute = Callable[[object, int, int, object], None]


def forces_row_split_device(compute: DeviceRowCompute, own, n: int, group=None):
    """Device-resident row split of one set.  ``own`` is the (5, hi - lo)
    tensor of this rank's rows [lo, hi) (x, y, z, m, range2); the sources are
    all-gathered, the rank's rows evaluated against all n of them, and the
    (4, n) result all-gathered, every tensor on ``own``'s device.  Returns
    (sources, result)."""
    import torch.distributed as dist
    nranks = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = gpu_row_range(n, nranks, rank)
    if own.shape[1] != hi - lo:
        raise ValueError(f"rank {rank} holds {own.shape[1]} rows, its slice is {hi - lo}")
    src = allgather_rows(own, n, group)
    out = src.new_zeros((4, n))
    compute(src, lo, hi - lo, out)
    return src, allgather_rows(out[:, lo:hi], n, group)


class RowSplitStep:
    """One gravity step of the reference's multi-GPU row split, as bench.py
    times it: this rank owns rows [lo, hi) of one set of n particles
    (main.f:283-295) and holds their (x, y, z, m, range2) in ``own``; each
    call all-gathers the sources, evaluates the owned rows and all-gathers
    the (4, n) result (forces_row_split_device)."""

    def __init__(self, compute: DeviceRowCompute, own, n: int, group=None):
        import torch.distributed as dist
        self.compute, self.own, self.n, self.group = compute, own, n, group
        self.lo, self.hi = gpu_row_range(n, dist.get_world_size(group), dist.get_rank(group))
        if own.shape[1] != self.hi - self.lo:
            raise ValueError(f"own holds {own.shape[1]} rows, the rank's slice is {self.hi - self.lo}")

    def __call__(self, own=None):
        """Returns (sources, result); ``own`` replaces the owned rows' data
        (e.g. positions freshly copied from the host)."""
        return forces_row_split_device(self.compute, self.own if own is None else own, self.n,
                                       self.group)


def gpu_compute_device(ctx, nkernel: int = 0, precision: str = "f32split") -> DeviceRowCompute:
    """Per-rank computation with the GPU library on device tensors, stream
    ordered: the library is pointed at torch's current stream, where the
    gathered sources and the zeroed outputs were written and where the
    collective that follows is enqueued, so no host synchronisation is
    needed between the all-gathers and the gravity call."""
    import torch

    def f(src, i_begin, ni, out):
        # torch's default stream reports handle 0, which the library reads as
        # "the context's own stream"; pass cudaStreamLegacy (handle 1), the
        # same default stream, instead
        ctx.set_stream(torch.cuda.current_stream(src.device).cuda_stream or 1)
        n = src.shape[1]
        ctx.forces_device(n, src[0], src[1], src[2], src[3], src[4], out[0], out[1], out[2],
                          out[3], nkernel=nkernel, precision=precision, i_begin=i_begin, ni=ni)
    return f
