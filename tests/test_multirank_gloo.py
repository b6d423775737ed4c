"""World-size-2 gloo tests (CPU) of the multi-rank host logic: row split of
one set (main.f:283-295) and whole-set sharding of a batch, each rank
evaluating its share with the oracle, results gathered on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from starsmasher_b200 import inputs, multirank


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_compute(x, y, z, m, r2, i_begin, ni):
    import oracle
    rows = np.arange(i_begin, i_begin + ni, dtype=np.int32)
    return oracle.rows(x, y, z, m, r2, 0, row_idx=rows, nthreads=2)


def _worker(rank, world, port, mode, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        if mode == "rows":
            s = inputs.single_polytrope(701, 1.5, seed=3)
            res = multirank.forces_row_split(_oracle_compute, s.x, s.y, s.z, s.m, s.range2)
        else:
            b = inputs.batch_models(5, 64, 400, seed=9)
            res = multirank.forces_set_shard(_oracle_compute, b.offsets, b.x, b.y, b.z, b.m,
                                             b.range2)
        q.put((rank, [np.asarray(a) for a in res]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["rows", "sets"])
def test_two_rank_split_equals_single(mode):
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    if mode == "rows":
        s = inputs.single_polytrope(701, 1.5, seed=3)
        ref = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0)
    else:
        b = inputs.batch_models(5, 64, 400, seed=9)
        ref = [np.zeros(b.n) for _ in range(4)]
        for k in range(b.nsets):
            p = b.subset(k)
            a, e = b.offsets[k], b.offsets[k + 1]
            r = oracle.rows(p.x, p.y, p.z, p.m, p.range2, 0)
            for qd in range(4):
                ref[qd][a:e] = r[qd]
    for rank in (0, 1):
        for a, r in zip(got[rank], ref):
            np.testing.assert_array_equal(a, r)


def _oracle_compute_tensor(src, i_begin, ni, out):
    import torch
    a = [src[q].numpy() for q in range(5)]
    r = _oracle_compute(*a, i_begin, ni)
    for q in range(4):
        out[q, i_begin:i_begin + ni] = torch.from_numpy(np.asarray(r[q]))


def _worker_device(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        s = inputs.single_polytrope(701, 1.5, seed=3)
        lo, hi = multirank.gpu_row_range(s.n, world, rank)
        own = torch.from_numpy(np.stack([a[lo:hi] for a in (s.x, s.y, s.z, s.m, s.range2)]))
        # the step bench.py times, twice in a row (the second from fresh
        # owned data, as its end-to-end form does)
        step = multirank.RowSplitStep(_oracle_compute_tensor, own, s.n)
        step()
        src, res = step(own.clone())
        q.put((rank, src.numpy(), res.numpy()))
    finally:
        dist.destroy_process_group()


def test_two_rank_device_form_gathers_sources_and_rows():
    """The device-resident form on gloo host tensors: each rank starts with
    only its own rows' positions; sources and results are all-gathered."""
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_device, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {r: (src, res) for r, src, res in (q.get(timeout=120) for _ in range(2))}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    s = inputs.single_polytrope(701, 1.5, seed=3)
    ref = oracle.rows(s.x, s.y, s.z, s.m, s.range2, 0)
    for rank in (0, 1):
        src, res = got[rank]
        for qd, a in enumerate((s.x, s.y, s.z, s.m, s.range2)):
            np.testing.assert_array_equal(src[qd], a)
        for qd in range(4):
            np.testing.assert_array_equal(res[qd], ref[qd])


def test_row_ranges_and_set_shards():
    assert multirank.gpu_row_range(1001, 4, 3) == (753, 1001)
    assert [multirank.gpu_row_range(10, 3, r) for r in range(3)] == [(0, 4), (4, 8), (8, 10)]
    sh = multirank.shard_sets([100, 10, 90, 50, 60], 2)
    assert sorted(sum(sh, [])) == [0, 1, 2, 3, 4]
    cost = [sum(v ** 2 for v in np.array([100, 10, 90, 50, 60])[s]) for s in sh]
    assert max(cost) / min(cost) < 1.3
