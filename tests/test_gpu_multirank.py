"""The multi-rank host logic under a real NCCL process group (one rank, one
GPU, in a spawned process): collective buffers must be CUDA tensors there,
which the gloo tests on CPU cannot show.  Both forms, host arrays
(forces_row_split) and device-resident (forces_row_split_device), must equal
a plain call of the library."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(port, q):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["NCCL_NVLS_ENABLE"] = "0"
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    from starsmasher_b200 import Context, inputs, multirank
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        s = inputs.single_polytrope(3001, 1.5, seed=5)
        with Context(0) as ctx:
            want = ctx.forces(s.x, s.y, s.z, s.m, s.range2, 0, "fp64")
            host = multirank.forces_row_split(multirank.gpu_compute(ctx, 0, "fp64"),
                                              s.x, s.y, s.z, s.m, s.range2)
            own = torch.from_numpy(np.stack([s.x, s.y, s.z, s.m, s.range2])).cuda()
            src, dev = multirank.forces_row_split_device(
                multirank.gpu_compute_device(ctx, 0, "fp64"), own, s.n)
            torch.cuda.synchronize()
            q.put(([np.asarray(a) for a in want], [np.asarray(a) for a in host],
                   dev.cpu().numpy(), bool(torch.equal(src, own))))
    except Exception as e:  # reported to the test, which fails on it
        q.put(repr(e))
    finally:
        dist.destroy_process_group()


def test_nccl_row_split_host_and_device_forms():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_worker, args=(_free_port(), q))
    p.start()
    got = q.get(timeout=300)
    p.join(timeout=120)
    assert not isinstance(got, str), got
    assert p.exitcode == 0
    want, host, dev, same_src = got
    assert same_src
    for q_ in range(4):
        np.testing.assert_array_equal(host[q_], want[q_])
        # device arrays may take another work split: FP64 sums agree to rounding
        np.testing.assert_allclose(dev[q_], want[q_], rtol=1e-12, atol=0)
