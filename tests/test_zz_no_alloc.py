"""The entry point that allocates no device memory.

Some callers cannot call cudaMalloc (work issued while a CUDA graph is being
captured, hosts that own all device memory through their own pool, codes
that forbid allocations after start-up).  sphgrav_forces_fp64_noalloc takes
device inputs and outputs and keeps its scratch in a static device array.
These tests call it through the C-ABI and compare it with the existing FP64
entry point (sphgrav_forces_device), at the FP64 tolerance the other tests
use, on two calls in a row (the second call reuses the scratch the first one
left behind).  This file is collected last so that a run stopping at the
first failure has already run every other test; it also passes alone in a
fresh process.
"""
import ctypes

import numpy as np
import pytest

from starsmasher_b200 import _lib, inputs

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _noalloc(lib, n, X, outs, nkernel, stream):
    return lib.sphgrav_forces_fp64_noalloc(n, *(ctypes.c_void_p(t.data_ptr()) for t in X),
                                           nkernel,
                                           *(ctypes.c_void_p(t.data_ptr()) for t in outs),
                                           ctypes.c_void_p(stream))


def _rel(a, b):
    ax, ay, az, pot = a
    bx, by, bz, bp = b
    da = np.sqrt((ax - bx) ** 2 + (ay - by) ** 2 + (az - bz) ** 2)
    amag = np.sqrt(bx ** 2 + by ** 2 + bz ** 2)
    ok = amag > 1e-3 * np.median(amag)
    return float((da / amag)[ok].max()), float((np.abs(pot - bp) / np.abs(bp)).max())


# The last case fills the scratch exactly: at SPHGRAV_NOALLOC_MAX_N one chunk's
# 4 n partial sums are the whole static array.
@pytest.mark.parametrize("nkernel,n,seed", [(0, 6000, 71), (1, 4099, 73), (2, 1537, 72),
                                            (1, "max", 74)])
def test_noalloc_matches_forces_device_twice(gpu_ctx, nkernel, n, seed):
    import torch
    lib = _lib.load()
    if n == "max":
        n = _noalloc_max_n()
    s = inputs.single_polytrope(n, 1.5, seed=seed)
    s.range2[::97] *= -1.0  # some point masses
    X = [_dev(a) for a in (s.x, s.y, s.z, s.m, s.range2)]
    ref = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(4)]
    gpu_ctx.forces_device(n, *X, *ref, nkernel=nkernel, precision="fp64")
    gpu_ctx.sync()
    want = [t.cpu().numpy() for t in ref]
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        outs = [torch.full((n,), np.nan, dtype=torch.float64, device="cuda") for _ in range(4)]
        assert _noalloc(lib, n, X, outs, nkernel, stream) == _lib.OK
        torch.cuda.synchronize()
        got = [t.cpu().numpy() for t in outs]
        acc_err, pot_err = _rel(got, want)
        assert acc_err <= FP64_TOL and pot_err <= FP64_TOL, (call, acc_err, pot_err)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu_ctx):
    lib = _lib.load()
    n = _noalloc_max_n() + 1
    null = ctypes.c_void_p(0)
    st = lib.sphgrav_forces_fp64_noalloc(n, null, null, null, null, null, 0, null, null, null,
                                         null, null)
    assert st == _lib.ERR_TOO_LARGE
    assert lib.sphgrav_forces_fp64_noalloc(10, null, null, null, null, null, 5, null, null,
                                           null, null, null) == _lib.ERR_INVALID_ARGUMENT


def _noalloc_max_n():
    import os
    import re
    from conftest import ROOT
    hdr = open(os.path.join(ROOT, "include", "sphgrav_b200.h")).read()
    return int(re.search(r"#define SPHGRAV_NOALLOC_MAX_N (\d+)", hdr).group(1))
