"""The reference's own GPU library against this one, on the benchmark workloads.

oracle/_ref/libsphgrav_ref.so is SPHgrav_lib2 (parallel_bleeding_edge/src/
SPHgrav_lib2/grav_force_direct.cu: FP32 pair terms on absolute coordinates,
float-float "ds64" sums) compiled unchanged for sm_100a by oracle/Makefile.
Both libraries are driven through the same legacy ABI, firsthalf_grav_forces_ /
lasthalf_grav_forces_ (grav.f:25, balAV3.f:418), from host arrays with every
copy inside the timed region, and both are scored against this library's FP64
kernel (<= 1e-12 of the CPU path).  Each case prints one JSON line with the
pair rates and errors of both.
"""
import ctypes
import json
import os
import time

import numpy as np
import pytest

import oracle
from conftest import err_report
from starsmasher_b200 import api, inputs

pytestmark = pytest.mark.gpu


def _ref_lib():
    if not os.path.exists(oracle.REF_GPU_LIB):
        pytest.skip("reference GPU library not built (make -C oracle ref)")
    return ctypes.CDLL(oracle.REF_GPU_LIB, mode=ctypes.RTLD_LOCAL)


def _legacy_call(lib, n, arrs, outs, nkernel=0):
    P = ctypes.POINTER(ctypes.c_double)
    ia = [ctypes.c_int(v) for v in (n, 1, n, 1, nkernel)]
    lib.firsthalf_grav_forces_(*(ctypes.byref(v) for v in ia[:3]), *(a.ctypes.data_as(P) for a in arrs),
                               ctypes.byref(ia[3]), ctypes.byref(ia[4]))
    rk = ctypes.c_int(0)
    lib.lasthalf_grav_forces_(ctypes.byref(ia[0]), *(a.ctypes.data_as(P) for a in outs), ctypes.byref(rk))


def _best_seconds(fn, reps=2):
    fn()  # warm-up: allocations, first launch
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        best = min(best, time.perf_counter() - t0)
    return best


@pytest.mark.parametrize("workload", ["config2", "config3"])
def test_faster_and_more_accurate_than_reference_gpu_library(gpu_ctx, workload):
    ref = _ref_lib()
    s = inputs.cached(workload)
    n = s.n
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (s.x, s.y, s.z, s.m, s.range2)]
    fp64 = gpu_ctx.forces(*arrs, 0, "fp64")

    out_ref = [np.zeros(n) for _ in range(4)]
    t_ref = _best_seconds(lambda: _legacy_call(ref, n, arrs, out_ref))

    out_our = [np.zeros(n) for _ in range(4)]
    api.set_legacy_precision("f32split")

    def run_ours():
        api.firsthalf_grav_forces(n, 1, n, *arrs)
        api.lasthalf_grav_forces(n, *out_our)

    t_our = _best_seconds(run_ours)
    r_ref = err_report(*out_ref, *fp64)
    r_our = err_report(*out_our, *fp64)
    pairs = float(n) * n
    print(json.dumps({"workload": workload, "n": n, "path": "legacy ABI, host arrays, copies included",
                      "reference_gpu_lib": {"gpairs_s": pairs / t_ref / 1e9, "seconds": t_ref, **r_ref},
                      "this_lib_f32split": {"gpairs_s": pairs / t_our / 1e9, "seconds": t_our, **r_our}}))
    assert t_our < t_ref
    assert r_our["acc_max"] <= r_ref["acc_max"]
    assert r_our["acc_rms"] <= r_ref["acc_rms"]


def test_batched_launch_beats_reference_per_set_calls(gpu_ctx):
    """Config 4 (64 models, N log-uniform in [4,096, 131,072]).  The reference
    library has no batch entry point, so its way to evaluate the models is one
    firsthalf/lasthalf call per model; this library evaluates all of them in
    one persistent launch (sphgrav_batch_forces, host arrays in and out)."""
    ref = _ref_lib()
    b = inputs.cached("config4")
    offs = [int(v) for v in b.offsets]
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (b.x, b.y, b.z, b.m, b.range2)]
    subsets = [[a[offs[s]:offs[s + 1]].copy() for a in arrs] for s in range(b.nsets)]
    out_ref = [[np.zeros(offs[s + 1] - offs[s]) for _ in range(4)] for s in range(b.nsets)]

    def run_ref():
        for s in range(b.nsets):
            _legacy_call(ref, offs[s + 1] - offs[s], subsets[s], out_ref[s])

    t_ref = _best_seconds(run_ref)
    got = {}

    def run_ours():
        got["r"] = gpu_ctx.batch_forces(offs, *arrs, 0, "f32split")

    t_our = _best_seconds(run_ours)
    fp64 = [np.zeros(b.n) for _ in range(4)]
    for s in range(b.nsets):
        o = gpu_ctx.forces(*subsets[s], 0, "fp64")
        for c in range(4):
            fp64[c][offs[s]:offs[s + 1]] = o[c]
    r_ref = err_report(*(np.concatenate([out_ref[s][c] for s in range(b.nsets)]) for c in range(4)), *fp64)
    r_our = err_report(*got["r"][:4], *fp64)
    pairs = float(b.pairs)
    print(json.dumps({"workload": "config4", "nsets": b.nsets, "n": b.n,
                      "path": "reference: 64 legacy-ABI calls; this lib: one sphgrav_batch_forces; host arrays",
                      "reference_gpu_lib": {"gpairs_s": pairs / t_ref / 1e9, "seconds": t_ref, **r_ref},
                      "this_lib_batched": {"gpairs_s": pairs / t_our / 1e9, "seconds": t_our, **r_our}}))
    assert t_our < t_ref
    assert r_our["acc_max"] <= r_ref["acc_max"]
