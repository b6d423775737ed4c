"""CPU oracle for the gravity path -- TEST INFRASTRUCTURE ONLY.

Loads ``liboracle_grav.so`` (grav_oracle.c, a C restatement of the
reference's CPU gravity path parallel_bleeding_edge/src/cpu_grav.f:1-381).
Only the tests, the smoke check and the benchmark's CPU-baseline leg use
this module; the GPU library never does.

Parity pin: the potentials of the reference's own snapshot files
(example_input/{collision,3_stars}/sph.start{1,2}u store grpot) are matched
by ``rows(..., nkernel=0)`` to the FP32 level they were written at; see
tests/golden/make_golden.py and tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_grav.so")
REF_GPU_LIB = os.path.join(HERE, "_ref", "libsphgrav_ref.so")
REF_SRC = "/root/reference/parallel_bleeding_edge/src/SPHgrav_lib2/grav_force_direct.cu"

_lib = None


def build(reference: bool = True) -> None:
    """Compile the oracle (and, where the reference tree is mounted, the
    reference's own GPU library into _ref/, as a comparator)."""
    subprocess.run(["make", "-C", HERE, "liboracle_grav.so"], check=True, capture_output=True)
    if reference and os.path.exists(REF_SRC):
        subprocess.run(["make", "-C", HERE, "ref"], check=True, capture_output=True)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build(reference=False)
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    I = ctypes.c_int
    lib.oracle_triangle.argtypes = [I, P, P, P, P, P, I, I, I, I, P, P, P, P]
    lib.oracle_triangle.restype = I
    lib.oracle_rows.argtypes = [I, P, P, P, P, P, I, I, P, I, P, P, P, P]
    lib.oracle_rows.restype = I
    lib.oracle_gpu_row_split.argtypes = [I, I, I, ctypes.POINTER(I), ctypes.POINTER(I)]
    lib.oracle_gpu_row_split.restype = None
    lib.oracle_cpu_row_split.argtypes = [I, I, P]
    lib.oracle_cpu_row_split.restype = None
    lib.oracle_max_threads.argtypes = []
    lib.oracle_max_threads.restype = I
    _lib = lib
    return lib


def _c(a, dtype=np.float64):
    return np.ascontiguousarray(a, dtype=dtype)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def max_threads() -> int:
    return int(load().oracle_max_threads())


def triangle(x, y, z, m, range2, nkernel=0, i_lo=0, i_hi=None, nthreads=None):
    """Faithful cpu_grav.f triangle over rows [i_lo, i_hi); returns gx, gy, gz, grpot."""
    x, y, z, m, range2 = (_c(a) for a in (x, y, z, m, range2))
    n = x.shape[0]
    i_hi = n if i_hi is None else i_hi
    nthreads = max_threads() if nthreads is None else nthreads
    out = [np.zeros(n) for _ in range(4)]
    rc = load().oracle_triangle(n, _p(x), _p(y), _p(z), _p(m), _p(range2), int(nkernel), int(i_lo),
                                int(i_hi), int(nthreads), *(_p(a) for a in out))
    if rc:
        raise ValueError(f"oracle_triangle rejected the input (code {rc})")
    return tuple(out)


def rows(x, y, z, m, range2, nkernel=0, row_idx=None, nthreads=None):
    """Row form (compensated sums) for the listed rows; returns ax, ay, az, pot."""
    x, y, z, m, range2 = (_c(a) for a in (x, y, z, m, range2))
    n = x.shape[0]
    idx = np.arange(n, dtype=np.int32) if row_idx is None else _c(row_idx, np.int32)
    nthreads = max_threads() if nthreads is None else nthreads
    out = [np.zeros(idx.shape[0]) for _ in range(4)]
    rc = load().oracle_rows(n, _p(x), _p(y), _p(z), _p(m), _p(range2), int(nkernel),
                            int(idx.shape[0]), _p(idx), int(nthreads), *(_p(a) for a in out))
    if rc:
        raise ValueError(f"oracle_rows rejected the input (code {rc})")
    return tuple(out)


def gpu_row_split(n: int, nranks: int, rank: int):
    lo, hi = ctypes.c_int(), ctypes.c_int()
    load().oracle_gpu_row_split(n, nranks, rank, ctypes.byref(lo), ctypes.byref(hi))
    return lo.value, hi.value


def cpu_row_split(n: int, nranks: int):
    b = np.zeros(nranks + 1, dtype=np.int32)
    load().oracle_cpu_row_split(n, nranks, _p(b))
    return b
