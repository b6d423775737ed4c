"""Build the B200 gravity library in-tree.

Outputs (next to this file):
  libsphgrav_b200.so  -- shared library: the C-ABI of include/sphgrav_b200.h
  libSPHgrav.a        -- static archive with the same objects, the name the
                         StarSmasher Makefile links (-lSPHgrav, plus -lcudart
                         -lstdc++), so the Fortran host relinks unchanged.

Every object is compiled for sm_100a only.  Usage: ``python -m starsmasher_b200.build``.

``--phases`` also builds libsphgrav_b200_phases.so, a diagnostic copy whose
split-FP32 kernel is compiled with -DSG_PHASES: its warps count SM cycles per
phase (sphgrav_phase_read); load it with SPHGRAV_B200_BUILD=phases.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["sg_prep.cu", "sg_f64.cu", "sg_f32.cu", "sg_refine.cu", "sg_tree.cu", "sg_api.cu",
           "sg_noalloc.cu"]
SO_NAME = "libsphgrav_b200.so"
PHASES_SO_NAME = "libsphgrav_b200_phases.so"
A_NAME = "libSPHgrav.a"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-v",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose: bool, extra=(), suffix: str = "") -> str:
    stem = os.path.splitext(src)[0] + suffix
    obj = os.path.join(OBJDIR, stem + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", CSRC, "-I", INCLUDE, "-c", os.path.join(CSRC, src),
           "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(OBJDIR, stem + ".ptxas.txt")
    with open(log, "w") as f:
        f.write(res.stdout + res.stderr)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"compiled {src}")
    return obj


def _stale(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(INCLUDE, "sphgrav_b200.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    so = os.path.join(HERE, SO_NAME)
    if not force and not _stale(so):
        return so
    os.makedirs(OBJDIR, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    tmp = so + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, so)
    a = os.path.join(HERE, A_NAME)
    if os.path.exists(a):
        os.remove(a)
    res = subprocess.run(["ar", "rcs", a, *objs], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"ar failed:\n{res.stderr}")
    return so


def build_phases(force: bool = False, verbose: bool = False) -> str:
    """The diagnostic library: the default objects with sg_f32.cu compiled
    with -DSG_PHASES."""
    so = os.path.join(HERE, PHASES_SO_NAME)
    if not force and not _stale(so):
        return so
    os.makedirs(OBJDIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        if src == "sg_f32.cu":
            continue
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        objs.append(obj if os.path.exists(obj) and not _stale(obj) else _compile(src, verbose))
    objs.append(_compile("sg_f32.cu", verbose, extra=("-DSG_PHASES",), suffix="_phases"))
    tmp = so + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, so)
    return so


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    if "--phases" in sys.argv:
        print(build_phases(force="--force" in sys.argv, verbose=True))
