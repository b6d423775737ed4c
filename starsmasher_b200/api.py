"""Python host API over the C-ABI.

Two layers:
  * module functions with the reference's Fortran-facing names and argument
    meaning -- ``gpu_init_dev``, ``firsthalf_grav_forces``,
    ``lasthalf_grav_forces`` (grav_force_direct.cu:648-677; callers grav.f:25,
    balAV3.f:418, main.f:270) -- and ``gravforce`` (grav.f:1-26 plus the
    lasthalf call of balAV3.f:418);
  * ``Context``: the status-returning API, device-resident and batched calls,
    graph capture and tuning.

Host arrays are numpy float64; device arrays are anything exposing
``data_ptr()`` (torch CUDA tensors) or plain integer device pointers.
"""
from __future__ import annotations

import ctypes
from contextlib import contextmanager
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import F32SPLIT, FP64, TREE, check, load

PRECISIONS = {"fp64": FP64, "f32split": F32SPLIT, "tree": TREE, FP64: FP64, F32SPLIT: F32SPLIT,
              TREE: TREE}


def _prec(p) -> int:
    try:
        return PRECISIONS[p]
    except KeyError:
        raise ValueError(f"unknown precision {p!r}") from None


def _host(a, n: Optional[int] = None, writable: bool = False) -> np.ndarray:
    arr = np.ascontiguousarray(a, dtype=np.float64)
    if writable and arr is not a:
        raise TypeError("output arrays must be contiguous float64 numpy arrays")
    if n is not None and arr.shape[0] < n:
        raise ValueError(f"array of length {arr.shape[0]} < {n}")
    return arr


def _hp(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def _dp(t) -> ctypes.c_void_p:
    if t is None:
        return ctypes.c_void_p(0)
    if isinstance(t, int):
        return ctypes.c_void_p(t)
    return ctypes.c_void_p(t.data_ptr())


class Graph:
    """A captured CUDA graph of context calls (replay with ``launch``)."""

    def __init__(self, handle: ctypes.c_void_p):
        self._h = handle

    def launch(self, repeats: int = 1) -> None:
        check(load().sphgrav_graph_launch(self._h, int(repeats)), "sphgrav_graph_launch")

    @property
    def valid(self) -> bool:
        """False once a call on its context changed the work plan or buffers
        (other sizes, precision or variant) or the context was destroyed."""
        return bool(self._h) and bool(load().sphgrav_graph_valid(self._h))

    def close(self) -> None:
        if self._h:
            load().sphgrav_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One device, one stream, grow-only device buffers (sphgrav_create)."""

    def __init__(self, device: int = 0):
        self._lib = load()
        h = ctypes.c_void_p()
        check(self._lib.sphgrav_create(ctypes.byref(h), int(device)), "sphgrav_create")
        self._h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.sphgrav_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ----------------------------------------------------------- plumbing
    def set_stream(self, stream) -> None:
        """Run on an external cudaStream_t (int handle, or torch.cuda.Stream)."""
        ptr = getattr(stream, "cuda_stream", stream)
        check(self._lib.sphgrav_set_stream(self._h, ctypes.c_void_p(ptr or 0)), "sphgrav_set_stream")

    def sync(self) -> None:
        check(self._lib.sphgrav_sync(self._h), "sphgrav_sync")

    def force_variant(self, precision, variant: int) -> None:
        check(self._lib.sphgrav_force_variant(self._h, _prec(precision), int(variant)),
              "sphgrav_force_variant")

    def set_theta(self, theta: float) -> None:
        """Tree mode: opening angle (default 0.3; 0 opens every node)."""
        check(self._lib.sphgrav_set_theta(self._h, float(theta)), "sphgrav_set_theta")

    def tree_stats(self) -> tuple:
        """Tree mode: (walking groups, groups handed to the direct FP64 sum) of the last call."""
        g, h = ctypes.c_int(0), ctypes.c_int(0)
        check(self._lib.sphgrav_tree_stats(self._h, ctypes.byref(g), ctypes.byref(h)), "sphgrav_tree_stats")
        return g.value, h.value

    def set_fp64_band(self, factor: float) -> None:
        """Split-FP32: evaluate pairs with r < factor * max(H) in FP64 (default 1)."""
        check(self._lib.sphgrav_set_fp64_band(self._h, float(factor)), "sphgrav_set_fp64_band")

    def set_refine(self, threshold: float) -> None:
        """Split-FP32: recompute in FP64 the rows whose error scale G exceeds
        threshold * |a| (default 1.0; 0 turns the refine off)."""
        check(self._lib.sphgrav_set_refine(self._h, float(threshold)), "sphgrav_set_refine")

    def last_refine_rows(self) -> int:
        """Rows the last split-FP32 call recomputed in FP64 (synchronises)."""
        v = ctypes.c_longlong(0)
        check(self._lib.sphgrav_last_refine_rows(self._h, ctypes.byref(v)), "sphgrav_last_refine_rows")
        return int(v.value)

    def keep_error_scale(self, on: bool = True) -> None:
        """Keep the per-row error scale G of later split-FP32 calls."""
        check(self._lib.sphgrav_keep_error_scale(self._h, 1 if on else 0), "sphgrav_keep_error_scale")

    def error_scale(self, n: int) -> np.ndarray:
        """G of the last split-FP32 call (caller order, all n particles)."""
        out = np.zeros(n)
        check(self._lib.sphgrav_error_scale(self._h, int(n), _hp(out)), "sphgrav_error_scale")
        return out

    def plan_info(self) -> dict:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._lib.sphgrav_last_plan_info(self._h, ctypes.byref(a), ctypes.byref(b),
                                               ctypes.byref(c)), "sphgrav_last_plan_info")
        return {"nitems": a.value, "nchunks_max": b.value, "variant": c.value}

    # ----------------------------------------------------- host buffers
    def firsthalf(self, x, y, z, mass, range2, nkernel: int = 0, precision="f32split",
                  i_begin: int = 0, ni: Optional[int] = None) -> None:
        x, y, z, mass, range2 = (_host(a) for a in (x, y, z, mass, range2))
        n = x.shape[0]
        ni = n - i_begin if ni is None else ni
        self._keep = (x, y, z, mass, range2)
        check(self._lib.sphgrav_firsthalf(self._h, n, i_begin, ni, _hp(x), _hp(y), _hp(z),
                                          _hp(mass), _hp(range2), int(nkernel), _prec(precision)),
              "sphgrav_firsthalf")
        self._pending = (n, i_begin, ni)

    def lasthalf(self, ax=None, ay=None, az=None, pot=None):
        n = self._pending[0]
        outs = [np.zeros(n) if a is None else a for a in (ax, ay, az, pot)]
        for a in outs:
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError("outputs must be contiguous float64 arrays")
        check(self._lib.sphgrav_lasthalf(self._h, *(_hp(a) for a in outs)), "sphgrav_lasthalf")
        return tuple(outs)

    def forces(self, x, y, z, mass, range2, nkernel: int = 0, precision="f32split",
               i_begin: int = 0, ni: Optional[int] = None):
        """firsthalf + lasthalf: returns (ax, ay, az, pot), length n (rows filled)."""
        self.firsthalf(x, y, z, mass, range2, nkernel, precision, i_begin, ni)
        return self.lasthalf()

    def gravforce(self, x, y, z, am, hp, u, ngrav_lower: int = 1, ngrav_upper: Optional[int] = None,
                  nkernel: int = 0, precision="f32split"):
        x, y, z, am, hp, u = (_host(a) for a in (x, y, z, am, hp, u))
        n = x.shape[0]
        ngrav_upper = n if ngrav_upper is None else ngrav_upper
        outs = [np.zeros(n) for _ in range(4)]
        check(self._lib.sphgrav_gravforce(self._h, n, ngrav_lower, ngrav_upper, _hp(x), _hp(y),
                                          _hp(z), _hp(am), _hp(hp), _hp(u), int(nkernel),
                                          _prec(precision), *(_hp(a) for a in outs)),
              "sphgrav_gravforce")
        return tuple(outs)

    def gravforce_device(self, ntot: int, x, y, z, am, hp, u, gx, gy, gz, grpot,
                         ngrav_lower: int = 1, ngrav_upper: Optional[int] = None,
                         nkernel: int = 0, precision="f32split") -> None:
        """Device-resident gravforce: range2 built on the device, rows
        [ngrav_lower, ngrav_upper] (1-based) of gx, gy, gz, grpot written."""
        ngrav_upper = ntot if ngrav_upper is None else ngrav_upper
        check(self._lib.sphgrav_gravforce_device(self._h, int(ntot), int(ngrav_lower), int(ngrav_upper),
                                                 _dp(x), _dp(y), _dp(z), _dp(am), _dp(hp), _dp(u),
                                                 int(nkernel), _prec(precision), _dp(gx), _dp(gy),
                                                 _dp(gz), _dp(grpot)),
              "sphgrav_gravforce_device")

    def batch_forces(self, offsets: Sequence[int], x, y, z, mass, range2, nkernel: int = 0,
                     precision="f32split"):
        offs = np.ascontiguousarray(offsets, dtype=np.int32)
        x, y, z, mass, range2 = (_host(a) for a in (x, y, z, mass, range2))
        n = int(offs[-1])
        outs = [np.zeros(n) for _ in range(4)]
        W = np.zeros(len(offs) - 1)
        check(self._lib.sphgrav_batch_forces(self._h, len(offs) - 1, _hp(offs), _hp(x), _hp(y),
                                             _hp(z), _hp(mass), _hp(range2), int(nkernel),
                                             _prec(precision), *(_hp(a) for a in outs), _hp(W)),
              "sphgrav_batch_forces")
        return (*outs, W)

    # --------------------------------------------------- device buffers
    def forces_device(self, n: int, x, y, z, mass, range2, ax, ay, az, pot, W=None,
                      nkernel: int = 0, precision="f32split", i_begin: int = 0,
                      ni: Optional[int] = None) -> None:
        ni = n - i_begin if ni is None else ni
        check(self._lib.sphgrav_forces_device(self._h, int(n), int(i_begin), int(ni), _dp(x),
                                              _dp(y), _dp(z), _dp(mass), _dp(range2),
                                              int(nkernel), _prec(precision), _dp(ax), _dp(ay),
                                              _dp(az), _dp(pot), _dp(W)),
              "sphgrav_forces_device")

    def batch_forces_device(self, offsets: Sequence[int], x, y, z, mass, range2, ax, ay, az, pot,
                            W=None, nkernel: int = 0, precision="f32split") -> None:
        offs = np.ascontiguousarray(offsets, dtype=np.int32)
        check(self._lib.sphgrav_batch_forces_device(self._h, len(offs) - 1, _hp(offs), _dp(x),
                                                    _dp(y), _dp(z), _dp(mass), _dp(range2),
                                                    int(nkernel), _prec(precision), _dp(ax),
                                                    _dp(ay), _dp(az), _dp(pot), _dp(W)),
              "sphgrav_batch_forces_device")

    def kick_device(self, n: int, x, y, z, sigma: float, seed: int) -> None:
        check(self._lib.sphgrav_kick_positions_device(self._h, int(n), _dp(x), _dp(y), _dp(z),
                                                      float(sigma), int(seed)),
              "sphgrav_kick_positions_device")

    def kick_reset(self, counter: int = 0) -> None:
        check(self._lib.sphgrav_kick_reset(self._h, int(counter)), "sphgrav_kick_reset")

    @contextmanager
    def capture(self):
        """``with ctx.capture() as cap: ...`` then ``cap.graph.launch(n)``."""
        check(self._lib.sphgrav_capture_begin(self._h), "sphgrav_capture_begin")

        class _Cap:
            graph: Optional[Graph] = None

        cap = _Cap()
        ok = False
        try:
            yield cap
            ok = True
        finally:
            g = ctypes.c_void_p()
            st = self._lib.sphgrav_capture_end(self._h, ctypes.byref(g))
            if ok:
                check(st, "sphgrav_capture_end")
                cap.graph = Graph(g)
            elif g:
                self._lib.sphgrav_graph_destroy(g)

    # ------------------------------------------------------------ tuning
    def autotune(self, offsets, x, y, z, mass, range2, nkernel: int = 0, precision="f32split"):
        offs = np.ascontiguousarray(offsets, dtype=np.int32)
        check(self._lib.sphgrav_autotune(self._h, len(offs) - 1, _hp(offs), _dp(x), _dp(y),
                                         _dp(z), _dp(mass), _dp(range2), int(nkernel),
                                         _prec(precision)), "sphgrav_autotune")

    def tuning_save(self, path: str) -> None:
        check(self._lib.sphgrav_tuning_save(self._h, path.encode()), "sphgrav_tuning_save")

    def tuning_load(self, path: str) -> None:
        check(self._lib.sphgrav_tuning_load(self._h, path.encode()), "sphgrav_tuning_load")

    def profile_enable(self, on: bool = True) -> None:
        check(self._lib.sphgrav_profile_enable(self._h, int(bool(on))), "sphgrav_profile_enable")

    def profile_read(self):
        """(summed pair-kernel ms, launches) since the last read."""
        ms, n = ctypes.c_double(), ctypes.c_int()
        check(self._lib.sphgrav_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n)),
              "sphgrav_profile_read")
        return ms.value, n.value

    PHASES = ("item", "rows", "wait_full", "far", "checked", "near", "end",
              "producer_wait", "producer_work", "n_far", "n_checked", "n_near", "n_items")

    def phase_read(self) -> dict:
        """Split-FP32 phase cycles summed over warps since the last read (the
        diagnostic build only; the default build raises SphgravError with
        status ERR_UNSUPPORTED).  Counted while profiling is enabled."""
        buf = (ctypes.c_ulonglong * 16)()
        check(self._lib.sphgrav_phase_read(self._h, buf, 16), "sphgrav_phase_read")
        return {k: int(buf[i]) for i, k in enumerate(self.PHASES)}

    def fp32_peak_probe(self, iters: int = 20000) -> float:
        t = ctypes.c_double()
        check(self._lib.sphgrav_fp32_peak_probe(self._h, int(iters), ctypes.byref(t)),
              "sphgrav_fp32_peak_probe")
        return t.value

    def selftest_wait_timeout(self, polls: int = 1024) -> int:
        """Run the device-timeout self-test; returns its status
        (ERR_DEVICE_TIMEOUT when the failure path works)."""
        return int(self._lib.sphgrav_selftest_wait_timeout(self._h, int(polls)))

    def fp64_peak_probe(self, iters: int = 20000) -> float:
        t = ctypes.c_double()
        check(self._lib.sphgrav_fp64_peak_probe(self._h, int(iters), ctypes.byref(t)),
              "sphgrav_fp64_peak_probe")
        return t.value


def variant_names(precision) -> list:
    lib = load()
    p = _prec(precision)
    return [lib.sphgrav_variant_name(p, v).decode() for v in range(lib.sphgrav_variant_count(p))]


def launch_count() -> int:
    return int(load().sphgrav_launch_count())


def plan_preview(offsets: Sequence[int], precision="f32split", variant: int = 0,
                 resident: int = 148) -> dict:
    """The work plan of a call on whole sets, computed on the host (no GPU):
    {"nitems", "nslots", "items"}; items is an (nitems, 6) int array of
    (set, row tile, chunk, partial slot, first source, end source) in queue
    order, `resident` persistent CTAs."""
    lib = load()
    offs = np.ascontiguousarray(offsets, dtype=np.int32)
    ni, ns = ctypes.c_int(), ctypes.c_int()
    check(lib.sphgrav_plan_preview(len(offs) - 1, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   _prec(precision), int(variant), int(resident),
                                   ctypes.byref(ni), ctypes.byref(ns), None, 0),
          "sphgrav_plan_preview")
    items = np.zeros((max(ni.value, 1), 6), dtype=np.int32)
    check(lib.sphgrav_plan_preview(len(offs) - 1, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   _prec(precision), int(variant), int(resident),
                                   ctypes.byref(ni), ctypes.byref(ns),
                                   items.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ni.value),
          "sphgrav_plan_preview")
    return {"nitems": ni.value, "nslots": ns.value, "items": items[:ni.value]}


# ------------------------------------------- reference-named module functions
def gpu_init_dev(myrank: int, theta: float = 0.3) -> None:
    """gpu_init_dev(myrank, theta) of main.f:265-275: select device ``myrank``."""
    r = ctypes.c_int(myrank)
    t = ctypes.c_double(theta)
    load().gpu_init_dev_(ctypes.byref(r), ctypes.byref(t))


def set_legacy_precision(precision) -> None:
    check(load().sphgrav_legacy_set_precision(_prec(precision)), "sphgrav_legacy_set_precision")


_legacy_keep = None


def firsthalf_grav_forces(ntot: int, ngrav_lower: int, mygravlength: int, x, y, z, am, range2,
                          q: int = 1, nkernel: int = 0) -> None:
    """The Fortran call of grav.f:25-26 (1-based ngrav_lower)."""
    global _legacy_keep
    arrs = [_host(a, ntot) for a in (x, y, z, am, range2)]
    _legacy_keep = arrs
    P = ctypes.POINTER(ctypes.c_double)
    ia = [ctypes.c_int(v) for v in (ntot, ngrav_lower, mygravlength, q, nkernel)]
    load().firsthalf_grav_forces_(ctypes.byref(ia[0]), ctypes.byref(ia[1]), ctypes.byref(ia[2]),
                                  *(a.ctypes.data_as(P) for a in arrs), ctypes.byref(ia[3]),
                                  ctypes.byref(ia[4]))


def lasthalf_grav_forces(ntot: int, gx: np.ndarray, gy: np.ndarray, gz: np.ndarray,
                         grpot: np.ndarray) -> None:
    """The Fortran call of balAV3.f:418: fills the rows listed by firsthalf."""
    for a in (gx, gy, gz, grpot):
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                and a.shape[0] >= ntot):
            raise TypeError("outputs must be contiguous float64 arrays of length ntot")
    P = ctypes.POINTER(ctypes.c_double)
    n = ctypes.c_int(ntot)
    # five arguments, as the Fortran caller passes: myrank is never read
    load().lasthalf_grav_forces_(ctypes.byref(n), *(a.ctypes.data_as(P) for a in (gx, gy, gz, grpot)),
                                 None)
