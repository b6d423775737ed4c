"""ctypes binding of libsphgrav_b200.so (the C-ABI declared in include/sphgrav_b200.h).

The library is built in-tree (``python -m starsmasher_b200.build``).  Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# SPHGRAV_B200_BUILD=phases loads the diagnostic build whose split-FP32 kernel
# counts cycles per phase (`python -m starsmasher_b200.build --phases`)
_BUILDS = {"": "libsphgrav_b200.so", "default": "libsphgrav_b200.so",
           "phases": "libsphgrav_b200_phases.so"}
LIB_PATH = os.path.join(HERE, _BUILDS[os.environ.get("SPHGRAV_B200_BUILD", "")])

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_INVALID_INPUT = 2
ERR_CUDA = 3
ERR_NO_DEVICE = 4
ERR_OUT_OF_MEMORY = 5
ERR_PROTOCOL = 6
ERR_DEVICE_TIMEOUT = 7
ERR_TOO_LARGE = 8
ERR_UNSUPPORTED = 9

FP64 = 0
F32SPLIT = 1
TREE = 2

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); the complete exported C-ABI.
SIGNATURES = {
    "firsthalf_grav_forces_": (None, [_PI, _PI, _PI, _PD, _PD, _PD, _PD, _PD, _PI, _PI]),
    "lasthalf_grav_forces_": (None, [_PI, _PD, _PD, _PD, _PD, _PI]),
    "gpu_init_dev_": (None, [_PI, _PD]),
    "sphgrav_legacy_set_precision": (_I, [_I]),
    "sphgrav_create": (_I, [ctypes.POINTER(_P), _I]),
    "sphgrav_destroy": (_I, [_P]),
    "sphgrav_set_stream": (_I, [_P, _P]),
    "sphgrav_sync": (_I, [_P]),
    "sphgrav_firsthalf": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _I, _I]),
    "sphgrav_lasthalf": (_I, [_P, _P, _P, _P, _P]),
    "sphgrav_forces_device": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P]),
    "sphgrav_batch_forces_device": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P]),
    "sphgrav_batch_forces": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P, _P]),
    "sphgrav_gravforce": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
    "sphgrav_gravforce_device": (_I, [_P, _I, _I, _I, _P, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P, _P]),
    "sphgrav_kick_positions_device": (_I, [_P, _I, _P, _P, _P, _D, ctypes.c_ulonglong]),
    "sphgrav_kick_reset": (_I, [_P, ctypes.c_ulonglong]),
    "sphgrav_capture_begin": (_I, [_P]),
    "sphgrav_capture_end": (_I, [_P, ctypes.POINTER(_P)]),
    "sphgrav_graph_launch": (_I, [_P, _I]),
    "sphgrav_graph_valid": (_I, [_P]),
    "sphgrav_graph_destroy": (_I, [_P]),
    "sphgrav_autotune": (_I, [_P, _I, _P, _P, _P, _P, _P, _P, _I, _I]),
    "sphgrav_tuning_save": (_I, [_P, ctypes.c_char_p]),
    "sphgrav_tuning_load": (_I, [_P, ctypes.c_char_p]),
    "sphgrav_force_variant": (_I, [_P, _I, _I]),
    "sphgrav_set_fp64_band": (_I, [_P, _D]),
    "sphgrav_set_refine": (_I, [_P, _D]),
    "sphgrav_last_refine_rows": (_I, [_P, ctypes.POINTER(ctypes.c_longlong)]),
    "sphgrav_keep_error_scale": (_I, [_P, _I]),
    "sphgrav_error_scale": (_I, [_P, _I, _P]),
    "sphgrav_set_theta": (_I, [_P, _D]),
    "sphgrav_tree_stats": (_I, [_P, _PI, _PI]),
    "sphgrav_variant_count": (_I, [_I]),
    "sphgrav_variant_name": (ctypes.c_char_p, [_I, _I]),
    "sphgrav_status_string": (ctypes.c_char_p, [_I]),
    "sphgrav_last_error_message": (ctypes.c_char_p, []),
    "sphgrav_launch_count": (ctypes.c_ulonglong, []),
    "sphgrav_last_plan_info": (_I, [_P, _PI, _PI, _PI]),
    "sphgrav_fp32_peak_probe": (_I, [_P, _I, _PD]),
    "sphgrav_fp64_peak_probe": (_I, [_P, _I, _PD]),
    "sphgrav_selftest_wait_timeout": (_I, [_P, _I]),
    "sphgrav_forces_fp64_noalloc": (_I, [_I, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P]),
    "sphgrav_profile_enable": (_I, [_P, _I]),
    "sphgrav_profile_read": (_I, [_P, _PD, _PI]),
    "sphgrav_plan_preview": (_I, [_I, _PI, _I, _I, _I, _PI, _PI, _PI, _I]),
    "sphgrav_phase_read": (_I, [_P, ctypes.POINTER(ctypes.c_ulonglong), _I]),
}

_lib = None


class SphgravError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__(f"{where}: status {status}: {message}")


def load() -> ctypes.CDLL:
    """Load the in-tree library (once) and declare every C-ABI signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m starsmasher_b200.build` "
            "(the gravity path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != OK:
        lib = load()
        msg = lib.sphgrav_last_error_message().decode(errors="replace")
        raise SphgravError(status, where, msg)
