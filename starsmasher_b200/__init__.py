"""B200-native direct-summation SPH self-gravity (StarSmasher SPHgrav_lib2 replacement).

The product is the CUDA library ``libsphgrav_b200.so`` (C-ABI in
``include/sphgrav_b200.h``); this package binds it (``api``), generates seeded
workloads (``inputs``) and reads StarSmasher dumps (``snapshot``).
"""
from .api import (Context, Graph, firsthalf_grav_forces, gpu_init_dev, lasthalf_grav_forces,
                  launch_count, set_legacy_precision, variant_names)
from ._lib import F32SPLIT, FP64, LIB_PATH, SphgravError, load

__all__ = [
    "Context", "Graph", "firsthalf_grav_forces", "gpu_init_dev", "lasthalf_grav_forces",
    "launch_count", "set_legacy_precision", "variant_names", "F32SPLIT", "FP64", "LIB_PATH",
    "SphgravError", "load",
]
