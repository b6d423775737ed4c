"""CPU tests of the drop-in boundary: the library loads and exports every
function declared in include/sphgrav_b200.h (no GPU compute here)."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT
from starsmasher_b200 import _lib

HEADER = os.path.join(ROOT, "include", "sphgrav_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_header_declares_reference_symbols():
    names = declared_functions()
    for legacy in ("firsthalf_grav_forces_", "lasthalf_grav_forces_", "gpu_init_dev_"):
        assert legacy in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(line.split()[-1] for line in out.splitlines() if " T " in line)
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)


def test_python_binding_covers_the_header():
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_fortran_module_binds_declared_symbols():
    """Every bind(C) name of the Fortran interface module is a declared,
    exported symbol, and its precision constants match the header's enum (no
    Fortran compiler here: the module is checked as text)."""
    f90 = open(os.path.join(ROOT, "starsmasher_b200", "fortran", "sphgrav_b200_mod.f90")).read()
    bound = re.findall(r'bind\(C,\s*name="(\w+)"\)', f90)
    assert len(bound) >= 10
    declared = set(declared_functions())
    for name in bound:
        assert name in declared, name
    hdr = open(HEADER).read()
    for const in ("SPHGRAV_FP64", "SPHGRAV_F32SPLIT", "SPHGRAV_TREE"):
        want = re.search(rf"{const}\s*=\s*(\d+)", hdr).group(1)
        got = re.search(rf"{const}\s*=\s*(\d+)", f90).group(1)
        assert got == want, const


def test_static_archive_for_fortran_link():
    a = os.path.join(os.path.dirname(_lib.LIB_PATH), "libSPHgrav.a")
    assert os.path.exists(a)
    out = subprocess.run(["nm", a], capture_output=True, text=True, check=True).stdout
    for sym in ("firsthalf_grav_forces_", "lasthalf_grav_forces_", "gpu_init_dev_"):
        assert re.search(rf" T {sym}$", out, flags=re.M), sym


def test_status_strings_and_variants():
    lib = _lib.load()
    assert lib.sphgrav_status_string(0) == b"ok"
    assert lib.sphgrav_status_string(2) == b"invalid particle data"
    assert lib.sphgrav_variant_count(0) >= 1
    assert lib.sphgrav_variant_count(1) >= 1
    assert lib.sphgrav_variant_count(7) == 0
    assert lib.sphgrav_variant_name(1, 0).startswith(b"f32split")


def test_invalid_arguments_are_rejected_without_a_device():
    lib = _lib.load()
    assert lib.sphgrav_create(None, 0) == _lib.ERR_INVALID_ARGUMENT
    assert lib.sphgrav_sync(None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.sphgrav_lasthalf(None, None, None, None, None) == _lib.ERR_INVALID_ARGUMENT
    assert lib.sphgrav_legacy_set_precision(9) == _lib.ERR_INVALID_ARGUMENT


def test_create_without_gpu_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.sphgrav_create(ctypes.byref(h), 0) == _lib.ERR_NO_DEVICE
    assert not h.value
