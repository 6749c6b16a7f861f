"""The C ABI library loads, exports every symbol include/mach_b200.h declares, and rejects
bad arguments before touching the GPU (these checks run without a GPU)."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
HEADER = REPO / "include" / "mach_b200.h"
LIB = REPO / "mach_b200" / "libmach_b200.so"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    return re.findall(r"MACH_B200_API\s+[\w\s\*]+?\b(mach_b200_\w+)\s*\(", text)


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("mach_b200_beamform_f32", "mach_b200_beamform_c64", "mach_b200_beamform_compound",
              "mach_b200_last_error"):
        assert n in names


def test_library_exports_declared_symbols():
    lib = ctypes.CDLL(str(LIB))
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\b(mach_b200_\w+)\b", out))
    assert exported == set(declared_symbols())


def test_library_is_built_for_sm100a():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", str(LIB)], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def _lib():
    lib = ctypes.CDLL(str(LIB))
    lib.mach_b200_last_error.restype = ctypes.c_char_p
    lib.mach_b200_nvcc_version.restype = ctypes.c_char_p
    f = lib.mach_b200_beamform_compound
    f.restype = ctypes.c_int
    F, P, U32 = ctypes.c_float, ctypes.c_void_p, ctypes.c_uint32
    f.argtypes = [ctypes.c_int32, P, P, P, P, P, U32, U32, U32, ctypes.c_uint64, U32, F, F, F, F, F, F,
                  ctypes.c_int32, F, P, U32]
    return lib


def _call(lib, storage=1, alpha=0.5, interp=1, n_vox=4, out=1):
    return lib.mach_b200_beamform_compound(storage, 1, 1, 1, 1, out, 1, 1, 1, n_vox, 1, 1.0, 0.0, 1e6, 1540.0,
                                           0.0, alpha, interp, 1.0, None, 0)


def test_rejects_bad_arguments_without_gpu():
    lib = _lib()
    assert _call(lib, alpha=1.5) == 1
    assert b"tukey_alpha must be in range [0, 1]" in lib.mach_b200_last_error()
    assert _call(lib, alpha=-0.1) == 1
    assert _call(lib, storage=9) == 1
    assert b"storage" in lib.mach_b200_last_error()
    assert _call(lib, interp=3) == 1
    assert b"interp_type" in lib.mach_b200_last_error()
    assert _call(lib, out=None) == 1
    assert _call(lib, n_vox=0) == 0  # empty output: nothing to do


def test_nvcc_version_string():
    v = _lib().mach_b200_nvcc_version().decode()
    major, minor, _ = v.split(".")
    assert int(major) >= 12 and int(minor) >= 0
