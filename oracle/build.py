"""Build recipe for the checkers under oracle/ (test infrastructure only).

* ``oracle/_build/libdas_oracle.so`` -- the FP64 C restatement (das_oracle.c), gcc + OpenMP.
* ``oracle/_ref/libmachref.so``      -- mach's own CUDA kernel, compiled for sm_100a from the
  unmodified reference source ``src/mach/kernel.cu`` where it lies in the reference
  checkout, with the nanobind stand-in headers in ``oracle/ref_shim/``.  Only built when
  the reference checkout is present; the built file travels with the repository
  snapshot to the GPU machine.

Run ``python oracle/build.py`` (or call :func:`build_all`).
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD_DIR = HERE / "_build"
REF_DIR = HERE / "_ref"
ORACLE_LIB = BUILD_DIR / "libdas_oracle.so"
REF_LIB = REF_DIR / "libmachref.so"
# The mach checkout: MACH_REFERENCE_ROOT, else a checkout named "reference" beside this repository.
REFERENCE_ROOT = Path(os.environ.get("MACH_REFERENCE_ROOT", HERE.parent.parent / "reference"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources if s.exists())


def build_oracle(force: bool = False) -> Path:
    src = HERE / "das_oracle.c"
    if force or _stale(ORACLE_LIB, [src]):
        BUILD_DIR.mkdir(exist_ok=True)
        cmd = ["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-std=gnu11", "-o", str(ORACLE_LIB), str(src), "-lm"]
        subprocess.run(cmd, check=True)
    return ORACLE_LIB


def _nvcc_version() -> str:
    out = subprocess.run([NVCC, "--version"], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        if "release" in line and ", V" in line:
            return line.rsplit(", V", 1)[1].strip()
    return "0.0.0"


def build_reference(force: bool = False) -> Path | None:
    """Compile the reference kernel; returns None when the reference checkout is absent."""
    kernel = REFERENCE_ROOT / "src" / "mach" / "kernel.cu"
    if not kernel.exists():
        return REF_LIB if REF_LIB.exists() else None
    shim = HERE / "ref_shim" / "machref_shim.cu"
    stubs = [HERE / "ref_shim" / "nanobind" / "nanobind.h", HERE / "ref_shim" / "nanobind" / "ndarray.h"]
    if not (force or _stale(REF_LIB, [kernel, shim, *stubs])):
        return REF_LIB
    REF_DIR.mkdir(exist_ok=True)
    ver = _nvcc_version()
    major, minor = ver.split(".")[:2]
    cmd = [
        NVCC,
        "-std=c++17",
        "-O3",
        "--generate-line-info",
        "-gencode",
        "arch=compute_100a,code=sm_100a",
        "-Xcompiler",
        "-fPIC",
        "-shared",
        f"-I{HERE / 'ref_shim'}",
        f"-I{REFERENCE_ROOT / 'src' / 'mach' / 'vendor'}",
        f"-I{REFERENCE_ROOT / 'src' / 'mach'}",
        f'-DNVCC_VERSION_STR="{ver}"',
        f"-DNVCC_MAJOR={major}",
        f"-DNVCC_MINOR={minor}",
        "-o",
        str(REF_LIB),
        str(shim),
    ]
    subprocess.run(cmd, check=True)
    return REF_LIB


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_LIB, REF_LIB if REF_LIB.exists() else "(reference not built)")
