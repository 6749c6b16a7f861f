"""Compile the mach_b200 CUDA library in-tree: ``mach_b200/libmach_b200.so`` (sm_100a).

Each ``*.cu`` in this folder becomes an object file (compiled in parallel), then one
shared library is linked.  ``python -m mach_b200.csrc.build`` or :func:`build`.
"""

from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PKG = CSRC.parent
REPO = PKG.parent
OBJ_DIR = REPO / "_build" / "mach_b200"
LIB_PATH = PKG / "libmach_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_version() -> str:
    out = subprocess.run([NVCC, "--version"], check=True, capture_output=True, text=True).stdout
    for line in out.splitlines():
        if "release" in line and ", V" in line:
            return line.rsplit(", V", 1)[1].strip()
    return "0.0.0"


def _flags() -> list[str]:
    return [
        "-std=c++17",
        "-O3",
        "-lineinfo",
        *ARCH,
        "-Xcompiler",
        "-fPIC",
        "-Xcompiler",
        "-fvisibility=hidden",
        f"-I{REPO / 'include'}",
        f"-I{CSRC}",
        f'-DMACH_B200_NVCC_VERSION="{nvcc_version()}"',
        "-Xptxas",
        "-v" if os.environ.get("MACH_B200_PTXAS_VERBOSE") else "-O3",
    ]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + [REPO / "include" / "mach_b200.h"]


def _compile(src: Path, flags: list[str], force: bool) -> tuple[Path, str]:
    obj = OBJ_DIR / (src.stem + ".o")
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if not force and obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj, ""
    cmd = [NVCC, *flags, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    return obj, res.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    flags = _flags()
    sources = sorted(CSRC.glob("*.cu"))
    jobs = max(1, min(len(sources), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(jobs) as pool:
        results = list(pool.map(lambda s: _compile(s, flags, force), sources))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log, file=sys.stderr)
    if force or not LIB_PATH.exists() or any(o.stat().st_mtime > LIB_PATH.stat().st_mtime for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB_PATH), *map(str, objs)]
        subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
