"""The ctypes mirrors of the C ABI's structs match include/mach_b200.h field by field.

A C program compiled with the host compiler against the header prints sizeof and offsetof of
every field of `mach_b200_options` and `mach_b200_job`; the Python structures that the
package passes through the C ABI (`_cuda_impl.Options`, `batch._Job`) must agree, or a
launch option or job field would be read from the wrong bytes.  No GPU is needed: the
library only has to load.
"""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _c_layout(tmp_path: Path, struct: str, fields: list[str]) -> dict[str, int]:
    lines = [f'printf("size %zu\\n", sizeof({struct}));']
    lines += [f'printf("{f} %zu\\n", offsetof({struct}, {f}));' for f in fields]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "mach_b200.h"\nint main(void) {\n'
                   + "\n".join(lines) + "\nreturn 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(REPO / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (line.split() for line in out.splitlines())}


def _check(tmp_path: Path, struct: str, cls) -> None:
    import ctypes

    fields = [name for name, *_ in cls._fields_]
    c = _c_layout(tmp_path, struct, fields)
    assert c["size"] == ctypes.sizeof(cls), f"sizeof({struct})"
    for name in fields:
        assert c[name] == getattr(cls, name).offset, f"{struct}.{name}"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_options_layout(tmp_path):
    from mach_b200 import _cuda_impl

    _check(tmp_path, "mach_b200_options", _cuda_impl.Options)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_job_layout(tmp_path):
    from mach_b200 import batch

    _check(tmp_path, "mach_b200_job", batch._Job)
