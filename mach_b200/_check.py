"""Contiguity helpers (mirror of mach's src/mach/_check.py:10-41)."""

from __future__ import annotations

import warnings
from typing import Any

import numpy as np

from mach_b200 import _dlpack
from mach_b200._array_api import array_namespace


def is_contiguous(array: Any) -> bool:
    """True if C-contiguous.  Like mach, optimistic for types without a layout query."""
    if isinstance(array, np.ndarray):
        return bool(array.flags["C_CONTIGUOUS"])
    if _dlpack.is_torch(array):
        return bool(array.is_contiguous())
    return True


def ensure_contiguous(array: Any, *, warn: bool = True) -> Any:
    """Return a C-contiguous array, warning when a copy is made (src/mach/_check.py:25-41)."""
    if is_contiguous(array):
        return array
    if warn:
        warnings.warn("array is not contiguous, rearranging will add latency", stacklevel=2)
    return array_namespace(array).ascontiguousarray(array)
