"""Array-namespace helpers (mirror of mach's src/mach/_array_api.py).

mach resolves namespaces with ``array_api_compat``, which is not installed here.
This module does the small part mach needs for NumPy and PyTorch (and CuPy /
JAX when they are importable): dtype names, ``zeros``, ``astype``, contiguity,
and the math used by ``wavefront`` and ``geometry``.
"""

from __future__ import annotations

from enum import Enum
from typing import Any, Protocol, runtime_checkable

import numpy as np

from mach_b200 import _dlpack


class DLPackDevice(int, Enum):
    """DLPack device types used by mach (src/mach/_array_api.py:9-17)."""

    CPU = 1
    CUDA = 2


@runtime_checkable
class Array(Protocol):
    """Minimal array protocol (src/mach/_array_api.py:90-117)."""

    dtype: Any
    shape: tuple[int, ...]

    def __dlpack_device__(self, /) -> tuple[int, int]: ...


class _NumpyNS:
    name = "numpy"
    float32, float64, complex64, complex128 = np.float32, np.float64, np.complex64, np.complex128
    float16, int16 = np.float16, np.int16

    @staticmethod
    def zeros(shape, dtype, like=None):
        return np.zeros(shape, dtype=dtype)

    @staticmethod
    def astype(x, dtype, copy=False):
        return np.asarray(x).astype(dtype, copy=copy)

    @staticmethod
    def ascontiguousarray(x):
        return np.ascontiguousarray(x)

    @staticmethod
    def is_contiguous(x) -> bool:
        return bool(x.flags["C_CONTIGUOUS"])

    @staticmethod
    def is_complex(x) -> bool:
        return np.iscomplexobj(x)

    @staticmethod
    def is_numeric(x) -> bool:
        return np.issubdtype(x.dtype, np.number)

    @staticmethod
    def is_real(x) -> bool:
        return np.issubdtype(x.dtype, np.integer) or np.issubdtype(x.dtype, np.floating)

    asarray = staticmethod(np.asarray)
    stack = staticmethod(np.stack)
    sqrt = staticmethod(np.sqrt)
    sin = staticmethod(np.sin)
    cos = staticmethod(np.cos)
    sign = staticmethod(np.sign)
    abs = staticmethod(np.abs)

    @staticmethod
    def vecdot(a, b, axis=-1):
        return np.sum(np.asarray(a) * np.asarray(b), axis=axis)

    @staticmethod
    def vector_norm(x, axis=-1):
        x = np.asarray(x)
        return np.sqrt(np.sum(x * x, axis=axis))


class _TorchNS:
    name = "torch"

    def __init__(self):
        import torch

        self.torch = torch
        self.float32, self.float64 = torch.float32, torch.float64
        self.complex64, self.complex128 = torch.complex64, torch.complex128
        self.float16, self.int16, self.bfloat16 = torch.float16, torch.int16, torch.bfloat16

    def zeros(self, shape, dtype, like=None):
        device = like.device if like is not None and hasattr(like, "device") else None
        return self.torch.zeros(shape, dtype=dtype, device=device)

    def astype(self, x, dtype, copy=False):
        return x.to(dtype=dtype, copy=copy)

    def ascontiguousarray(self, x):
        return x.contiguous()

    def is_contiguous(self, x) -> bool:
        return bool(x.is_contiguous())

    def is_complex(self, x) -> bool:
        return bool(x.is_complex())

    def is_numeric(self, x) -> bool:
        return x.dtype != self.torch.bool

    def is_real(self, x) -> bool:
        return x.dtype != self.torch.bool and not x.is_complex()

    def asarray(self, x, like=None, dtype=None):
        device = like.device if like is not None and hasattr(like, "device") else None
        return self.torch.as_tensor(x, dtype=dtype, device=device)

    def stack(self, xs, axis=0):
        return self.torch.stack(list(xs), dim=axis)

    def sqrt(self, x):
        return self.torch.sqrt(x)

    def sin(self, x):
        return self.torch.sin(x)

    def cos(self, x):
        return self.torch.cos(x)

    def sign(self, x):
        return self.torch.sign(x)

    def abs(self, x):
        return self.torch.abs(x)

    def vecdot(self, a, b, axis=-1):
        return (a * b).sum(dim=axis)

    def vector_norm(self, x, axis=-1):
        return self.torch.linalg.vector_norm(x, dim=axis)


_NUMPY = _NumpyNS()
_TORCH = None


def array_namespace(*arrays: Any):
    """Namespace of the first array-like argument (NumPy default for scalars/lists)."""
    global _TORCH
    for a in arrays:
        if _dlpack.is_torch(a):
            if _TORCH is None:
                _TORCH = _TorchNS()
            return _TORCH
    for a in arrays:
        if isinstance(a, np.ndarray):
            return _NUMPY
    for a in arrays:
        if hasattr(a, "__dlpack__") and not isinstance(a, np.ndarray):
            raise TypeError(
                f"arrays of type {type(a).__name__} are accepted through DLPack only; "
                "convert them with torch.from_dlpack or numpy.from_dlpack first"
            )
    return _NUMPY


def is_writeable_array(x: Any) -> bool:
    if isinstance(x, np.ndarray):
        return bool(x.flags.writeable)
    return True
