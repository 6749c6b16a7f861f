"""Zero-copy views of array objects (NumPy, PyTorch, and any DLPack producer).

mach's binding receives its arrays through nanobind's DLPack support
(src/mach/kernel.cu:1032-1048).  This module extracts the same information --
data pointer, shape, strides, dtype and device -- without copying, so the
C ABI in ``libmach_b200.so`` can be called with plain pointers.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Any

import numpy as np

CPU, CUDA, CUDA_HOST, CUDA_MANAGED = 1, 2, 3, 13


class NullView:
    """Stands for an absent array: a NULL pointer."""

    ptr = 0


@dataclass
class ArrayView:
    ptr: int
    shape: tuple[int, ...]
    strides: tuple[int, ...]  # in elements
    dtype: str  # "float32", "complex64", "float16", "bfloat16", "int16", ...
    itemsize: int
    device_type: int  # DLPack device type
    device_id: int
    writeable: bool
    owner: Any  # keeps the producer (or its capsule) alive

    @property
    def on_cuda(self) -> bool:
        return self.device_type in (CUDA, CUDA_MANAGED)

    @property
    def c_contiguous(self) -> bool:
        expected = 1
        for dim, stride in zip(reversed(self.shape), reversed(self.strides), strict=True):
            if dim != 1 and stride != expected:
                return False
            expected *= dim
        return True

    @property
    def size(self) -> int:
        n = 1
        for d in self.shape:
            n *= d
        return n


# ---- generic DLPack capsule decoding -------------------------------------------------


class _DLDevice(ctypes.Structure):
    _fields_ = [("device_type", ctypes.c_int), ("device_id", ctypes.c_int)]


class _DLDataType(ctypes.Structure):
    _fields_ = [("code", ctypes.c_uint8), ("bits", ctypes.c_uint8), ("lanes", ctypes.c_uint16)]


class _DLTensor(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("device", _DLDevice),
        ("ndim", ctypes.c_int),
        ("dtype", _DLDataType),
        ("shape", ctypes.POINTER(ctypes.c_int64)),
        ("strides", ctypes.POINTER(ctypes.c_int64)),
        ("byte_offset", ctypes.c_uint64),
    ]


_capsule_get_pointer = ctypes.pythonapi.PyCapsule_GetPointer
_capsule_get_pointer.restype = ctypes.c_void_p
_capsule_get_pointer.argtypes = [ctypes.py_object, ctypes.c_char_p]

_DL_CODES = {(0, 16): "int16", (0, 32): "int32", (0, 64): "int64", (0, 8): "int8", (1, 8): "uint8",
             (1, 16): "uint16", (1, 32): "uint32", (1, 64): "uint64", (2, 16): "float16",
             (2, 32): "float32", (2, 64): "float64", (4, 16): "bfloat16", (5, 64): "complex64",
             (5, 128): "complex128", (5, 32): "complex32", (6, 8): "bool"}


def _from_capsule(obj: Any) -> ArrayView:
    capsule = obj.__dlpack__()
    raw = _capsule_get_pointer(capsule, b"dltensor")
    t = _DLTensor.from_address(raw)  # DLManagedTensor starts with its DLTensor
    ndim = t.ndim
    shape = tuple(int(t.shape[i]) for i in range(ndim))
    if t.strides:
        strides = tuple(int(t.strides[i]) for i in range(ndim))
    else:
        strides, acc = [], 1
        for d in reversed(shape):
            strides.append(acc)
            acc *= d
        strides = tuple(reversed(strides))
    dtype = _DL_CODES.get((t.dtype.code, t.dtype.bits), f"dl{t.dtype.code}_{t.dtype.bits}")
    if t.dtype.lanes != 1:
        dtype = f"{dtype}x{t.dtype.lanes}"
    return ArrayView(
        ptr=(t.data or 0) + int(t.byte_offset),
        shape=shape,
        strides=strides,
        dtype=dtype,
        itemsize=max(1, t.dtype.bits // 8),
        device_type=int(t.device.device_type),
        device_id=int(t.device.device_id),
        writeable=True,
        owner=(obj, capsule),
    )


def _torch_view(t: Any) -> ArrayView:
    dtype = str(t.dtype).replace("torch.", "")
    if dtype == "complex32":
        dtype = "complex32"
    dev = t.device
    return ArrayView(
        ptr=int(t.data_ptr()),
        shape=tuple(int(d) for d in t.shape),
        strides=tuple(int(s) for s in t.stride()),
        dtype=dtype,
        itemsize=int(t.element_size()),
        device_type=CUDA if dev.type == "cuda" else CPU,
        device_id=int(dev.index or 0) if dev.type == "cuda" else 0,
        writeable=True,
        owner=t,
    )


def _numpy_view(a: np.ndarray) -> ArrayView:
    item = a.itemsize
    return ArrayView(
        ptr=int(a.__array_interface__["data"][0]) if a.size else 0,
        shape=tuple(int(d) for d in a.shape),
        strides=tuple(int(s) // item for s in a.strides),
        dtype=str(a.dtype),
        itemsize=item,
        device_type=CPU,
        device_id=0,
        writeable=bool(a.flags.writeable),
        owner=a,
    )


def is_torch(x: Any) -> bool:
    return type(x).__module__.startswith("torch")


def view(x: Any) -> ArrayView:
    """Describe ``x`` without copying it."""
    if isinstance(x, np.ndarray):
        return _numpy_view(x)
    if is_torch(x):
        return _torch_view(x)
    if hasattr(x, "__dlpack__"):
        return _from_capsule(x)
    raise TypeError(f"{type(x).__name__} does not support the DLPack protocol")


def dlpack_device(x: Any) -> tuple[int, int]:
    if isinstance(x, np.ndarray):
        return CPU, 0
    if is_torch(x):
        return (CUDA, int(x.device.index or 0)) if x.device.type == "cuda" else (CPU, 0)
    if hasattr(x, "__dlpack_device__"):
        d = x.__dlpack_device__()
        return int(d[0]), int(d[1])
    raise TypeError(f"{type(x).__name__} does not support the DLPack protocol")
