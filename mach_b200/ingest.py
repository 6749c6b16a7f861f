"""Channel-data ingest on the GPU: acquisition order to the beamformer's layout.

UFF files and PyMUST hand channel data as ``[n_samples, n_elements, n_waves(, n_frames)]``;
the beamformer wants ``[n_waves, n_elements, n_samples, n_frames]`` in its storage type.
mach rearranges with einops on the host and casts with NumPy (src/mach/io/uff.py:70-105,
examples/doppler.py:193-195).  :func:`ingest` does both in one pass of one kernel
(``mach_b200_ingest``), reading and writing each sample once.
"""

from __future__ import annotations

from typing import Any

from mach_b200 import _cuda_impl

_lib = _cuda_impl._lib

_DTYPES = {  # storage code -> (torch dtype, trailing (I, Q) axis)
    "f32": ("float32", False), "c64": ("complex64", False), "f16": ("float16", False), "cf16": ("float16", True),
    "bf16": ("bfloat16", False), "cbf16": ("bfloat16", True), "i16": ("int16", False), "ci16": ("int16", True),
}


def storage_of_tensor(t, complex_pairs: bool | None = None) -> str:
    """Storage code of a torch tensor in acquisition order.  16-bit data is complex (a trailing
    (I, Q) axis of 2) when ``complex_pairs`` says so, or by default when it has 5 dimensions."""
    name = str(t.dtype).replace("torch.", "")
    if name == "complex64":
        return "c64"
    if name == "float32":
        return "f32"
    codes = {"float16": "f16", "bfloat16": "bf16", "int16": "i16"}
    if name not in codes:
        raise TypeError(f"unsupported channel dtype {t.dtype}")
    pairs = complex_pairs if complex_pairs is not None else t.dim() == 5
    if pairs and t.shape[-1] != 2:
        raise ValueError("16-bit complex data needs a trailing (I, Q) axis of length 2")
    return ("c" + codes[name]) if pairs else codes[name]


def ingest(signal: Any, storage: str | None = None, *, scale: float = 1.0, complex_pairs: bool | None = None,
           out: Any = None, sync: bool = True) -> Any:
    """Rearrange and convert channel data on the GPU.

    Args:
        signal: torch tensor ``[n_samples, n_elements, n_waves]`` or ``[..., n_frames]``
            (float32, complex64, float16, bfloat16, int16), with a trailing ``(I, Q)`` axis of 2
            for 16-bit complex data (say ``complex_pairs=True`` when the shape alone is
            ambiguous).  A CPU tensor is copied to the current GPU.
        storage: destination storage code (``"f32"``, ``"c64"``, ``"f16"``, ``"cf16"``, ``"bf16"``,
            ``"cbf16"``, ``"i16"``, ``"ci16"``); default: the source's.
        scale: every value is multiplied by it before rounding to the destination type
            (int16 destinations saturate).
        out: optional destination tensor ``[n_waves, n_elements, n_samples, n_frames(, 2)]``.

    Returns:
        The channel data in the beamformer's layout, on the GPU.
    """
    import torch

    src = storage_of_tensor(signal, complex_pairs)
    pairs_in = src in ("cf16", "cbf16", "ci16")
    core = signal.shape[:-1] if pairs_in else signal.shape
    if len(core) == 3:
        core = (*core, 1)
    if len(core) != 4:
        raise ValueError("signal must be [n_samples, n_elements, n_waves] or [n_samples, n_elements, n_waves, n_frames]")
    n_s, n_e, n_w, n_f = (int(d) for d in core)
    dst = storage or src
    if dst not in _DTYPES:
        raise ValueError(f"unknown storage {dst!r}")
    if (src in ("c64", "cf16", "cbf16", "ci16")) != (dst in ("c64", "cf16", "cbf16", "ci16")):
        raise ValueError("source and destination must both be real or both be complex")
    dt_name, pairs_out = _DTYPES[dst]
    shape = (n_w, n_e, n_s, n_f) + ((2,) if pairs_out else ())
    if out is None:
        out = torch.empty(shape, dtype=getattr(torch, dt_name), device="cuda")
    elif tuple(out.shape) != shape or not out.is_cuda or not out.is_contiguous():
        raise ValueError(f"out must be a contiguous CUDA tensor of shape {list(shape)}")
    sig = signal.contiguous()
    stream = torch.cuda.current_stream().cuda_stream
    flags = 0 if (sync or not sig.is_cuda) else _cuda_impl.FLAG_ASYNC
    rc = _lib.mach_b200_ingest(_cuda_impl.STORAGE_CODES[src], sig.data_ptr(), _cuda_impl.STORAGE_CODES[dst],
                               out.data_ptr(), n_s, n_e, n_w, n_f, float(scale), stream, flags)
    _cuda_impl._raise_for(rc)
    return out
