"""Tensors of the reference's memory layer, backed by torch storage.

Mirrors ``python/blade/_memory/__init__.py`` (array_tensor, phasor_tensor,
delay_tensor, tensor) and the nanobind ``Vector``/``Duet`` classes of
``python/blade/ext_mem.cc:11-84``: a ``Vector`` has a shape, a dtype, a device and a
data pointer; a ``Duet`` holds two Vectors for the Runner's two in-flight slots and
a *fixed* Vector that is re-pointed at slot ``i`` by ``duet[i]``
(``include/blade/memory/helper.hh:13-49``), so modules that hold the fixed Vector
read the current slot's data pointer at ``process()`` time.

PyTorch only provides the device/pinned-host allocations; every kernel that
touches the data is in ``libblade_b200.so``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .constants import Constant, cpu, cuda, unified, f32, dtypes

# Storage per element type: (torch dtype, trailing pair axis?, C-ABI type code, numpy dtype)
_STORAGE = {
    "i8": (torch.int8, False, _lib.I8, np.int8),
    "i32": (torch.int32, False, _lib.I32, np.int32),
    "f16": (torch.float16, False, _lib.F16, np.float16),
    "f32": (torch.float32, False, _lib.F32, np.float32),
    "f64": (torch.float64, False, _lib.F64, np.float64),
    "ci8": (torch.int8, True, _lib.CI8, np.int8),
    "cf16": (torch.float16, True, _lib.CF16, np.float16),
    "cf32": (torch.complex64, False, _lib.CF32, np.complex64),
    "cf64": (torch.complex128, False, _lib.CF64, np.complex128),
}

_SHAPE_RANK = {"array_tensor": 4, "phasor_tensor": 5, "delay_tensor": 2, "tensor": 1}


def type_code(dtype: str) -> int:
    return _STORAGE[dtype][2]


def element_bytes(dtype: str) -> int:
    t, pair, _, _ = _STORAGE[dtype]
    return torch.empty((), dtype=t).element_size() * (2 if pair else 1)


class Shape(tuple):
    """Named-axis shape (ArrayShape / PhasorShape / DelayShape / VectorShape,
    include/blade/memory/custom.hh:10-163)."""

    kind = "tensor"

    def __new__(cls, dims, kind="tensor"):
        obj = super().__new__(cls, tuple(int(d) for d in dims))
        obj.kind = kind
        return obj

    @property
    def size(self):
        n = 1
        for d in self:
            n *= d
        return n

    # ArrayShape [A, F, T, P]
    @property
    def number_of_aspects(self):
        return self[0]

    @property
    def number_of_frequency_channels(self):
        return self[1] if self.kind == "array_tensor" else self[2]

    @property
    def number_of_time_samples(self):
        return self[2] if self.kind == "array_tensor" else self[3]

    @property
    def number_of_polarizations(self):
        return self[3] if self.kind == "array_tensor" else self[4]

    # PhasorShape [B, A, F, T, P] and DelayShape [B, A]
    @property
    def number_of_beams(self):
        return self[0]

    @property
    def number_of_antennas(self):
        return self[1]


class Vector:
    """A typed, shaped buffer on the host (pinned) or on the current CUDA device."""

    def __init__(self, shape, dtype="f32", device="cuda", kind="tensor", unified_=False, storage=None):
        if isinstance(shape, int):
            shape = (shape,)
        self._shape = Shape(shape, kind)
        self._dtype = dtype
        self._device = device
        self._unified = unified_
        tdtype, pair, _, _ = _STORAGE[dtype]
        full = tuple(self._shape) + ((2,) if pair else ())
        if storage is not None:
            self._t = storage
        elif device == "cuda":
            self._t = torch.zeros(full, dtype=tdtype, device="cuda")
        else:
            pin = torch.cuda.is_available()
            self._t = torch.zeros(full, dtype=tdtype, pin_memory=pin)

    # -- reference surface -------------------------------------------------
    @property
    def shape(self) -> Shape:
        return self._shape

    @property
    def dtype(self) -> str:
        return self._dtype

    @property
    def device(self) -> str:
        return self._device

    @property
    def unified(self) -> bool:
        return self._unified

    def size(self) -> int:
        return self._shape.size

    @property
    def nbytes(self) -> int:
        return self._shape.size * element_bytes(self._dtype)

    def data_ptr(self) -> int:
        return self._t.data_ptr()

    def as_torch(self) -> torch.Tensor:
        """Storage view: complex64/complex128 for cf32/cf64, [..., 2] pairs for ci8/cf16."""
        return self._t

    def as_numpy(self) -> np.ndarray:
        if self._device != "cpu":
            raise RuntimeError("as_numpy() is only available for host (bl.cpu) tensors")
        return self._t.numpy()

    def __repr__(self):
        return f"Vector({list(self._shape)}, dtype={self._dtype}, device={self._device})"

    # -- fixed-slot re-pointing (Duet) -------------------------------------
    def _alias(self, other: "Vector") -> None:
        self._t = other._t


class Duet:
    """Two Vectors for the Runner's two slots plus a fixed alias of the current one."""

    def __init__(self, shape, dtype="f32", device="cuda", kind="tensor", unified_=False):
        self._slots = [Vector(shape, dtype, device, kind, unified_), Vector(shape, dtype, device, kind, unified_)]
        self._fixed = Vector(shape, dtype, device, kind, unified_, storage=self._slots[0]._t)

    def set(self, index: int) -> None:
        self._fixed._alias(self._slots[index])

    def at(self, index: int) -> Vector:
        return self._slots[index]

    def __getitem__(self, index: int) -> Vector:
        self.set(index)
        return self._fixed

    def __call__(self) -> Vector:
        return self._fixed

    @property
    def shape(self):
        return self._fixed.shape

    @property
    def dtype(self):
        return self._fixed.dtype

    def __repr__(self):
        return f"Duet({list(self.shape)}, dtype={self.dtype})"


def _create(kind, shape, dtype, device):
    from .runtime import _fetch_pipeline

    _dtype = dtype.value if isinstance(dtype, Constant) else str(dtype)
    _device = device.value if isinstance(device, Constant) else str(device)
    if _dtype not in _STORAGE:
        raise ValueError(f"unsupported dtype {_dtype}")
    is_unified = _device == "unified"
    if is_unified:
        _device = "cuda"
    if isinstance(shape, int):
        shape = (shape,)
    if len(shape) != _SHAPE_RANK[kind]:
        raise ValueError(f"{kind} expects rank {_SHAPE_RANK[kind]}, got shape {tuple(shape)}")
    if _fetch_pipeline() is not None and _device == "cuda":
        return Duet(shape, _dtype, _device, kind, is_unified)
    return Vector(shape, _dtype, _device, kind, is_unified)


def array_tensor(shape, dtype=f32, device=cuda):
    """[A, F, T, P] tensor (python/blade/_memory/__init__.py:22-33)."""
    return _create("array_tensor", shape, dtype, device)


def phasor_tensor(shape, dtype=f32, device=cuda):
    """[B, A, F, T, P] tensor (python/blade/_memory/__init__.py:35-46)."""
    return _create("phasor_tensor", shape, dtype, device)


def delay_tensor(shape, dtype=f32, device=cuda):
    """[B, A] tensor (python/blade/_memory/__init__.py:48-59)."""
    return _create("delay_tensor", shape, dtype, device)


def tensor(shape, dtype=f32, device=cuda):
    """1-D tensor (python/blade/_memory/__init__.py:61-72)."""
    return _create("tensor", shape, dtype, device)


def as_vector(obj) -> Vector:
    """A Duet stands for its fixed Vector (python/blade/_internal/__init__.py:81-100)."""
    if isinstance(obj, Duet):
        return obj()
    return obj


def copy(dst, src, stream=None) -> None:
    """Asynchronous copy between Vectors (include/blade/memory/copy.hh:11-33):
    shapes and dtypes must match; any host/device direction."""
    dst, src = as_vector(dst), as_vector(src)
    if tuple(dst.shape) != tuple(src.shape) or dst.dtype != src.dtype:
        raise RuntimeError(f"copy: shape/dtype mismatch {dst!r} <- {src!r}")
    if stream is None:
        dst._t.copy_(src._t, non_blocking=True)
    else:
        with torch.cuda.stream(stream):
            dst._t.copy_(src._t, non_blocking=True)


__all__ = ["Vector", "Duet", "Shape", "array_tensor", "phasor_tensor", "delay_tensor", "tensor", "copy",
           "as_vector", "type_code", "element_bytes", "dtypes"]
