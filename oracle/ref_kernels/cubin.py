"""Test-only launcher of the reference's device-only kernels.

oracle/_ref/ref_*.cubin hold the reference's polarizer, gather (accumulate) and
permutation kernels, built from the reference sources by build.sh (one kernel per
cubin; ref_device_only.cu says why they are device code only).  This module
loads a cubin into the current CUDA context through the driver API and launches
its kernel with the by-value argument bytes of the reference's
Vector<Device::CUDA, T, ArrayShape> (include/blade/memory/vector.hh:215-218:
Shape _shape; T* _data; U64* _refs; bool _unified), whose ArrayShape is Shape<4>
(include/blade/memory/shape.hh:75-77: U64 _shape[4]; U64 _strides[4]; U64 _size;
strides and size as Shape::computeCache fills them, shape.hh:111-123).  _refs is
null, so the kernels' by-value copies never touch a reference count.

Used only by tests/golden/make_golden.py, on a GPU machine; the product path
never imports it.
"""

from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(os.path.dirname(HERE), "_ref")


class RefShape(C.Structure):
    _fields_ = [("shape", C.c_uint64 * 4), ("strides", C.c_uint64 * 4), ("size", C.c_uint64)]


class RefVector(C.Structure):
    _fields_ = [("shape", RefShape), ("data", C.c_void_p), ("refs", C.c_void_p), ("unified", C.c_bool)]


assert C.sizeof(RefShape) == 72 and C.sizeof(RefVector) == 96


def ref_shape(shape) -> RefShape:
    s = RefShape()
    dims = [int(d) for d in shape]
    assert len(dims) == 4
    size = 1
    for i, d in enumerate(dims):
        s.shape[i] = d
        size *= d
        st = 1
        for d2 in dims[i + 1:]:
            st *= d2
        s.strides[i] = st
    s.size = size
    return s


def ref_vector(ptr: int, shape) -> RefVector:
    v = RefVector()
    v.shape = ref_shape(shape)
    v.data = ptr
    v.refs = None
    v.unified = False
    return v


_cuda = None


def _driver():
    global _cuda
    if _cuda is None:
        _cuda = C.CDLL("libcuda.so.1")
    return _cuda


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what}: CUresult {rc}")


class Kernel:
    """The single kernel of oracle/_ref/ref_<name>.cubin in the current context."""

    def __init__(self, name: str):
        cu = _driver()
        path = os.path.join(REF_DIR, f"ref_{name}.cubin")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is missing: run oracle/ref_kernels/build.sh")
        self.module = C.c_void_p()
        _check(cu.cuModuleLoad(C.byref(self.module), path.encode()), "cuModuleLoad")
        n = C.c_uint(0)
        _check(cu.cuModuleGetFunctionCount(C.byref(n), self.module), "cuModuleGetFunctionCount")
        if n.value != 1:
            raise RuntimeError(f"{path}: expected one kernel, found {n.value}")
        fns = (C.c_void_p * 1)()
        _check(cu.cuModuleEnumerateFunctions(fns, C.c_uint(1), self.module), "cuModuleEnumerateFunctions")
        self.fn = C.c_void_p(fns[0])

    def launch(self, grid: int, block: int, *args) -> None:
        """Launches on the legacy default stream and waits for completion."""
        cu = _driver()
        params = (C.c_void_p * len(args))(*[C.cast(C.pointer(a), C.c_void_p) for a in args])
        _check(cu.cuLaunchKernel(self.fn, C.c_uint(grid), C.c_uint(1), C.c_uint(1), C.c_uint(block), C.c_uint(1),
                                 C.c_uint(1), C.c_uint(0), None, params, None), "cuLaunchKernel")
        _check(cu.cuCtxSynchronize(), "cuCtxSynchronize")


def pad_grid(n: int, block: int) -> int:
    """Module::PadGridSize (include/blade/module.hh:85-89)."""
    return (n + block - 1) // block
