"""Helpers for the GPU parity tests: numpy <-> device tensors and C-ABI calls."""

import numpy as np
import torch

from blade_b200 import _lib


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t: torch.Tensor) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def c64(a) -> torch.Tensor:
    return dev(np.asarray(a, dtype=np.complex64))


def ptr(t) -> int:
    return t.data_ptr() if t is not None else None


def stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def call(name, *args):
    return _lib.call(name, *args)


def rel_l2(a, ref) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(ref) else np.float64)
    ref = np.asarray(ref, dtype=a.dtype)
    return float(np.linalg.norm((a - ref).ravel()) / max(np.linalg.norm(ref.ravel()), 1e-300))


def crand(rng, shape, dtype=np.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
