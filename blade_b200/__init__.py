"""blade_b200: a B200-native (sm_100a) implementation of BLADE's beamform ->
channelize -> detect path behind BLADE's Module / Pipeline / Runner interface.

Usage mirrors the reference's Python package (python/blade/__init__.py)::

    import blade_b200 as bl

    @bl.runner
    class Pipeline:
        def __init__(self, shape, phasor_shape):
            self.input.buf = bl.array_tensor(shape, dtype=bl.cf32)
            self.input.phasors = bl.phasor_tensor(phasor_shape, dtype=bl.cf32)
            self.module.beamformer = bl.module(bl.beamformer, {}, (self.input.buf, self.input.phasors),
                                               telescope=bl.ata)
        ...

The compute path is ``libblade_b200.so`` (hand-written sm_100a CUDA behind a C
ABI, include/blade_b200.h); PyTorch only supplies device memory and streams.
"""

from . import _lib, autotune
from .constants import *  # noqa: F401,F403  (bl.cf32, bl.ata, bl.beamformer, bl.pol, bl.result, ...)
from .constants import Constant, Taint, pol, result
from .memory import Duet, Vector, array_tensor, delay_tensor, phasor_tensor, tensor
from .memory import copy as _mem_copy
from .modules import (BeamformDetect, BeamformerATA, BeamformerMeerKAT, Cast, Channelizer, Detector, Duplicate,
                      Gather, ModeB, ModeH, Module, Permutation, Phasor, Polarizer)
from .runtime import Pipeline, Runner, module, runner
from .guppi import GuppiReader, GuppiWriter
from .bfr5 import Bfr5Reader

__version__ = "1.0.0"


def copy(dst, src):
    """Synchronous-looking copy outside a runner (python/blade/_copy)."""
    import torch

    _mem_copy(dst, src)
    if torch.cuda.is_available():
        torch.cuda.current_stream().synchronize()
    return result.success


def stream():
    """The default stream handle (modules created outside a pipeline use it)."""
    import torch

    return torch.cuda.current_stream()


def device_status() -> int:
    """Reads and clears the device status word of the pipelined kernels (non-zero:
    a bounded in-kernel wait expired)."""
    import ctypes

    v = ctypes.c_uint32(0)
    _lib.call("blade_device_status", ctypes.byref(v))
    return int(v.value)
