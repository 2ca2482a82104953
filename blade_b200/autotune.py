"""Launch-shape autotuning (the C ABI's blade_*_autotune / blade_autotune_query).

The reference fixes one launch knob per module (``blockSize``,
include/blade/modules/beamformer/generic.hh:20).  Here a tuning call times every
launch candidate of a kernel family on the caller's shape with CUDA events,
keeps only candidates whose output is bit-identical to the default's, and stores
the fastest in a per-device cache that every later launch of that shape reads::

    import blade_b200 as bl
    bl.autotune.tensor_core(B=64, A=64, F=256, T=8192, rate=1, integration=8)
    bl.autotune.query(bl.autotune.TC, (64, 64, 256, 8192, 2, 1, 8, 4))
    # {'params': [1, 4, 0, 1, 15, 0, 0, 0], 'us': 254.1, 'tuned': True}

Tuning synchronises the stream and allocates its own inputs: call it at start-up,
outside stream capture.
"""

from __future__ import annotations

import ctypes as C

from . import _lib

TC, F32, SPECTROMETER = 1, 2, 3


def _stream(stream):
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def tensor_core(B, A, F, T, rate=1, integration=1, P=2, stream=None) -> dict:
    """Tunes the tensor-core chain (blade_beamform_detect_tc family) for one shape."""
    _lib.call("blade_beamform_detect_tc_autotune", B, A, F, T, P, rate, integration, _stream(stream))
    return query(TC, (B, A, F, T, P, rate, integration, 4))


def fp32(B, A, F, T, rate=1, integration=1, in_type=_lib.CI8, P=2, stream=None) -> dict:
    """Tunes the fused FP32 chain (blade_beamform_detect_f32) for one shape."""
    _lib.call("blade_beamform_detect_f32_autotune", in_type, B, A, F, T, P, rate, integration, _stream(stream))
    return query(F32, (B, A, F, T, P, rate, integration, in_type))


def spectrometer(A, F, T, rate=65536, integration=1, out_pols=1, in_type=_lib.CI8, out_type=_lib.F32, P=2,
                 stream=None) -> dict:
    """Tunes the fused spectrometer (blade_spectrometer) for one shape."""
    _lib.call("blade_spectrometer_autotune", in_type, out_type, A, F, T, P, rate, integration, out_pols,
              _stream(stream))
    return query(SPECTROMETER, (A, F, T, P, rate, integration, out_pols, in_type))


def query(family: int, shape) -> dict:
    """The launch choice a launch of `shape` uses now on the current device."""
    key = _lib.u64_array(list(shape))
    params = (C.c_uint32 * 8)()
    us = C.c_float(0.0)
    tuned = C.c_int(0)
    _lib.call("blade_autotune_query", family, key, params, C.byref(us), C.byref(tuned))
    return {"params": list(params), "us": float(us.value), "tuned": bool(tuned.value)}


def clear() -> None:
    """Forgets every tuned choice."""
    _lib.call("blade_autotune_clear")
