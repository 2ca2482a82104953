"""Modules of the beamform -> channelize -> detect path.

Each class mirrors the reference module of the same name: the ``Config`` fields
and keyword names of the nanobind bindings (``python/blade/ext_*.cc``), the
``Input`` fields, the output shape, the taint and compute ratio, and the
constructor checks (a failed check raises ``RuntimeError``, which is what the
reference's ``BL_CHECK_THROW`` becomes in Python, ``python/blade/ext_hidden.cc:17-24``).
``process(step, stream)`` enqueues the module's kernel through the C ABI
(``libblade_b200.so``) on ``stream`` and returns a ``result`` code.

Output buffers are allocated per Runner slot when the module lives in a
pipeline (``Duet``), so the two in-flight slots never share an intermediate
buffer (the reference shares them, ``src/runner.cc:17-68``).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .constants import Taint, pol, result
from .memory import Duet, Vector, as_vector, element_bytes, type_code

_COMPLEX = {"ci8", "cf16", "cf32", "cf64"}


def _stream_handle(stream) -> Optional[int]:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream if torch.cuda.is_available() else None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _fail(msg: str):
    raise RuntimeError(msg)


class Module:
    """Base class (include/blade/module.hh:20-115)."""

    taint = Taint.NONE

    def __init__(self):
        self._owned: list = []  # Duets owned by this module (per-slot outputs)

    def get_taint(self) -> Taint:
        return self.taint

    def get_compute_ratio(self) -> int:
        return 1

    def name(self) -> str:
        return type(self).__name__

    def process(self, step: int = 0, stream=None) -> result:  # pragma: no cover - overridden
        return result.success

    # -- helpers ---------------------------------------------------------------
    def _alloc(self, shape, dtype, kind="array_tensor"):
        """Output buffer: one per Runner slot inside a pipeline, else a single Vector."""
        from .runtime import _fetch_pipeline

        if _fetch_pipeline() is not None:
            d = Duet(shape, dtype, "cuda", kind)
            self._owned.append(d)
            return d
        return Vector(shape, dtype, "cuda", kind)

    def _set_slot(self, index: int) -> None:
        for d in self._owned:
            d.set(index)

    def __repr__(self):
        return f"{self.name()}()"


def _out(buf):
    return as_vector(buf)


# =============================================================================
# Cast
# =============================================================================

class Cast(Module):
    """Modules::Cast<IT, OT> (include/blade/modules/cast.hh, src/modules/cast/base.cc:12-66)."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input, self._it, self._ot = config, input, it, ot
        buf = as_vector(input.buffer)
        if (it in _COMPLEX) != (ot in _COMPLEX):
            _fail("Cannot cast between complex and non-complex types.")
        if buf.dtype != it:
            _fail(f"Cast input buffer is {buf.dtype}, expected {it}.")
        if it == ot:
            self._output = input.buffer  # bypass (Link), base.cc:45-49
        else:
            self._output = self._alloc(buf.shape, ot)

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        if self._it == self._ot:
            return result.success
        i, o = as_vector(self._input.buffer), _out(self._output)
        _lib.call("blade_cast", type_code(self._it), type_code(self._ot), i.data_ptr(), o.data_ptr(), i.size(),
                  _stream_handle(stream))
        return result.success


# =============================================================================
# Beamformer (ATA)
# =============================================================================

class BeamformerATA(Module):
    """Modules::Beamformer::ATA<CF32, CF32> (include/blade/modules/beamformer/{generic,ata}.hh,
    src/modules/beamformer/ata.cc:7-74, generic.cc:9-33).

    ``block_size`` is accepted for interface parity; the kernel has no block-size
    constraint, so the reference's T % blockSize and B <= blockSize checks
    (generic.cc:17-21, ata.cc:13-17), which only guard its launch geometry, are
    not applied."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        enable_incoherent_beam: bool = False
        enable_incoherent_beam_sqrt: bool = False
        block_size: int = 512

    @dataclass
    class input:
        buffer: object
        phasors: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        buf, ph = as_vector(input.buffer), as_vector(input.phasors)
        if it != "cf32" or ot != "cf32" or buf.dtype != "cf32" or ph.dtype != "cf32":
            _fail("Beamformer::ATA supports CF32 -> CF32 only.")
        A, F, T, P = buf.shape
        B, Ap, Fp, Tp, Pp = ph.shape
        if Fp != F:
            _fail(f"Number of frequency channels mismatch between phasors ({Fp}) and buffer ({F}).")
        if Pp != P:
            _fail(f"Number of polarizations mismatch between phasors ({Pp}) and buffer ({P}).")
        if Ap != A:
            _fail(f"Number of antennas mismatch between phasors ({Ap}) and buffer ({A}).")
        if Tp != 1:
            _fail("Phasor time axis must be 1.")
        self._shape = (B + (1 if config.enable_incoherent_beam else 0), F, T, P)
        self._output = self._alloc(self._shape, "cf32")

    def get_config(self):
        return self.config

    def get_input_buffer(self):
        return self._input.buffer

    def get_input_phasors(self):
        return self._input.phasors

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, ph, out = as_vector(self._input.buffer), as_vector(self._input.phasors), _out(self._output)
        A, F, T, P = buf.shape
        B = ph.shape[0]
        _lib.call("blade_beamform_f32", buf.data_ptr(), ph.data_ptr(), out.data_ptr(), B, A, F, T, P,
                  int(self.config.enable_incoherent_beam), int(self.config.enable_incoherent_beam_sqrt),
                  _stream_handle(stream))
        return result.success


class BeamformerMeerKAT(BeamformerATA):
    """Modules::Beamformer::MeerKAT<CF32, CF32> (include/blade/modules/beamformer/meerkat.hh,
    src/modules/beamformer/meerkat.cc:8-39, kernel beamformer.cu:81-117): one weight
    per (beam, antenna) for every channel and polarisation, read as the first B*A
    values of the [B, A, F, 1, P] phasor tensor (as the reference kernel indexes it).
    The incoherent beam is sized as in the reference, which never writes it; here it
    is zero."""

    def process(self, step=0, stream=None):
        buf, ph, out = as_vector(self._input.buffer), as_vector(self._input.phasors), _out(self._output)
        A, F, T, P = buf.shape
        B = ph.shape[0]
        _lib.call("blade_beamform_meerkat_f32", buf.data_ptr(), ph.data_ptr(), out.data_ptr(), B, A, F, T, P,
                  int(self.config.enable_incoherent_beam), _stream_handle(stream))
        return result.success


# =============================================================================
# Channelizer
# =============================================================================

class Channelizer(Module):
    """Modules::Channelizer<CF32, CF32> (include/blade/modules/channelizer/base.hh:12-87,
    src/modules/channelizer/base.cc:9-146).

    rate == 1 and rate == T run in place (the reference's Link), any other even
    rate dividing T (rejected by the reference, base.cc:30-35) writes its own
    [A, F*rate, T/rate, P] buffer."""

    taint = Taint.CONSUMER | Taint.MODIFIER

    @dataclass
    class config:
        rate: int = 4
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        buf = as_vector(input.buffer)
        if buf.dtype != "cf32":
            _fail("Channelizer supports CF32 only.")
        A, F, T, P = buf.shape
        C = int(config.rate)
        if C <= 0 or T % C != 0:
            _fail(f"The number of time samples ({T}) should be divisable by the channelizer rate ({C}).")
        if C % 2 != 0 and C != 1:
            _fail(f"The channelizer rate ({C}) should be divisable by 2.")
        if P not in (1, 2):
            _fail(f"Number of polarizations ({P}) of the input should be one or two.")
        self._shape = (A, F * C, T // C, P)
        self._inplace = C in (1, T)
        if self._inplace:
            self._output = _reshaped(input.buffer, self._shape)
        else:
            self._output = self._alloc(self._shape, "cf32")
        wsb = _lib.load().blade_channelize_workspace_size(A, F, T, P, C)
        self._ws = torch.empty(int(wsb), dtype=torch.uint8, device="cuda") if wsb else None

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        if self.config.rate == 1:
            return result.success
        buf, out = as_vector(self._input.buffer), _out(self._output)
        A, F, T, P = buf.shape
        _lib.call("blade_channelize", buf.data_ptr(), out.data_ptr(),
                  self._ws.data_ptr() if self._ws is not None else None, A, F, T, P, int(self.config.rate),
                  _stream_handle(stream))
        return result.success


def _reshaped(buf, shape):
    v = as_vector(buf)
    if tuple(v.shape) == tuple(shape):
        return buf
    return _ReshapedVector(buf, shape)


class _ReshapedVector(Vector):
    def __init__(self, src, shape):
        self._src = src
        v = as_vector(src)
        self._shape_fixed = shape
        super().__init__(shape, v.dtype, v.device, "array_tensor", storage=v.as_torch())

    def data_ptr(self):
        return as_vector(self._src).data_ptr()

    def as_torch(self):
        return as_vector(self._src).as_torch().reshape(self._shape_fixed if self.dtype not in ("ci8", "cf16")
                                                       else tuple(self._shape_fixed) + (2,))


# =============================================================================
# Polarizer
# =============================================================================

class Polarizer(Module):
    """Modules::Polarizer<T, T> (include/blade/modules/polarizer.hh:9-71,
    src/modules/polarizer/base.cc:12-68); in place, bypassed when the input and
    output bases are equal."""

    taint = Taint.MODIFIER

    @dataclass
    class config:
        inputPolarization: int = pol.xy
        outputPolarization: int = pol.lr
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        if it != ot:
            _fail(f"This module requires the type of the input ({it}) and output ({ot}) to be the same.")
        buf = as_vector(input.buffer)
        if buf.dtype not in ("cf32", "cf16"):
            _fail("Polarizer supports CF32 and CF16.")
        if buf.shape[3] != 2:
            _fail("Polarizer needs two polarizations.")
        self._output = input.buffer

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        if int(self.config.inputPolarization) == int(self.config.outputPolarization):
            return result.success
        buf = as_vector(self._input.buffer)
        A, F, T, P = buf.shape
        _lib.call("blade_polarize", type_code(buf.dtype), buf.data_ptr(), buf.data_ptr(), A * F * T,
                  _stream_handle(stream))
        return result.success


# =============================================================================
# Detector
# =============================================================================

class Detector(Module):
    """Modules::Detector<CF32, F32> (include/blade/modules/detector.hh:12-81,
    src/modules/detector/base.cc:9-85)."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        integration_size: int = 1
        number_of_output_polarizations: int = 4
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="f32"):
        super().__init__()
        self.config, self._input = config, input
        buf = as_vector(input.buffer)
        if buf.dtype != "cf32" or ot != "f32":
            _fail("Detector supports CF32 -> F32 only.")
        A, F, T, P = buf.shape
        I = int(config.integration_size)
        if I <= 0:
            _fail(f"Integration size ({I}) should be more than zero.")
        if T % I != 0:
            _fail(f"The number of time samples ({T}) should be divisable by the integration size ({I}).")
        if P != 2:
            _fail(f"Number of polarizations ({P}) should be two (2).")
        if A <= 0:
            _fail(f"Number of aspects ({A}) should be more than zero.")
        if config.number_of_output_polarizations not in (1, 4):
            _fail(f"Number of output polarizations ({config.number_of_output_polarizations}) not supported.")
        self._shape = (A, F, T // I, int(config.number_of_output_polarizations))
        self._output = self._alloc(self._shape, "f32")

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, out = as_vector(self._input.buffer), _out(self._output)
        A, F, T, P = buf.shape
        _lib.call("blade_detect", buf.data_ptr(), out.data_ptr(), A, F, T, P, int(self.config.integration_size),
                  int(self.config.number_of_output_polarizations), _stream_handle(stream))
        return result.success


# =============================================================================
# Gather
# =============================================================================

class Gather(Module):
    """Modules::Gather<T, T> (include/blade/modules/gather.hh:12-95,
    src/modules/gather/base.cc:12-111); CHRONOUS with compute ratio = multiplier."""

    taint = Taint.CONSUMER | Taint.PRODUCER | Taint.CHRONOUS

    @dataclass
    class config:
        axis: int = 0
        multiplier: int = 1
        copy_size_threshold: int = 512
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        if it != ot:
            _fail(f"Input ({it}) and output ({ot}) types aren't the same. Casting isn't supported by Gather yet.")
        buf = as_vector(input.buffer)
        if config.axis >= 4:
            _fail(f"Selected input axis ({config.axis}) is larger than input shape dimensions (4).")
        if config.multiplier <= 0:
            _fail(f"Multiplier ({config.multiplier}) should be more than zero.")
        shape = list(buf.shape)
        shape[config.axis] *= config.multiplier
        self._shape = tuple(shape)
        self._output = self._alloc(self._shape, buf.dtype)

    def get_compute_ratio(self):
        return int(self.config.multiplier)

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, out = as_vector(self._input.buffer), _out(self._output)
        shape = _lib.u64_array(buf.shape)
        _lib.call("blade_gather", element_bytes(buf.dtype), buf.data_ptr(), out.data_ptr(), shape,
                  int(self.config.axis), int(self.config.multiplier), int(step), _stream_handle(stream))
        return result.success


# =============================================================================
# Permutation
# =============================================================================

class Permutation(Module):
    """Modules::Permutation<T, T> (include/blade/modules/permutation.hh:11-78,
    src/modules/permutation/base.cc:12-73)."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        indexes: Sequence[int] = (0, 1, 2, 3)
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        if it != ot:
            _fail(f"Input ({it}) and output ({ot}) types aren't the same. "
                  "Casting isn't supported by Permutation yet.")
        buf = as_vector(input.buffer)
        idx = [int(i) for i in config.indexes]
        if len(idx) != 4:
            _fail(f"Selected input rank ({len(idx)}) doesn't match input shape rank (4).")
        if len(set(idx)) != 4:
            dup = [i for i in idx if idx.count(i) > 1][0]
            _fail(f"Repeated index {dup} in permutation.")
        if any(i < 0 or i > 3 for i in idx):
            _fail("Permutation index out of range.")
        self._idx = idx
        self._shape = tuple(buf.shape[i] for i in idx)
        self._output = self._alloc(self._shape, buf.dtype)

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, out = as_vector(self._input.buffer), _out(self._output)
        _lib.call("blade_permute", element_bytes(buf.dtype), buf.data_ptr(), out.data_ptr(),
                  _lib.u64_array(buf.shape), _lib.u64_array(self._idx), _stream_handle(stream))
        return result.success


# =============================================================================
# Duplicate
# =============================================================================

class Duplicate(Module):
    """Modules::Duplicate<T, T> (include/blade/modules/duplicate.hh:11-64,
    src/modules/duplicate/base.cc:12-37)."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        pass

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        if it != ot:
            _fail(f"Input ({it}) and output ({ot}) types aren't the same. "
                  "Casting isn't supported by Duplicate yet.")
        buf = as_vector(input.buffer)
        self._output = self._alloc(buf.shape, buf.dtype)

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, out = as_vector(self._input.buffer), _out(self._output)
        _lib.call("blade_duplicate", buf.data_ptr(), out.data_ptr(), buf.nbytes, _stream_handle(stream))
        return result.success


# =============================================================================
# Phasor (delay -> phasor)
# =============================================================================

class Phasor(Module):
    """Modules::Phasor::ATA<CF32> (src/modules/phasor/ata.cc), two input forms.

    Geometric (the reference's interface): config carries the antenna positions
    (ECEF metres), the reference antenna, the array reference position, the
    boresight and beam coordinates (ICRS RA/Dec radians); the inputs are the
    block's julian date and DUT1 (host F64 tensors [1]).  Each step computes the
    geometric delays (ata.cc:9-173, blade_geometric_delays: published astrometry
    in FP64, the A x B projections on the device), then the phasors.
    Delays: the input is a device F64 delay_tensor [B, A] of seconds.
    Both then compute the phasors on the GPU in FP64 (ata.cc:176-208)."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        number_of_beams: int = 1
        number_of_antennas: int = 1
        number_of_frequency_channels: int = 1
        number_of_polarizations: int = 2
        observation_frequency_hz: float = 0.0
        channel_bandwidth_hz: float = 0.0
        total_bandwidth_hz: float = 0.0
        frequency_start_index: int = 0
        antenna_calibrations: object = None  # CF64 [A, F, 1, P] (numpy or Vector), None = unit
        block_size: int = 512
        reference_antenna_index: int = 0
        array_reference_position: object = None  # bl.lla(lon, lat, alt)
        boresight_coordinate: object = None  # bl.ra_dec(ra, dec)
        antenna_positions: object = None  # [bl.xyz(x, y, z)] * A, ECEF metres
        beam_coordinates: object = None  # [bl.ra_dec(ra, dec)] * B

    @dataclass
    class input:
        # geometric form: (block_julian_date, block_dut1), host F64 tensors [1];
        # delays form: (delays,), a device F64 delay_tensor [B, A]
        block_julian_date: object = None
        block_dut1: object = None
        delays: object = None

    def __init__(self, config, input, stream=None, it="f64", ot="cf32"):
        super().__init__()
        self.config, self._input = config, input
        c = config
        self._geometric = c.antenna_positions is not None
        if self._geometric:
            pos = np.asarray([tuple(p) for p in c.antenna_positions], dtype=np.float64)
            beams = np.asarray([tuple(b) for b in c.beam_coordinates or []], dtype=np.float64)
            if pos.ndim != 2 or pos.shape[1] != 3:
                _fail("antenna_positions must be a list of bl.xyz.")
            if beams.ndim != 2 or beams.shape[1] != 2 or len(beams) == 0:
                _fail("beam_coordinates must be a non-empty list of bl.ra_dec.")
            if c.boresight_coordinate is None:
                _fail("boresight_coordinate is required with antenna_positions.")
            if c.number_of_antennas != len(pos):
                _fail(f"number_of_antennas ({c.number_of_antennas}) != {len(pos)} antenna positions.")
            if input.block_julian_date is None or input.block_dut1 is None:
                _fail("The geometric Phasor takes (block_julian_date, block_dut1) inputs.")
            c.number_of_beams = len(beams)
            self._pos = np.ascontiguousarray(pos)
            self._beams = np.ascontiguousarray(beams)
            lla = c.array_reference_position
            self._lla = np.asarray(tuple(lla), dtype=np.float64) if lla is not None else None
            self._delays = torch.empty((c.number_of_beams, c.number_of_antennas), dtype=torch.float64, device="cuda")
        else:
            d = as_vector(self._delays_in())
            if d.dtype != "f64" or tuple(d.shape) != (c.number_of_beams, c.number_of_antennas):
                _fail("Phasor delays must be an F64 delay_tensor [B, A].")
        self._cal = None
        if c.antenna_calibrations is not None:
            cal = c.antenna_calibrations
            arr = cal.as_numpy() if isinstance(cal, Vector) else np.asarray(cal)
            exp = (c.number_of_antennas, c.number_of_frequency_channels, 1, c.number_of_polarizations)
            if tuple(arr.shape) != exp:
                _fail(f"Calibrations shape {arr.shape} != {exp}.")
            self._cal = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.complex128)).cuda()
        self._shape = (c.number_of_beams, c.number_of_antennas, c.number_of_frequency_channels, 1,
                       c.number_of_polarizations)
        self._output = self._alloc(self._shape, "cf32", "phasor_tensor")

    def _delays_in(self):
        # delays form: the single input (a tuple input fills the first field)
        i = self._input
        return i.delays if i.delays is not None else i.block_julian_date

    def get_config(self):
        return self.config

    def get_phasors(self):
        return self._output

    get_output = get_phasors

    def get_delays(self):
        """Device F64 [B, A] delays of the last step (geometric form) or the input delays."""
        return self._delays if self._geometric else as_vector(self._delays_in()).as_torch()

    def process(self, step=0, stream=None):
        c = self.config
        s = _stream_handle(stream)
        if self._geometric:
            # the block's date and DUT1 are host values, read as the reference reads them
            jd = float(as_vector(self._input.block_julian_date).as_torch().reshape(-1)[0])
            dut1 = float(as_vector(self._input.block_dut1).as_torch().reshape(-1)[0])
            bo = tuple(c.boresight_coordinate)
            _lib.call("blade_geometric_delays", self._pos.ctypes.data, c.number_of_antennas,
                      c.reference_antenna_index, self._lla.ctypes.data if self._lla is not None else None,
                      float(bo[0]), float(bo[1]), self._beams.ctypes.data, c.number_of_beams, jd, dut1,
                      self._delays.data_ptr(), s)
            dptr = self._delays.data_ptr()
        else:
            dptr = as_vector(self._delays_in()).data_ptr()
        out = _out(self._output)
        _lib.call("blade_phasor_from_delays", dptr, self._cal.data_ptr() if self._cal is not None else None,
                  out.data_ptr(), c.number_of_beams, c.number_of_antennas, c.number_of_frequency_channels,
                  c.number_of_polarizations, float(c.observation_frequency_hz), float(c.channel_bandwidth_hz),
                  float(c.total_bandwidth_hz), int(c.frequency_start_index), s)
        return result.success


# =============================================================================
# Fused chain: Cast -> Beamformer -> Channelizer -> Detector (Stokes-I)
# =============================================================================

class BeamformDetect(Module):
    """The beamform + channelize + detect chain of Bundles::ATA::ModeB
    (include/blade/bundles/ata/mode_b.hh:99-199: Beamformer -> [Channelizer] ->
    Detector) as one fused launch.

    precision = "fp16_split": tcgen05 tensor cores, CI8 input, FP16 hi+lo phasors,
    FP32 accumulation in TMEM.  precision = "fp32": FP32 CUDA cores (CI8 or CF32
    input).  "auto" takes the tensor-core path whenever the shape allows it."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        rate: int = 1
        integration_size: int = 1
        number_of_output_polarizations: int = 1
        precision: str = "auto"
        block_size: int = 512
        autotune: bool = False  # time the launch candidates of this shape at construction

    @dataclass
    class input:
        buffer: object
        phasors: object

    def __init__(self, config, input, stream=None, it="ci8", ot="f32"):
        super().__init__()
        self.config, self._input = config, input
        buf, ph = as_vector(input.buffer), as_vector(input.phasors)
        if buf.dtype not in ("ci8", "cf32") or ph.dtype != "cf32" or ot != "f32":
            _fail("BeamformDetect takes CI8 or CF32 voltages, CF32 phasors and produces F32.")
        if config.number_of_output_polarizations != 1:
            _fail("BeamformDetect produces Stokes-I (number_of_output_polarizations = 1).")
        A, F, T, P = buf.shape
        B = ph.shape[0]
        if tuple(ph.shape) != (B, A, F, 1, P):
            _fail(f"Phasor shape {tuple(ph.shape)} does not match voltages {tuple(buf.shape)}.")
        R, I = int(config.rate), int(config.integration_size)
        if R <= 0 or I <= 0 or T % (R * I) != 0:
            _fail(f"T ({T}) must be a multiple of rate ({R}) x integration ({I}).")
        lib = _lib.load()
        tc_ok = buf.dtype == "ci8" and lib.blade_beamform_detect_tc_supported(B, A, F, T, P, R, I) == 1
        prec = config.precision
        if prec == "auto":
            prec = "fp16_split" if tc_ok else "fp32"
        if prec == "fp16_split" and not tc_ok:
            _fail("The tensor-core path needs CI8 input, P = 2, A <= 64, T % 128 == 0, rate in {1, 2, 4} and an "
                  "integration that is a power of two <= 32.")
        if prec not in ("fp16_split", "fp32"):
            _fail(f"Unknown precision {prec!r}.")
        self.precision = prec
        self._shape = (B, F * R, T // (R * I), 1)
        self._output = self._alloc(self._shape, "f32")
        self._plan = None
        if prec == "fp16_split":
            # the phasor image is rebuilt every step: one per Runner slot
            n = int(lib.blade_beamform_tc_plan_size(B, A, F, P))
            self._plan = self._alloc((n,), "i8", "tensor")
        if config.autotune:
            from . import autotune

            if prec == "fp16_split":
                autotune.tensor_core(B, A, F, T, R, I, P=P, stream=stream)
            else:
                autotune.fp32(B, A, F, T, R, I, in_type=type_code(buf.dtype), P=P, stream=stream)

    def get_config(self):
        return self.config

    def get_input_buffer(self):
        return self._input.buffer

    def get_input_phasors(self):
        return self._input.phasors

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, ph, out = as_vector(self._input.buffer), as_vector(self._input.phasors), _out(self._output)
        A, F, T, P = buf.shape
        B = ph.shape[0]
        R, I = int(self.config.rate), int(self.config.integration_size)
        s = _stream_handle(stream)
        if self.precision == "fp16_split":
            plan = _out(self._plan)
            _lib.call("blade_beamform_prepare_detect_tc", ph.data_ptr(), plan.data_ptr(), buf.data_ptr(),
                      out.data_ptr(), B, A, F, T, P, R, I, s)
        else:
            _lib.call("blade_beamform_detect_f32", type_code(buf.dtype), buf.data_ptr(), ph.data_ptr(),
                      out.data_ptr(), B, A, F, T, P, R, I, s)
        return result.success


class ModeH(Module):
    """Bundles::Generic::ModeH<IT, OT> (include/blade/bundles/generic/mode_h.hh:55-106,
    Python binding python/blade/ext_modeh.cc:21-45):
    Cast -> Channelizer -> Polarizer -> Detector -> output Cast, fused into two
    kernels (blade_spectrometer) so that only the input, an FP32 workspace and the
    detector products touch device memory.  rate defaults to the number of time
    samples as in ModeH; the fused path runs rate 65536 (256 x 256) with up to 16
    spectra per block (the module chain covers every other rate)."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        input_shape: Sequence[int]
        output_shape: Sequence[int]
        polarizer_convert_to_circular: bool
        detector_integration_size: int
        detector_number_of_output_polarizations: int
        cast_block_size: int = 512
        polarizer_block_size: int = 512
        channelizer_block_size: int = 512
        detector_block_size: int = 512
        rate: int = 0  # not in the reference: 0 = the number of time samples, as ModeH

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="ci8", ot="f32"):
        super().__init__()
        self.config, self._input = config, input
        buf = as_vector(input.buffer)
        if buf.dtype not in ("ci8", "cf32") or ot not in ("f32", "f16"):
            _fail("ModeH takes CI8 or CF32 voltages and produces F32 or F16.")
        A, F, T, P = buf.shape
        if tuple(config.input_shape) != tuple(buf.shape):
            _fail(f"Expected input buffer size ({tuple(config.input_shape)}) mismatch with actual size "
                  f"({tuple(buf.shape)}).")
        R = int(config.rate) or T
        I, OP = int(config.detector_integration_size), int(config.detector_number_of_output_polarizations)
        if P != 2:
            _fail(f"The polarizer needs two polarizations (P = {P}).")
        if R <= 0 or T % R != 0:
            _fail(f"The number of time samples ({T}) should be divisible by the channelizer rate ({R}).")
        if I <= 0 or (T // R) % I != 0:
            _fail(f"The number of spectra ({T // R}) should be divisible by the integration size ({I}).")
        if OP not in (1, 4):
            _fail(f"Number of output polarizations ({OP}) not supported.")
        lib = _lib.load()
        n = int(lib.blade_spectrometer_workspace_size(A, F, T, P, R))
        if n == 0:
            _fail(f"The fused spectrometer runs rate 65536; use the module chain for rate {R}.")
        self._rate, self._ot = R, ot
        self._workspace = torch.empty(n, dtype=torch.uint8, device="cuda")
        self._shape = (A, F * R, T // (R * I), OP)
        if tuple(config.output_shape) != self._shape:
            _fail(f"Expected output buffer size ({tuple(config.output_shape)}) mismatch with actual size "
                  f"({self._shape}).")
        self._output = self._alloc(self._shape, ot)

    def get_config(self):
        return self.config

    def get_input_buffer(self):
        return self._input.buffer

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        buf, out = as_vector(self._input.buffer), _out(self._output)
        A, F, T, P = buf.shape
        c = self.config
        _lib.call("blade_spectrometer", type_code(buf.dtype), buf.data_ptr(), type_code(self._ot), out.data_ptr(),
                  self._workspace.data_ptr(), A, F, T, P, self._rate, int(c.detector_integration_size),
                  int(c.detector_number_of_output_polarizations), 1 if c.polarizer_convert_to_circular else 0,
                  _stream_handle(stream))
        return result.success


class _ModeBTensorCore(Module):
    """ModeB on CI8 voltages with the detector (Stokes-I) at channelizer rate 2 or 4:
    the pre-beamformer Cast -> Channelizer -> [Polarizer] into an exact CF16 buffer
    (blade_prechannelize_cf16), then the per-fine-channel phasor split and the
    tensor-core Beamformer -> Detector at rate 1 (blade_beamform_prepare_detect_tc_cf16:
    the split, then the chain overlapping its end), and with the incoherent beam its detected row
    (blade_incoherent_detect_cf16).  Three or four launches."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    def __init__(self, buffer, phasors, rate, integration, circular, incoherent=False):
        super().__init__()
        self._buffer, self._phasors = buffer, phasors
        self._R, self._I, self._circ, self._inc = int(rate), int(integration), bool(circular), bool(incoherent)
        A, F, T, P = as_vector(buffer).shape
        B = as_vector(phasors).shape[0]
        R = self._R
        self._pre = self._alloc((A, F * R, T // R, P), "cf16")
        n = int(_lib.load().blade_beamform_tc_plan_size(B, A, F * R, P))
        self._plan = self._alloc((n,), "i8", "tensor")
        self._output = self._alloc((B + int(self._inc), F * R, T // (R * self._I), 1), "f32")

    @staticmethod
    def applies(it, A, F, T, P, B, R, I, detector, OP) -> bool:
        if it != "ci8" or not detector or OP != 1 or P != 2 or R not in (2, 4) or T % R:
            return False
        return _lib.load().blade_beamform_detect_tc_supported(B, A, F * R, T // R, P, 1, I) == 1

    def get_output(self):
        return self._output

    def process(self, step=0, stream=None):
        x, ph = as_vector(self._buffer), as_vector(self._phasors)
        pre, plan, out = _out(self._pre), _out(self._plan), _out(self._output)
        A, F, T, P = x.shape
        B, R, sh = ph.shape[0], self._R, _stream_handle(stream)
        _lib.call("blade_prechannelize_cf16", x.data_ptr(), pre.data_ptr(), A, F, T, P, R, int(self._circ), sh)
        _lib.call("blade_beamform_prepare_detect_tc_cf16", ph.data_ptr(), plan.data_ptr(), pre.data_ptr(),
                  out.data_ptr(), B, A, F * R, T // R, P, self._I, sh)
        if self._inc:  # beam row B: the incoherent beam through the detector
            row = out.data_ptr() + B * F * R * (T // (R * self._I)) * 4
            _lib.call("blade_incoherent_detect_cf16", pre.data_ptr(), ph.data_ptr(), row, A, F * R, T // R, P,
                      self._I, sh)
        return result.success


class ModeB(Module):
    """Bundles::ATA::ModeB<IT, OT> (include/blade/bundles/ata/mode_b.hh:17-225, Python
    binding python/blade/ext_modeb.cc:20-114): Cast -> Channelizer (pre-beamformer,
    rate R) -> Polarizer -> Phasor -> Beamformer::ATA -> [Detector] on one stream.

    The geometric half of the phasor stage (ERFA astrometry from antenna positions,
    beam coordinates, julian date and DUT1, src/modules/phasor/ata.cc:9-173) is not
    part of this library: the input carries either the phasors themselves
    (``phasors``, CF32 [B, A, F*R, 1, P]) or per-beam delays (``delays``, F64 [B, A]
    seconds), which the Phasor stage turns into phasors with the ``phasor_*``
    frequency fields and ``phasor_antenna_calibrations`` (ata.cc:176-208).  The
    position and coordinate fields are accepted and unused.

    With the detector enabled the incoherent beam is square-rooted, as the bundle
    configures it (mode_b.hh:146-147).  When the chain is Beamformer -> Detector
    alone (rate 1, no circular conversion, no incoherent beam, Stokes-I), it runs
    as one fused launch (tensor cores for CI8 input, FP32 CUDA cores for CF32).
    CI8 input at rate 2 or 4 with Stokes-I runs the pre-beamformer stages into
    exact FP16 and the tensor-core chain on the fine channels, plus the detected
    incoherent beam when enabled (``tensor_cores`` is True); every other
    configuration runs the module kernels in order."""

    taint = Taint.CONSUMER | Taint.PRODUCER

    @dataclass
    class config:
        input_shape: Sequence[int]
        output_shape: Sequence[int]
        pre_beamformer_channelizer_rate: int = 1
        pre_beamformer_polarizer_convert_to_circular: bool = False
        phasor_observation_frequency_hz: float = 0.0
        phasor_channel_bandwidth_hz: float = 0.0
        phasor_total_bandwidth_hz: float = 0.0
        phasor_frequency_start_index: int = 0
        phasor_reference_antenna_index: int = 0
        phasor_array_reference_position: object = None
        phasor_boresight_coordinate: object = None
        phasor_antenna_positions: object = None
        phasor_antenna_calibrations: object = None  # CF64 [A, F*R, 1, P], None = unit
        phasor_beam_coordinates: object = None
        beamformer_incoherent_beam: bool = False
        detector_enable: bool = False
        detector_integration_size: int = 1
        detector_number_of_output_polarizations: int = 1
        cast_block_size: int = 512
        channelizer_block_size: int = 512
        phasor_block_size: int = 512
        beamformer_block_size: int = 512
        polarizer_block_size: int = 512
        detector_block_size: int = 512

    @dataclass
    class input:
        buffer: object
        phasors: object = None
        delays: object = None

    def __init__(self, config, input, stream=None, it="ci8", ot="f32"):
        super().__init__()
        self.config, self._input = config, input
        c = config
        buf = as_vector(input.buffer)
        if buf.dtype != it or it not in ("ci8", "cf32"):
            _fail(f"ModeB takes CI8 or CF32 voltages (buffer is {buf.dtype}, expected {it}).")
        if ot not in ("f32", "cf32") or (ot == "f32") != bool(c.detector_enable):
            _fail("ModeB produces F32 with the detector enabled and CF32 without it.")
        if tuple(c.input_shape) != tuple(buf.shape):
            _fail(f"Expected input buffer size ({tuple(c.input_shape)}) mismatch with actual size "
                  f"({tuple(buf.shape)}).")
        A, F, T, P = buf.shape
        R = int(c.pre_beamformer_channelizer_rate)
        if (input.phasors is None) == (input.delays is None):
            _fail("ModeB needs exactly one of input.phasors (CF32 [B, A, F*R, 1, P]) or input.delays (F64 [B, A]).")
        self._stages = []
        self._phasor = None
        if input.delays is not None:
            d = as_vector(input.delays)
            if len(d.shape) != 2:
                _fail("ModeB delays must be an F64 delay_tensor [B, A].")
            self._phasor = Phasor(Phasor.config(
                number_of_beams=d.shape[0], number_of_antennas=A, number_of_frequency_channels=F * R,
                number_of_polarizations=P, observation_frequency_hz=c.phasor_observation_frequency_hz,
                channel_bandwidth_hz=c.phasor_channel_bandwidth_hz, total_bandwidth_hz=c.phasor_total_bandwidth_hz,
                frequency_start_index=c.phasor_frequency_start_index,
                antenna_calibrations=c.phasor_antenna_calibrations, block_size=c.phasor_block_size),
                Phasor.input(delays=input.delays))
            phasors = self._phasor.get_phasors()
        else:
            phasors = input.phasors
        ph = as_vector(phasors)
        B = ph.shape[0]
        if tuple(ph.shape) != (B, A, F * R, 1, P):
            _fail(f"Phasor shape {tuple(ph.shape)} does not match the channelized voltages ({B}, {A}, {F * R}, 1, {P}).")
        I, OP = int(c.detector_integration_size), int(c.detector_number_of_output_polarizations)
        self.fused = (c.detector_enable and R == 1 and not c.pre_beamformer_polarizer_convert_to_circular
                      and not c.beamformer_incoherent_beam and OP == 1 and P == 2 and I > 0 and T % I == 0)
        self.tensor_cores = (not self.fused) and _ModeBTensorCore.applies(it, A, F, T, P, B, R, I,
                                                                          bool(c.detector_enable), OP)
        if self.tensor_cores:
            last = _ModeBTensorCore(input.buffer, phasors, R, I, c.pre_beamformer_polarizer_convert_to_circular,
                                    c.beamformer_incoherent_beam)
            self._stages.append(last)
        elif self.fused:
            last = BeamformDetect(BeamformDetect.config(rate=1, integration_size=I, number_of_output_polarizations=1),
                                  BeamformDetect.input(buffer=input.buffer, phasors=phasors), it=it, ot="f32")
            self._stages.append(last)
        else:
            cast = Cast(Cast.config(c.cast_block_size), Cast.input(input.buffer), it=it, ot="cf32")
            chan = Channelizer(Channelizer.config(R, c.channelizer_block_size), Channelizer.input(cast.get_output()))
            polz = Polarizer(Polarizer.config(pol.xy, pol.lr if c.pre_beamformer_polarizer_convert_to_circular
                                              else pol.xy, c.polarizer_block_size),
                             Polarizer.input(chan.get_output()))
            bf = BeamformerATA(BeamformerATA.config(bool(c.beamformer_incoherent_beam), bool(c.detector_enable),
                                                    c.beamformer_block_size),
                               BeamformerATA.input(polz.get_output(), phasors))
            self._stages += [cast, chan, polz, bf]
            last = bf
            if c.detector_enable:
                last = Detector(Detector.config(I, OP, c.detector_block_size), Detector.input(bf.get_output()))
                self._stages.append(last)
        self._last = last
        out_shape = tuple(as_vector(last.get_output()).shape)
        if tuple(c.output_shape) != out_shape:
            _fail(f"Expected output buffer size ({tuple(c.output_shape)}) mismatch with actual size ({out_shape}).")

    def _set_slot(self, index: int) -> None:
        super()._set_slot(index)
        for m in ([self._phasor] if self._phasor is not None else []) + self._stages:
            m._set_slot(index)

    def get_config(self):
        return self.config

    def get_input_buffer(self):
        return self._input.buffer

    def get_phasors(self):
        return self._phasor.get_phasors() if self._phasor is not None else self._input.phasors

    def get_output(self):
        return self._last.get_output()

    def process(self, step=0, stream=None):
        for m in ([self._phasor] if self._phasor is not None else []) + self._stages:
            res = m.process(step, stream)
            if res != result.success:
                return res
        return result.success


# Registry used by blade_b200.module(): (name, telescope) -> (class, {(it, ot)}).
_CAST_PAIRS = {("i8", "i8"), ("i8", "f32"), ("f16", "f32"), ("f16", "f16"), ("f32", "i32"), ("f32", "f16"),
               ("f32", "f32"), ("ci8", "cf32"), ("ci8", "cf16"), ("ci8", "ci8"), ("cf32", "cf16"),
               ("cf32", "cf32"), ("cf16", "cf32"), ("cf16", "cf16"),
               # instantiated by the reference but rejected at construction (complex <-> real)
               ("f16", "cf32"), ("f16", "cf16"), ("f32", "cf32"), ("f32", "cf16"), ("cf32", "f16"),
               ("cf32", "f32"), ("cf16", "f16"), ("cf16", "f32")}

REGISTRY = {
    ("cast", "generic"): (Cast, _CAST_PAIRS),
    ("beamformer", "ata"): (BeamformerATA, {("cf32", "cf32")}),
    ("beamformer", "meerkat"): (BeamformerMeerKAT, {("cf32", "cf32")}),
    ("channelizer", "generic"): (Channelizer, {("cf32", "cf32")}),
    ("polarizer", "generic"): (Polarizer, {("cf32", "cf32"), ("cf16", "cf16")}),
    ("detector", "generic"): (Detector, {("cf32", "f32")}),
    ("gather", "generic"): (Gather, {("f32", "f32"), ("cf32", "cf32"), ("cf16", "cf16"), ("ci8", "ci8")}),
    ("permutation", "generic"): (Permutation, {("cf32", "cf32"), ("cf16", "cf16"), ("ci8", "ci8")}),
    ("duplicate", "generic"): (Duplicate, {("cf32", "cf32"), ("cf16", "cf16"), ("ci8", "ci8"), ("f32", "f32")}),
    ("phasor", "ata"): (Phasor, {("f64", "cf32")}),
    ("phasor", "generic"): (Phasor, {("f64", "cf32")}),
    ("beamform_detect", "ata"): (BeamformDetect, {("ci8", "f32"), ("cf32", "f32")}),
    ("beamform_detect", "generic"): (BeamformDetect, {("ci8", "f32"), ("cf32", "f32")}),
    ("modeh", "generic"): (ModeH, {("ci8", "f32"), ("ci8", "f16"), ("cf32", "f32"), ("cf32", "f16")}),
    ("modeb", "ata"): (ModeB, {("ci8", "cf32"), ("cf32", "cf32"), ("ci8", "f32"), ("cf32", "f32")}),
}
