"""Constants of the reference's Python surface (python/blade/_internal/__init__.py:43-75,
python/blade/ext_const.cc): telescopes, devices, element types, module names,
polarisation bases and Result codes."""

from __future__ import annotations

import enum


class Constant:
    def __init__(self, value: str):
        self._value = value

    def __repr__(self):
        return f"Constant(value={self._value})"

    @property
    def value(self) -> str:
        return self._value

    def __eq__(self, other):
        return isinstance(other, Constant) and other._value == self._value

    def __hash__(self):
        return hash(self._value)


telescope_list = ["ata", "vla", "meerkat", "generic"]
device_list = ["cpu", "cuda", "unified"]
dtypes = ["f16", "f32", "f64", "i8", "i32", "cf16", "cf32", "cf64", "ci8"]
module_list = ["beamformer", "cast", "channelizer", "duplicate", "detector", "gather", "permutation", "phasor",
               "polarizer", "beamform_detect", "modeb", "modeh", "guppi_reader", "guppi_writer", "bfr5_reader"]

ata, vla, meerkat, generic = (Constant(n) for n in telescope_list)
cpu, cuda, unified = (Constant(n) for n in device_list)
f16, f32, f64, i8, i32, cf16, cf32, cf64, ci8 = (Constant(n) for n in dtypes)
(beamformer, cast, channelizer, duplicate, detector, gather, permutation, phasor, polarizer, beamform_detect,
 modeb, modeh, guppi_reader, guppi_writer, bfr5_reader) = (Constant(n) for n in module_list)


class pol(enum.IntEnum):
    """Polarisation bases (include/blade/types.hh:198-205)."""
    x = 0
    y = 1
    l = 2  # noqa: E741
    r = 3
    xy = 4
    lr = 5


class result(enum.IntEnum):
    """Blade::Result (include/blade/macros.hh:31-48); bit 4 marks soft errors."""
    success = 0
    error = 1
    cuda_error = 2
    assertion_error = 3
    runner_queue_full = 0 | (1 << 4)
    runner_queue_empty = 1 | (1 << 4)
    runner_queue_none_available = 2 | (1 << 4)
    pipeline_exhausted = 3 | (1 << 4)


class Taint(enum.IntFlag):
    """Module taints (include/blade/macros.hh:11-21)."""
    NONE = 0
    CONSUMER = 1 << 0
    PRODUCER = 1 << 1
    MODIFIER = 1 << 2
    CHRONOUS = 1 << 3


# Coordinates of the Phasor configuration (include/blade/types.hh:14-40; python
# helpers bl.xyz / bl.lla / bl.ra_dec as the reference's bindings name them).
from collections import namedtuple as _nt  # noqa: E402

XYZ = _nt("XYZ", "x y z")
LLA = _nt("LLA", "lon lat alt")
RA_DEC = _nt("RA_DEC", "ra dec")


def xyz(x, y, z):
    return XYZ(float(x), float(y), float(z))


def lla(lon, lat, alt):
    return LLA(float(lon), float(lat), float(alt))


def ra_dec(ra, dec):
    return RA_DEC(float(ra), float(dec))
