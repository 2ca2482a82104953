"""BFR5 beamformer recipes: the reader module Modules::Bfr5::Reader
(include/blade/modules/bfr5/reader.hh, src/modules/bfr5/base.cc:1-103).

A recipe carries what the Phasor module needs for a beamforming run: the array's
dimensions, the antenna positions and their frame, the array reference position,
the boresight (phase centre) and beam coordinates, and per-antenna calibration
coefficients.  The reference reads the file with bfr5c99 (an un-vendored HDF5
wrapper) and converts positions with radiointerferometryc99 (also un-vendored);
neither is in this tree, so:

  * the file layer reads the BFR5 groups through h5py when h5py is importable
    (``diminfo``: nants, npol, nchan, nbeams, ntimes; ``beaminfo``: ras, decs;
    ``calinfo``: cal_all [nchan][npol][nants] complex; ``obsinfo``:
    phase_center_ra, phase_center_dec; ``telinfo``: antenna_positions [nants][3],
    antenna_position_frame, latitude, longitude, altitude), and otherwise takes
    the same fields as a mapping (config ``recipe``);
  * the frame conversions restate the published conventions (Thompson, Moran &
    Swenson, Interferometry and Synthesis in Radio Astronomy, ch. 4): the
    array-centred XYZ frame has X in the reference meridian at the equator, Y
    towards hour angle -6 h (east), Z towards the north celestial pole;
      ECEF -> XYZ: subtract the reference position's ECEF (WGS84), rotate by
      -longitude about Z;
      ENU  -> XYZ: X = -sin(lat) N + cos(lat) U, Y = E, Z = cos(lat) N + sin(lat) U.
Parity with radiointerferometryc99 and bfr5c99 is therefore unpinned.

Deliberate differences from base.cc (each would read or write out of bounds
there): the calibrations are sized [nants, nchan * rate, 1, npol] (base.cc sizes
them [nbeams * nants, nchan, 1, npol] but writes nchan * rate channels and reads
nbeams * nants antennas of cal_all; reader.hh:110-116, base.cc:78-95), and a
frame other than xyz, ecef or enu is an error rather than left as is.  The two
reference call sites of the ECEF conversion pass latitude and longitude in
opposite orders (base.cc:49-54 latitude first, ata.cc:88-93 longitude first);
this module applies each angle as what it is.  At one beam and rate 1 the
calibrations agree.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Dict, List, Mapping, Optional

import numpy as np

from .constants import LLA, RA_DEC, XYZ, Taint, result
from .modules import REGISTRY, Module, _fail

# WGS84 ellipsoid
_WGS84_A = 6378137.0
_WGS84_F = 1.0 / 298.257223563
_WGS84_E2 = _WGS84_F * (2.0 - _WGS84_F)


def lla_to_ecef(longitude: float, latitude: float, altitude: float) -> np.ndarray:
    """Earth-centred, earth-fixed metres of a geodetic position (radians, metres)."""
    s, c = math.sin(latitude), math.cos(latitude)
    n = _WGS84_A / math.sqrt(1.0 - _WGS84_E2 * s * s)
    return np.array([(n + altitude) * c * math.cos(longitude), (n + altitude) * c * math.sin(longitude),
                     (n * (1.0 - _WGS84_E2) + altitude) * s])


def ecef_to_xyz(positions, longitude: float, latitude: float, altitude: float) -> np.ndarray:
    """[N][3] ECEF metres -> array-centred XYZ metres about the reference position."""
    p = np.asarray(positions, dtype=np.float64).reshape(-1, 3) - lla_to_ecef(longitude, latitude, altitude)
    c, s = math.cos(longitude), math.sin(longitude)
    return np.stack([c * p[:, 0] + s * p[:, 1], -s * p[:, 0] + c * p[:, 1], p[:, 2]], axis=1)


def enu_to_xyz(positions, longitude: float, latitude: float, altitude: float) -> np.ndarray:
    """[N][3] east-north-up metres about the reference position -> XYZ metres."""
    p = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    s, c = math.sin(latitude), math.cos(latitude)
    e, n, u = p[:, 0], p[:, 1], p[:, 2]
    return np.stack([-s * n + c * u, e, c * n + s * u], axis=1)


_FIELDS = {
    "diminfo": ("nants", "npol", "nchan", "nbeams", "ntimes"),
    "beaminfo": ("ras", "decs"),
    "calinfo": ("cal_all",),
    "obsinfo": ("phase_center_ra", "phase_center_dec"),
    "telinfo": ("antenna_positions", "antenna_position_frame", "latitude", "longitude", "altitude"),
}


def read_recipe(filepath: str) -> Dict[str, object]:
    """The recipe fields of a BFR5 file (HDF5, read through h5py)."""
    try:
        import h5py  # noqa: F401
    except ImportError:
        _fail(f"Reading '{filepath}' needs h5py (HDF5), which is not installed; pass the recipe's fields "
              "as the config's 'recipe' mapping instead.")
    import h5py

    out: Dict[str, object] = {}
    with h5py.File(filepath, "r") as fh:
        for grp, names in _FIELDS.items():
            for name in names:
                v = fh[grp][name][()]
                if isinstance(v, bytes):
                    v = v.decode()
                out[name] = v
    return out


class Bfr5Reader(Module):
    """Modules::Bfr5::Reader: config (filepath or recipe, channelizer_rate), no
    input, no output buffers; the getters of reader.hh:60-96."""

    taint = Taint.NONE

    @dataclass
    class config:
        filepath: str = ""
        channelizer_rate: int = 1
        block_size: int = 512
        recipe: Optional[Mapping[str, object]] = None

    @dataclass
    class input:
        pass

    def __init__(self, config, input, stream=None, it="cf64", ot="cf64"):
        super().__init__()
        self.config, self._input = config, input
        if config.channelizer_rate < 1:
            _fail(f"Channelizer rate ({config.channelizer_rate}) must be at least 1.")
        if config.recipe is not None:
            r = dict(config.recipe)
        else:
            import os

            if not os.path.exists(config.filepath):
                _fail(f"Input file ({config.filepath}) doesn't exist.")
            r = read_recipe(config.filepath)
        missing = [n for names in _FIELDS.values() for n in names if n not in r]
        if missing:
            _fail(f"Recipe is missing {', '.join(missing)}.")
        self._dims = {k: int(np.asarray(r[k]).reshape(-1)[0]) for k in _FIELDS["diminfo"]}
        nants, npol, nchan = self._dims["nants"], self._dims["npol"], self._dims["nchan"]
        ras = np.asarray(r["ras"], dtype=np.float64).reshape(-1)
        decs = np.asarray(r["decs"], dtype=np.float64).reshape(-1)
        if len(ras) != len(decs):
            _fail(f"Beam coordinates: {len(ras)} right ascensions against {len(decs)} declinations.")
        self._beams: List[RA_DEC] = [RA_DEC(float(a), float(d)) for a, d in zip(ras, decs)]
        self._lla = LLA(float(r["longitude"]), float(r["latitude"]), float(r["altitude"]))
        self._boresight = RA_DEC(float(r["phase_center_ra"]), float(r["phase_center_dec"]))
        pos = np.asarray(r["antenna_positions"], dtype=np.float64).reshape(-1, 3)
        if len(pos) != nants:
            _fail(f"{len(pos)} antenna positions for {nants} antennas.")
        frame = str(r["antenna_position_frame"]).strip()
        if frame.lower() == "ecef":
            pos = ecef_to_xyz(pos, *self._lla)
        elif frame.lower() == "enu":
            pos = enu_to_xyz(pos, *self._lla)
        elif frame.lower() != "xyz":
            _fail(f"Unknown antenna position frame '{frame}' (xyz, ecef or enu).")
        self._positions: List[XYZ] = [XYZ(*map(float, p)) for p in pos]
        cal = np.asarray(r["cal_all"])
        if cal.dtype.names:  # HDF5 compound (r, i) records
            re_name, im_name = cal.dtype.names[:2]
            cal = cal[re_name] + 1j * cal[im_name]
        cal = np.asarray(cal, dtype=np.complex128).reshape(nchan, npol, nants)
        rate = int(config.channelizer_rate)
        # [nants, nchan * rate, 1, npol]: every fine channel of a coarse channel
        # takes the coarse channel's coefficient (base.cc:77-95)
        self._cal = np.ascontiguousarray(np.repeat(cal.transpose(2, 0, 1), rate, axis=1)[:, :, None, :])

    def get_config(self):
        return self.config

    def get_total_shape(self):
        """[nbeams * nants, nchan, ntimes, npol], as reader.hh:60-67 defines it."""
        d = self._dims
        return (d["nbeams"] * d["nants"], d["nchan"], d["ntimes"], d["npol"])

    def get_reference_position(self) -> LLA:
        return self._lla

    def get_boresight_coordinates(self) -> RA_DEC:
        return self._boresight

    def get_antenna_positions(self) -> List[XYZ]:
        """Antenna positions in the array-centred XYZ frame (metres)."""
        return self._positions

    def get_beam_coordinates(self) -> List[RA_DEC]:
        return self._beams

    def get_antenna_calibrations(self) -> np.ndarray:
        """CF64 [nants, nchan * channelizer_rate, 1, npol] (the Phasor module's
        antenna_calibrations layout)."""
        return self._cal

    def process(self, step=0, stream=None):
        return result.success


REGISTRY[("bfr5_reader", "generic")] = (Bfr5Reader, {("cf64", "cf64")})
