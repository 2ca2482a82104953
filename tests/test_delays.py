"""Geometric delays (the astrometric half of Modules::Phasor::ATA, ata.cc:9-173).

The reference computes them with ERFA and checks them against astropy at rtol 0.5
(tests/modules/phasor/advanced.py); neither is available here, so parity with
ERFA is unpinned.  What is pinned: each published formula against the worked
examples of Meeus, Astronomical Algorithms (2nd ed.) — sidereal time (examples
12.a, 12.b), nutation (22.a, within the four-term series' stated 0.5" / 0.1"),
precession (21.b) — the reference's own route (array-centred XYZ, UVW of the hour
angle and declination) against the terrestrial-frame projection, and the
library's host astrometry and device delays against this oracle.  Inputs are the
reference test's ATA antenna positions, boresight and beams
(tests/modules/phasor/advanced.py:46-79, 97)."""

import ctypes as C
import math

import numpy as np
import pytest

from blade_b200 import _lib
from oracle import formulas as O

AS = math.pi / (180 * 3600)
POS = [(-2524041.5388905862, -4123587.965024342, 4147646.4222955606),
       (-2524068.187873109, -4123558.735413135, 4147656.21282186),
       (-2524087.2078100787, -4123532.397416349, 4147670.9866770394),
       (-2524103.384010733, -4123511.111598937, 4147682.4133068994),
       (-2524056.730228759, -4123515.287949227, 4147706.4850287656),
       (-2523986.279601761, -4123497.427940991, 4147766.732988923),
       (-2523824.598229116, -4123527.93080514, 4147833.98936114)]
LON, LAT, ALT = math.radians(-121.470733), math.radians(40.815987), 1020.86
BORESIGHT = (0.64169, 1.079896295)
BEAMS = [(0.63722, 1.07552424), (0.65063, 1.08426835)]
JD = 1649366473.0 / 86400 + 2440587.5


def test_sidereal_time_known_answers():
    assert abs(O.gmst_deg(2446895.5) - 197.693195) < 2e-6  # 1987 Apr 10, 0h UT: 13h10m46.3668s
    jd = 2446895.5 + (19 + 21 / 60) / 24                    # 19h21m UT: 8h34m57.0896s
    assert abs(O.gmst_deg(jd) - (8 + 34 / 60 + 57.0896 / 3600) * 15) < 2e-6


def test_nutation_known_answer():
    t = (2446895.5 - 2451545.0) / 36525                     # 1987 Apr 10, 0h TD
    dpsi, deps, eps0 = O.nutation(t)
    assert abs(dpsi / AS - (-3.788)) < 0.5
    assert abs(deps / AS - 9.443) < 0.1
    assert abs(eps0 / AS - (23 * 3600 + 26 * 60 + 27.407)) < 0.01
    assert abs((eps0 + deps) / AS - (23 * 3600 + 26 * 60 + 36.850)) < 0.1


def test_precession_known_answer():
    # theta Persei from J2000.0 to 2028 Nov 13.19 TD, proper motion applied first
    jde = 2462088.69
    yrs = (jde - 2451545.0) / 365.25
    ra0 = (2 + 44 / 60 + (11.986 + yrs * 0.03425) / 3600) * 15 * math.pi / 180
    de0 = (49 + 13 / 60 + (42.48 - yrs * 0.0895) / 3600) * math.pi / 180
    p = np.array([math.cos(de0) * math.cos(ra0), math.cos(de0) * math.sin(ra0), math.sin(de0)])
    q = O.precession_matrix((jde - 2451545.0) / 36525) @ p
    ra = math.atan2(q[1], q[0]) % (2 * math.pi)
    de = math.asin(q[2])
    assert abs(ra * 180 / math.pi / 15 * 3600 - (2 * 3600 + 46 * 60 + 11.331)) < 0.002  # seconds of time
    assert abs(de * 180 / math.pi * 3600 - (49 * 3600 + 20 * 60 + 54.54)) < 0.02        # arcseconds


def test_hour_angle_route_matches_projection():
    d1 = O.geometric_delays(POS, 0, BORESIGHT, BEAMS, JD, 0.0)
    d2 = O.delays_via_hour_angle(POS, 0, LON, BORESIGHT, BEAMS, JD, 0.0)
    assert np.abs(d1 - d2).max() < 1e-18
    assert np.all(d1[:, 0] == 0.0)                       # the reference antenna
    assert np.abs(d1).max() > 1e-9                       # beams ~0.3 deg off a ~300 m array
    d0 = O.geometric_delays(POS, 0, BORESIGHT, [BORESIGHT], JD, 0.0)
    assert np.all(d0 == 0.0)                             # a beam at the boresight


@pytest.mark.parametrize("ra,dec,jd,dut1", [(0.64169, 1.079896295, JD, 0.0), (3.5, -0.7, 2460000.25, 0.12),
                                            (5.9, 0.2, 2451545.0, -0.3)])
def test_host_astrometry_matches_oracle(ra, dec, jd, dut1):
    out = (C.c_double * 3)()
    _lib.call("blade_source_direction", ra, dec, jd, dut1, out)
    ref = O.source_itrs(ra, dec, jd, dut1)
    assert np.abs(np.array(out[:]) - ref).max() < 1e-13


@pytest.mark.gpu
def test_device_delays_match_oracle(cuda):
    import torch

    pos = np.ascontiguousarray(POS, dtype=np.float64)
    beams = np.ascontiguousarray(BEAMS, dtype=np.float64)
    lla = np.array([LON, LAT, ALT])
    d = torch.full((len(BEAMS), len(POS)), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call("blade_geometric_delays", pos.ctypes.data, len(POS), 2, lla.ctypes.data, BORESIGHT[0], BORESIGHT[1],
              beams.ctypes.data, len(BEAMS), JD, 0.05, d.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref = O.geometric_delays(POS, 2, BORESIGHT, BEAMS, JD, 0.05)
    assert np.abs(d.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.gpu
def test_phasor_module_geometric_form(cuda):
    import torch

    import blade_b200 as bl

    A, F, P = len(POS), 16, 2
    date = bl.tensor(1, dtype=bl.f64, device=bl.cpu)
    dut = bl.tensor(1, dtype=bl.f64, device=bl.cpu)
    date.as_torch()[0] = JD
    dut.as_torch()[0] = 0.0
    cfg = {"number_of_antennas": A, "number_of_frequency_channels": F, "number_of_polarizations": P,
           "observation_frequency_hz": 6500.125e6, "channel_bandwidth_hz": 0.5e6, "total_bandwidth_hz": 1.024e9,
           "frequency_start_index": 352, "reference_antenna_index": 0,
           "array_reference_position": bl.lla(LON, LAT, ALT), "boresight_coordinate": bl.ra_dec(*BORESIGHT),
           "antenna_positions": [bl.xyz(*p) for p in POS], "beam_coordinates": [bl.ra_dec(*b) for b in BEAMS]}
    mod = bl.module(bl.phasor, cfg, (date, dut), telescope=bl.ata)
    mod.process(0, bl.stream())
    torch.cuda.synchronize()
    delays = O.geometric_delays(POS, 0, BORESIGHT, BEAMS, JD, 0.0)
    ref = O.phasors_from_delays(delays, np.ones((A, F, 1, P)), 6500.125e6, 0.5e6, 1.024e9, 352)
    got = mod.get_phasors().as_torch().cpu().numpy()
    assert np.abs(got - ref).max() < 2e-6
