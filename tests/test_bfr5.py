"""BFR5 recipe reader (Modules::Bfr5::Reader, src/modules/bfr5/base.cc): frame
conversions against their defining properties, the calibration layout, the
getters, and the module plumbing.  CPU only; no BFR5 file or HDF5 library is in
this image, so the recipe fields are passed as a mapping."""

import math

import numpy as np
import pytest

import blade_b200 as bl
from blade_b200 import bfr5

LON, LAT, ALT = math.radians(-121.470733), math.radians(40.815987), 1020.86  # the ATA


def _recipe(**kw):
    rng = np.random.default_rng(3)
    r = dict(nants=5, npol=2, nchan=3, nbeams=1, ntimes=8192,
             ras=[0.63722, 0.65063], decs=[1.07552424, 1.08426835],
             cal_all=rng.standard_normal((3, 2, 5)) + 1j * rng.standard_normal((3, 2, 5)),
             phase_center_ra=0.64169, phase_center_dec=1.079896295,
             antenna_positions=rng.standard_normal((5, 3)) * 100.0, antenna_position_frame="xyz",
             latitude=LAT, longitude=LON, altitude=ALT)
    r.update(kw)
    return r


def test_lla_to_ecef_known_answers():
    a = 6378137.0
    assert np.allclose(bfr5.lla_to_ecef(0.0, 0.0, 0.0), [a, 0.0, 0.0], atol=1e-6)
    assert np.allclose(bfr5.lla_to_ecef(math.pi / 2, 0.0, 10.0), [0.0, a + 10.0, 0.0], atol=1e-6)
    b = a * (1 - 1 / 298.257223563)  # polar radius
    assert np.allclose(bfr5.lla_to_ecef(0.3, math.pi / 2, 0.0), [0.0, 0.0, b], atol=1e-6)


def test_ecef_to_xyz_frame():
    ref = bfr5.lla_to_ecef(LON, LAT, ALT)
    assert np.allclose(bfr5.ecef_to_xyz([ref], LON, LAT, ALT), 0.0, atol=1e-6)
    # local up -> (cos lat, 0, sin lat); local east -> (0, 1, 0); north pole direction -> Z
    up = np.array([math.cos(LAT) * math.cos(LON), math.cos(LAT) * math.sin(LON), math.sin(LAT)])
    east = np.array([-math.sin(LON), math.cos(LON), 0.0])
    got = bfr5.ecef_to_xyz(ref + 100.0 * np.stack([up, east, [0.0, 0.0, 1.0]]), LON, LAT, ALT) / 100.0
    assert np.allclose(got[0], [math.cos(LAT), 0.0, math.sin(LAT)], atol=1e-9)  # 6e6 m cancels
    assert np.allclose(got[1], [0.0, 1.0, 0.0], atol=1e-9)
    assert np.allclose(got[2], [0.0, 0.0, 1.0], atol=1e-9)


def test_enu_and_ecef_routes_agree():
    # an ENU offset placed in ECEF about the reference gives the same XYZ by both routes
    rng = np.random.default_rng(1)
    enu = rng.standard_normal((7, 3)) * 300.0
    sl, cl, sp, cp = math.sin(LON), math.cos(LON), math.sin(LAT), math.cos(LAT)
    rot = np.array([[-sl, -sp * cl, cp * cl], [cl, -sp * sl, cp * sl], [0.0, cp, sp]])  # columns: E, N, U in ECEF
    ecef = bfr5.lla_to_ecef(LON, LAT, ALT) + enu @ rot.T
    assert np.allclose(bfr5.enu_to_xyz(enu, LON, LAT, ALT), bfr5.ecef_to_xyz(ecef, LON, LAT, ALT), atol=1e-7)
    # rotations keep baseline lengths
    x = bfr5.enu_to_xyz(enu, LON, LAT, ALT)
    assert np.allclose(np.linalg.norm(x, axis=1), np.linalg.norm(enu, axis=1))


@pytest.mark.parametrize("rate", [1, 4])
def test_reader_getters_and_calibration_layout(rate):
    r = _recipe()
    m = bl.module(bl.bfr5_reader, {"recipe": r, "channelizer_rate": rate}, {})
    assert m.get_total_shape() == (1 * 5, 3, 8192, 2)
    assert m.get_reference_position() == bl.lla(LON, LAT, ALT)
    assert m.get_boresight_coordinates() == bl.ra_dec(0.64169, 1.079896295)
    assert m.get_beam_coordinates() == [bl.ra_dec(0.63722, 1.07552424), bl.ra_dec(0.65063, 1.08426835)]
    assert np.allclose(np.array(m.get_antenna_positions()), r["antenna_positions"])  # xyz: unchanged
    cal = m.get_antenna_calibrations()
    assert cal.shape == (5, 3 * rate, 1, 2) and cal.dtype == np.complex128
    for a in range(5):
        for f in range(3 * rate):
            for p in range(2):
                assert cal[a, f, 0, p] == r["cal_all"][f // rate, p, a]
    assert m.process(0) == bl.result.success


@pytest.mark.parametrize("frame", ["ecef", "ENU"])
def test_reader_converts_positions(frame):
    r = _recipe(antenna_position_frame=frame)
    m = bl.module(bl.bfr5_reader, {"recipe": r, "channelizer_rate": 1}, {})
    conv = bfr5.ecef_to_xyz if frame == "ecef" else bfr5.enu_to_xyz
    assert np.allclose(np.array(m.get_antenna_positions()), conv(r["antenna_positions"], LON, LAT, ALT))


def test_reader_errors():
    with pytest.raises(RuntimeError):
        bl.module(bl.bfr5_reader, {"recipe": _recipe(antenna_position_frame="uvw")}, {})
    with pytest.raises(RuntimeError):
        bl.module(bl.bfr5_reader, {"recipe": _recipe(antenna_positions=np.zeros((4, 3)))}, {})
    r = _recipe()
    del r["cal_all"]
    with pytest.raises(RuntimeError):
        bl.module(bl.bfr5_reader, {"recipe": r}, {})
    with pytest.raises(RuntimeError):
        bl.module(bl.bfr5_reader, {"filepath": "/nonexistent/recipe.bfr5"}, {})
    with pytest.raises(RuntimeError):
        bl.module(bl.bfr5_reader, {"recipe": _recipe(), "channelizer_rate": 0}, {})


def test_reader_needs_hdf5_for_files(tmp_path):
    p = tmp_path / "recipe.bfr5"
    p.write_bytes(b"\x89HDF\r\n\x1a\n")
    try:
        import h5py  # noqa: F401
    except ImportError:
        with pytest.raises(RuntimeError, match="h5py"):
            bl.module(bl.bfr5_reader, {"filepath": str(p), "channelizer_rate": 1}, {})
    else:
        pytest.skip("h5py present: the file layer is exercised by real recipes")
