"""CPU: GUPPI RAW reader and writer modules (blade_b200.guppi; the reference's
include/blade/modules/guppi/{reader,writer}.hh over guppirawc99, which is not
vendored, so these tests pin the restated file layout by round trips)."""

import os

import numpy as np
import pytest

import blade_b200 as bl
from blade_b200 import guppi

A, C, T, P = 3, 4, 16, 2


def _blocks(n, seed=0):
    rng = np.random.default_rng(seed)
    return [rng.integers(-128, 128, size=(A, C, T, P, 2), dtype=np.int8) for _ in range(n)]


HDR = {"CHAN_BW": 0.5, "OBSFREQ": 6000.25, "SCHAN": 352, "SYNCTIME": 1649366473, "PIPERBLK": 8, "DUT1": -0.125,
       "PKTIDX": 1000, "TBIN": 2e-6}


def test_header_records_round_trip():
    rec = b"".join(guppi._card(k, v) for k, v in {"BLOCSIZE": 1024, "OBSFREQ": 6000.25, "SRC_NAME": "3C84",
                                                   "DIRECTIO": 1, "ONSRC": True}.items())
    rec += b"END".ljust(80)
    assert len(rec) % 80 == 0
    hdr, n = guppi.parse_header(rec + b"\0" * 100)
    assert n == len(rec)
    assert hdr == {"BLOCSIZE": 1024, "OBSFREQ": 6000.25, "SRC_NAME": "3C84", "DIRECTIO": 1, "ONSRC": True}
    with pytest.raises(ValueError):
        guppi.parse_header(rec[:-80])
    with pytest.raises(ValueError):
        guppi._card("TOOLONGKEY", 1)


@pytest.mark.parametrize("directio,files", [(True, 2), (False, 1), (True, 3)])
def test_reader_full_block_steps_bit_exact(tmp_path, directio, files):
    blocks = _blocks(6)
    paths = guppi.write_ci8_recording(str(tmp_path / "rec"), blocks, HDR, directio=directio, files=files)
    assert len(paths) == files
    if directio:
        assert all(os.path.getsize(p) % 512 == 0 for p in paths)
    r = bl.module(bl.guppi_reader, {"filepath": paths[0]}, {})
    assert r.get_total_output_buffer_shape() == (A, C, 6 * T, P)
    assert r.get_step_output_buffer_shape() == (A, C, T, P)
    assert r.get_number_of_steps() == 6
    full = np.concatenate(blocks, axis=2)
    got = []
    while r.process() == bl.result.success:
        got.append(r.get_step_output_buffer().as_numpy().copy())
    assert len(got) == 6
    np.testing.assert_array_equal(np.concatenate(got, axis=2), full)


def test_reader_sub_steps_cover_channels_then_time(tmp_path):
    blocks = _blocks(3, seed=1)
    guppi.write_ci8_recording(str(tmp_path / "rec"), blocks, HDR)
    # stem path, steps of 2 channels x 24 time samples (crossing block boundaries)
    r = bl.module(bl.guppi_reader, {"filepath": str(tmp_path / "rec"), "step_number_of_time_samples": 24,
                                     "step_number_of_frequency_channels": 2}, {})
    full = np.concatenate(blocks, axis=2)
    assert r.get_number_of_steps() == (A * C * 3 * T) // (A * 2 * 24)
    expect = [(c0, t0) for t0 in (0, 24) for c0 in (0, 2)]
    for c0, t0 in expect:
        assert r.process() == bl.result.success
        np.testing.assert_array_equal(r.get_step_output_buffer().as_numpy(), full[:, c0:c0 + 2, t0:t0 + 24])
    assert r.process() == bl.result.pipeline_exhausted  # 0 samples left < 24


def test_reader_metadata_and_julian_date(tmp_path):
    guppi.write_ci8_recording(str(tmp_path / "rec"), _blocks(2), HDR)
    r = bl.module(bl.guppi_reader, {"filepath": str(tmp_path / "rec.0000.raw")}, {})
    assert r.get_channel_bandwidth() == 0.5e6
    assert r.get_total_bandwidth() == 0.5e6 * C
    assert r.get_channel_start_index() == 352
    assert r.get_observation_frequency() == 6000.25e6
    for block in range(2):
        assert r.process() == bl.result.success
        pktidx = HDR["PKTIDX"] + block * HDR["PIPERBLK"] + 0.5 * HDR["PIPERBLK"]
        unix = HDR["SYNCTIME"] + pktidx * (1.0 / 0.5e6) * T / HDR["PIPERBLK"]
        assert r.get_step_output_julian_date().as_numpy()[0] == pytest.approx(unix / 86400.0 + 2440587.5, abs=1e-9)
        assert r.get_step_output_dut().as_numpy()[0] == -0.125


def test_reader_rejects_bad_input(tmp_path):
    with pytest.raises(RuntimeError):
        bl.module(bl.guppi_reader, {"filepath": str(tmp_path / "missing")}, {})
    with pytest.raises(RuntimeError):
        bl.module(bl.guppi_reader, {"filepath": ""}, {})
    p = tmp_path / "trunc.0000.raw"
    guppi.write_ci8_recording(str(tmp_path / "trunc"), _blocks(1), HDR, directio=False)
    data = p.read_bytes()
    p.write_bytes(data[:-10])
    with pytest.raises(RuntimeError):
        bl.module(bl.guppi_reader, {"filepath": str(p)}, {})


@pytest.mark.parametrize("dtype,batches", [("cf32", 1), ("cf16", 1), ("cf32", 2)])
def test_writer_blocks_read_back(tmp_path, dtype, batches):
    rng = np.random.default_rng(3)
    buf = bl.array_tensor((A, C, T, P), dtype=getattr(bl, dtype), device=bl.cpu)
    w = bl.module(bl.guppi_writer, {"filepath": str(tmp_path / "out"), "directio": True,
                                     "input_frequency_batches": batches}, {"buffer": buf},
                  it=getattr(bl, dtype), ot=getattr(bl, dtype))
    w.header_put("OBSFREQ", 1420.0)
    w.header_put("SRC_NAME", "TEST")
    written = []
    for k in range(3):
        x = (rng.standard_normal((A, C, T, P)) + 1j * rng.standard_normal((A, C, T, P))).astype(np.complex64)
        if dtype == "cf32":
            buf.as_numpy()[...] = x
        else:
            buf.as_numpy()[...] = np.stack([x.real, x.imag], axis=-1).astype(np.float16)
        assert w.process() == bl.result.success
        written.append(buf.as_numpy().copy())
    blocks, first = guppi._scan(str(tmp_path / "out"))
    assert len(blocks) == 3
    item = 8 if dtype == "cf32" else 4
    for k, (fname, off, hdr) in enumerate(blocks):
        assert hdr["BLOCSIZE"] == A * C * T * P * item and hdr["OBSNCHAN"] == A * C and hdr["NANTS"] == A
        assert hdr["NPOL"] == 4 and hdr["NBITS"] == item * 4 and hdr["NBEAM"] == A
        assert hdr["DATATYPE"] == "FLOAT" and hdr["PKTIDX"] == T * k and hdr["OBSFREQ"] == 1420.0
        assert hdr["SRC_NAME"] == "TEST" and off % 512 == 0
        raw = np.fromfile(fname, dtype=np.uint8, count=hdr["BLOCSIZE"], offset=off)
        x = written[k]
        if batches > 1:
            x = np.concatenate([np.ascontiguousarray(b).reshape(-1) for b in np.split(x, batches, axis=1)])
        np.testing.assert_array_equal(raw, np.ascontiguousarray(x).view(np.uint8).reshape(-1))


def test_writer_rejects_device_buffers_and_bad_batches(tmp_path):
    buf = bl.array_tensor((A, C, T, P), dtype=bl.cf32, device=bl.cpu)
    with pytest.raises(RuntimeError):
        bl.module(bl.guppi_writer, {"filepath": str(tmp_path / "o"), "input_frequency_batches": 3}, {"buffer": buf})
