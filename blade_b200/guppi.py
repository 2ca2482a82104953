"""GUPPI RAW voltage files: the reader and writer modules of the path's input and
output side (include/blade/modules/guppi/{reader,writer}.hh, src/modules/guppi/
{reader,writer}.cc).

The reference delegates the file format to guppirawc99, an un-vendored submodule
(no source or version pin in the reference tree), so this module restates the
published GUPPI RAW layout; parity with that library is unpinned.  A file is a
sequence of blocks, each

  * a header of 80-character ASCII records ``KEYWORD = value`` (keyword left-
    justified in 8 columns, ``=`` in column 9, the value from column 11; strings
    in single quotes), closed by a record starting with ``END``; with
    ``DIRECTIO = 1`` the header is padded with spaces to a multiple of 512 bytes;
  * ``BLOCSIZE`` bytes of data, padded with zeros to a multiple of 512 bytes when
    ``DIRECTIO = 1``.

The data of a block is ``[NANTS][OBSNCHAN / NANTS][NTIME][NPOL]`` complex samples
of ``NBITS`` bits per component (NPOL = 4 in the header means two polarisations
of complex samples, as GUPPI writes them), so
``NTIME = BLOCSIZE * 8 / (OBSNCHAN * npol * 2 * NBITS)``.  A recording is a
numbered file sequence ``<stem>.0000.raw``, ``<stem>.0001.raw``, ...; the reader
concatenates the blocks of all files along time.

Reader steps (``get_step_output_buffer_shape``) tile the total
``[aspects, channels, time, pols]`` array: within one time window every
(aspect, channel) tile is produced before time advances, and the reader reports
``result.pipeline_exhausted`` when fewer than a step's time samples remain.  The
step's julian date is that of the packet index at the middle of the block
(``reader.cc:127-139``), unix = SYNCTIME + PKTIDX * TBIN * NTIME / PIPERBLK with
TBIN = 1 / CHAN_BW, and JD = unix / 86400 + 2440587.5.
"""

from __future__ import annotations

import os
import re
from dataclasses import dataclass
from typing import Dict, List, Tuple

import numpy as np

from .constants import Taint, result
from .memory import Vector, as_vector
from .modules import REGISTRY, Module, _fail

_CARD = 80
_DIRECTIO_ALIGN = 512


def _card(key: str, value) -> bytes:
    if len(key) > 8:
        raise ValueError(f"GUPPI header keyword {key!r} is longer than 8 characters")
    if isinstance(value, str):
        v = "'" + value.replace("'", "''").ljust(8) + "'"
    elif isinstance(value, bool):
        v = ("T" if value else "F").rjust(20)
    elif isinstance(value, (int, np.integer)):
        v = str(int(value)).rjust(20)
    else:
        v = repr(float(value)).rjust(20)
    text = f"{key.upper():<8}= {v}"
    if len(text) > _CARD:
        raise ValueError(f"GUPPI header record for {key!r} exceeds 80 characters")
    return text.ljust(_CARD).encode("ascii")


def _parse_value(raw: str):
    raw = raw.strip()
    if raw.startswith("'"):
        end = raw.rfind("'")
        return raw[1:end].replace("''", "'").rstrip()
    if raw in ("T", "F"):
        return raw == "T"
    try:
        return int(raw)
    except ValueError:
        pass
    try:
        return float(raw)
    except ValueError:
        return raw


def parse_header(buf: bytes) -> Tuple[Dict[str, object], int]:
    """Header records of one block -> (dict, header length in bytes before padding)."""
    hdr: Dict[str, object] = {}
    pos = 0
    while pos + _CARD <= len(buf):
        rec = buf[pos:pos + _CARD].decode("ascii", errors="replace")
        pos += _CARD
        if rec.startswith("END") and rec[3:].strip() == "":
            return hdr, pos
        if len(rec) > 9 and rec[8] == "=":
            hdr[rec[:8].strip()] = _parse_value(rec[9:])
    raise ValueError("GUPPI RAW header without an END record")


def _pad(n: int) -> int:
    return (n + _DIRECTIO_ALIGN - 1) // _DIRECTIO_ALIGN * _DIRECTIO_ALIGN


@dataclass(frozen=True)
class Datashape:
    n_aspect: int
    n_aspectchan: int
    n_time: int
    n_pol: int
    n_bit: int

    @staticmethod
    def from_header(h: Dict[str, object]) -> "Datashape":
        for key in ("BLOCSIZE", "OBSNCHAN", "NBITS"):
            if key not in h:
                raise ValueError(f"GUPPI RAW header lacks {key}")
        nants = int(h.get("NANTS", 1)) or 1
        npol = int(h.get("NPOL", 1))
        npol = 2 if npol == 4 else npol
        nchan, nbits, bloc = int(h["OBSNCHAN"]), int(h["NBITS"]), int(h["BLOCSIZE"])
        if nchan % nants:
            raise ValueError(f"OBSNCHAN ({nchan}) is not a multiple of NANTS ({nants})")
        bits_per_time = nchan * npol * 2 * nbits
        if (bloc * 8) % bits_per_time:
            raise ValueError("BLOCSIZE is not a whole number of time samples")
        return Datashape(nants, nchan // nants, bloc * 8 // bits_per_time, npol, nbits)


def _stem_and_start(path: str) -> Tuple[str, int]:
    m = re.match(r"^(.*)\.(\d{4})\.raw$", path)
    if m:
        return m.group(1), int(m.group(2))
    return path, 0


def _scan(path: str):
    """(blocks, first header): blocks = [(file, data offset, header dict)] over the file sequence."""
    stem, start = _stem_and_start(path)
    blocks = []
    idx = start
    while True:
        fname = f"{stem}.{idx:04d}.raw"
        if not os.path.exists(fname):
            break
        size = os.path.getsize(fname)
        with open(fname, "rb") as fh:
            off = 0
            while off < size:
                fh.seek(off)
                head = fh.read(min(size - off, 1 << 20))
                hdr, hlen = parse_header(head)
                directio = int(hdr.get("DIRECTIO", 0)) == 1
                data_off = off + (_pad(hlen) if directio else hlen)
                bloc = int(hdr["BLOCSIZE"])
                if data_off + bloc > size:
                    raise ValueError(f"{fname}: truncated block at byte {off}")
                blocks.append((fname, data_off, hdr))
                off = data_off + (_pad(bloc) if directio else bloc)
        idx += 1
    if not blocks:
        raise FileNotFoundError(f"no GUPPI RAW file at {stem}.{start:04d}.raw")
    return blocks, blocks[0][2]


class GuppiReader(Module):
    """Modules::Guppi::Reader<CI8> (include/blade/modules/guppi/reader.hh:16-128,
    src/modules/guppi/reader.cc:52-168).  Steps land in a host (pinned when CUDA is
    present) CI8 array_tensor [aspects, channels, time, pols]."""

    taint = Taint.PRODUCER

    @dataclass
    class config:
        filepath: str
        step_number_of_time_samples: int = 0
        step_number_of_frequency_channels: int = 0
        step_number_of_aspects: int = 0
        block_size: int = 512

    @dataclass
    class input:
        pass

    def __init__(self, config, input=None, stream=None, it=None, ot="ci8"):
        super().__init__()
        if ot != "ci8":
            _fail("The GUPPI reader produces CI8.")
        if not config.filepath:
            _fail(f"Input file ({config.filepath}) is invalid.")
        self.config = config
        try:
            self._blocks, self._hdr = _scan(config.filepath)
        except (OSError, ValueError) as e:
            _fail(f"Errored opening {config.filepath}: {e}")
        self._shape = Datashape.from_header(self._hdr)
        if self._shape.n_bit != 8:
            _fail(f"The GUPPI reader supports 8-bit samples (NBITS = {self._shape.n_bit}).")
        for _, _, h in self._blocks:
            if Datashape.from_header(h) != self._shape:
                _fail("GUPPI RAW blocks of one recording must share their data shape.")
        ds = self._shape
        c = config
        c.step_number_of_aspects = c.step_number_of_aspects or ds.n_aspect
        c.step_number_of_frequency_channels = c.step_number_of_frequency_channels or ds.n_aspectchan
        c.step_number_of_time_samples = c.step_number_of_time_samples or ds.n_time
        if ds.n_aspect % c.step_number_of_aspects or ds.n_aspectchan % c.step_number_of_frequency_channels:
            _fail("Step aspects and channels must divide the recording's aspects and channels.")
        self._piperblk = int(self._hdr.get("PIPERBLK", 0)) or ds.n_time
        self._pos = (0, 0, 0)  # (time, aspect, channel) of the next step
        self._step_buf = Vector(self.get_step_output_buffer_shape(), "ci8", "cpu", "array_tensor")
        self._jd = Vector((1,), "f64", "cpu", "tensor")
        self._dut1 = Vector((1,), "f64", "cpu", "tensor")

    # -- shapes and metadata (reader.hh:60-85, reader.cc:106-124) -------------
    def get_total_output_buffer_shape(self):
        ds = self._shape
        return (ds.n_aspect, ds.n_aspectchan, ds.n_time * len(self._blocks), ds.n_pol)

    def get_step_output_buffer_shape(self):
        c = self.config
        return (c.step_number_of_aspects, c.step_number_of_frequency_channels, c.step_number_of_time_samples,
                self._shape.n_pol)

    def get_number_of_steps(self) -> int:
        return int(np.prod(self.get_total_output_buffer_shape()) // np.prod(self.get_step_output_buffer_shape()))

    def get_channel_bandwidth(self) -> float:
        return float(self._hdr.get("CHAN_BW", 0.0)) * 1e6

    def get_total_bandwidth(self) -> float:
        return self.get_channel_bandwidth() * self.config.step_number_of_frequency_channels

    def get_channel_start_index(self) -> int:
        return int(self._hdr.get("SCHAN", 0))

    def get_observation_frequency(self) -> float:
        return float(self._hdr.get("OBSFREQ", 0.0)) * 1e6

    def get_config(self):
        return self.config

    def get_step_output_buffer(self):
        return self._step_buf

    def get_step_output_julian_date(self):
        return self._jd

    def get_step_output_dut(self):
        return self._dut1

    get_output = get_step_output_buffer

    # -- reading --------------------------------------------------------------
    def _block_samples(self, b: int) -> np.memmap:
        fname, off, _ = self._blocks[b]
        ds = self._shape
        return np.memmap(fname, dtype=np.int8, mode="r", offset=off,
                         shape=(ds.n_aspect, ds.n_aspectchan, ds.n_time, ds.n_pol, 2))

    def _julian_date(self, block: int) -> float:
        h = self._blocks[block][2]
        ds = self._shape
        tbin = 1.0 / self.get_channel_bandwidth() if self.get_channel_bandwidth() else 0.0
        pktidx = int(h.get("PKTIDX", 0)) + (0.5 * self._piperblk)
        unix = float(h.get("SYNCTIME", 0)) + pktidx * tbin * ds.n_time / self._piperblk
        return unix / 86400.0 + 2440587.5

    def process(self, step=0, stream=None):
        c, ds = self.config, self._shape
        t0, a0, c0 = self._pos
        total_t = ds.n_time * len(self._blocks)
        nt = c.step_number_of_time_samples
        if total_t - t0 < nt:
            return result.pipeline_exhausted
        out = self._step_buf.as_numpy().view(np.int8).reshape(c.step_number_of_aspects,
                                                               c.step_number_of_frequency_channels, nt, ds.n_pol, 2)
        na, nc = c.step_number_of_aspects, c.step_number_of_frequency_channels
        done = 0
        while done < nt:
            b, tb = divmod(t0 + done, ds.n_time)
            n = min(nt - done, ds.n_time - tb)
            out[:, :, done:done + n] = self._block_samples(b)[a0:a0 + na, c0:c0 + nc, tb:tb + n]
            done += n
        self._jd.as_numpy()[0] = self._julian_date(t0 // ds.n_time)
        self._dut1.as_numpy()[0] = float(self._blocks[t0 // ds.n_time][2].get("DUT1", 0.0))
        # channels first, then aspects, then time
        c0 += nc
        if c0 >= ds.n_aspectchan:
            c0 = 0
            a0 += na
            if a0 >= ds.n_aspect:
                a0 = 0
                t0 += nt
        self._pos = (t0, a0, c0)
        return result.success


class GuppiWriter(Module):
    """Modules::Guppi::Writer<CF16|CF32> (include/blade/modules/guppi/writer.hh:16-97,
    src/modules/guppi/writer.cc:9-65): one block per process() with the input's
    [aspects, channels, time, pols] host buffer as the data, to <filepath>.0000.raw.
    Header: the data shape (OBSNCHAN, NANTS, NPOL, NBITS, BLOCSIZE, DIRECTIO),
    NBEAM = aspects, DATATYPE = 'FLOAT', PKTIDX = time samples x blocks written,
    and whatever header_put() added.  input_frequency_batches > 1 writes the block
    as that many consecutive channel batches, each [aspects, channels / batches,
    time, pols]."""

    taint = Taint.CONSUMER

    @dataclass
    class config:
        filepath: str
        directio: bool = True
        input_frequency_batches: int = 1
        block_size: int = 512

    @dataclass
    class input:
        buffer: object

    def __init__(self, config, input, stream=None, it="cf32", ot=None):
        super().__init__()
        buf = as_vector(input.buffer)
        if it not in ("cf16", "cf32") or buf.dtype != it:
            _fail("The GUPPI writer takes CF16 or CF32 host buffers.")
        if buf.device != "cpu":
            _fail("The GUPPI writer takes a host buffer (device=bl.cpu).")
        A, F, T, P = buf.shape
        nb = int(config.input_frequency_batches) or 1
        if F % nb:
            _fail(f"Frequency batches ({nb}) must divide the channels ({F}).")
        self.config, self._input, self._it = config, input, it
        self._count = 0
        self._path = f"{config.filepath}.{0:04d}.raw"
        try:
            open(self._path, "wb").close()
        except OSError as e:
            _fail(f"Could not open '{self._path}': {e}")
        bits = 16 if it == "cf16" else 32
        self._hdr: Dict[str, object] = {
            "BLOCSIZE": A * F * T * P * 2 * bits // 8, "OBSNCHAN": A * F, "NANTS": A,
            "NPOL": 4 if P == 2 else P, "NBITS": bits, "DIRECTIO": 1 if config.directio else 0,
            "NBEAM": A, "DATATYPE": "FLOAT", "PKTIDX": 0,
        }

    def header_put(self, key: str, value) -> None:
        self._hdr[key.upper()] = value

    def get_config(self):
        return self.config

    def get_input(self):
        return self._input.buffer

    def _header_bytes(self) -> bytes:
        body = b"".join(_card(k, v) for k, v in self._hdr.items()) + b"END".ljust(_CARD)
        return body.ljust(_pad(len(body)), b" ") if self.config.directio else body

    def process(self, step=0, stream=None):
        buf = as_vector(self._input.buffer)
        A, F, T, P = buf.shape
        data = buf.as_numpy()
        nb = int(self.config.input_frequency_batches) or 1
        if nb > 1:  # consecutive channel batches, each [A, F / nb, T, P]
            data = np.concatenate([np.ascontiguousarray(x) for x in np.split(data, nb, axis=1)], axis=None)
        raw = np.ascontiguousarray(data).view(np.uint8).reshape(-1).tobytes()
        if self.config.directio:
            raw = raw.ljust(_pad(len(raw)), b"\0")
        try:
            with open(self._path, "ab") as fh:
                fh.write(self._header_bytes())
                fh.write(raw)
        except OSError:
            return result.error
        self._count += 1
        self._hdr["PKTIDX"] = T * self._count
        return result.success


def write_ci8_recording(stem: str, blocks: List[np.ndarray], header: Dict[str, object], directio: bool = True,
                        files: int = 1) -> List[str]:
    """Writes CI8 blocks ([NANTS, chans, NTIME, NPOL, 2] int8 each) as a GUPPI RAW
    recording spread over `files` numbered files; header gives the extra records
    (CHAN_BW, OBSFREQ, SCHAN, SYNCTIME, PIPERBLK, DUT1, ...).  PKTIDX advances by
    PIPERBLK per block."""
    paths = []
    per_file = (len(blocks) + files - 1) // files
    for fi in range(files):
        path = f"{stem}.{fi:04d}.raw"
        paths.append(path)
        with open(path, "wb") as fh:
            for bi in range(fi * per_file, min(len(blocks), (fi + 1) * per_file)):
                x = np.ascontiguousarray(blocks[bi], dtype=np.int8)
                A, C, T, P, _ = x.shape
                hdr = {"BLOCSIZE": x.nbytes, "OBSNCHAN": A * C, "NANTS": A, "NPOL": 4 if P == 2 else P, "NBITS": 8,
                       "DIRECTIO": 1 if directio else 0}
                hdr.update(header)
                hdr["PKTIDX"] = int(header.get("PKTIDX", 0)) + bi * int(header.get("PIPERBLK", T))
                body = b"".join(_card(k, v) for k, v in hdr.items()) + b"END".ljust(_CARD)
                fh.write(body.ljust(_pad(len(body)), b" ") if directio else body)
                data = x.tobytes()
                fh.write(data.ljust(_pad(len(data)), b"\0") if directio else data)
    return paths


REGISTRY[("guppi_reader", "generic")] = (GuppiReader, {("ci8", "ci8")})
REGISTRY[("guppi_writer", "generic")] = (GuppiWriter, {("cf16", "cf16"), ("cf32", "cf32")})
