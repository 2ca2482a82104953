"""FP64 numpy restatement of the reference's hot-path arithmetic.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Parity pinning: the reference ships no golden vectors (its tests draw unseeded
``np.random.random`` data).  This oracle is pinned two ways:

* against the reference's own CUDA kernels, built from the reference sources by
  ``oracle/ref_kernels/build.sh`` and run on the GPU; their outputs on seeded
  inputs are committed under ``tests/golden/`` (``tests/golden/make_golden.py``);
* against ``oracle/loops.py``, which restates the kernels' loop order literally.

Conventions.  Complex int8 (CI8) data is carried as an ``int8`` array with a
trailing axis of length 2 (re, im), which is the reference's in-memory layout of
``CI8`` (``include/blade/memory/types.hh``).  All other complex data is
``complex128`` here.  Shapes follow the reference: ArrayShape [A, F, T, P]
(``include/blade/memory/custom.hh:10-53``), PhasorShape [B, A, F, 1, P]
(``custom.hh:55-103``), DelayShape [B, A] (``custom.hh:105-138``).
"""

from __future__ import annotations

import numpy as np


# --------------------------------------------------------------------------- #
# Cast
# --------------------------------------------------------------------------- #

def ci8_to_complex(x: np.ndarray) -> np.ndarray:
    """[..., 2] int8 -> complex128 (exact)."""
    x = np.asarray(x)
    return x[..., 0].astype(np.float64) + 1j * x[..., 1].astype(np.float64)


def cast_scalars(x: np.ndarray, out_dtype) -> np.ndarray:
    """Per-scalar ``static_cast`` of a real array.

    Follows ``src/modules/cast/cast.cu:5-12`` (``output[tid] =
    static_cast<OT>(input[tid])`` over the scalar subtype, N = size x 2 for
    complex types, ``src/modules/cast/base.cc:27-36``).  float -> integer
    truncates toward zero (C conversion); float -> half rounds to nearest even.
    The reference test oracle is ``tests/modules/cast/cast.py:44``
    (``astype(float32)``).
    """
    x = np.asarray(x)
    out_dtype = np.dtype(out_dtype)
    if np.issubdtype(out_dtype, np.integer) and np.issubdtype(x.dtype, np.floating):
        return np.trunc(x).astype(out_dtype)
    return x.astype(out_dtype)


# --------------------------------------------------------------------------- #
# Phasor (delay -> phasor half of Phasor::ATA)
# --------------------------------------------------------------------------- #

def phasors_from_delays(delays: np.ndarray, calibrations: np.ndarray,
                        observation_frequency_hz: float, channel_bandwidth_hz: float,
                        total_bandwidth_hz: float, frequency_start_index: int) -> np.ndarray:
    """Phasors [B, A, F, 1, P] from delays [B, A] (seconds) and calibrations [A, F, 1, P].

    Follows ``src/modules/phasor/ata.cc:176-208``::

        fringe  = observationFrequencyHz - totalBandwidthHz / 2
        freq_f  = (f + frequencyStartIndex) * channelBandwidthHz
        phasor  = exp(-i 2 pi tau freq_f) * exp(-i 2 pi tau fringe) * cal[a, f, p]

    and the test oracle ``tests/bundles/ata/mode_b.py:302-313``.
    """
    delays = np.asarray(delays, dtype=np.float64)
    cal = np.asarray(calibrations, dtype=np.complex128)
    B, A = delays.shape
    Ac, F, _, P = cal.shape
    assert Ac == A
    fringe = observation_frequency_hz - total_bandwidth_hz / 2.0
    freqs = (np.arange(F, dtype=np.float64) + frequency_start_index) * channel_bandwidth_hz
    tau = delays[:, :, None]                                   # [B, A, 1]
    phase = -2.0 * np.pi * tau * freqs[None, None, :] + (-2.0 * np.pi * tau * fringe)
    ph = np.exp(1j * phase)                                    # [B, A, F]
    return ph[:, :, :, None, None] * cal[None, :, :, :, :]     # [B, A, F, 1, P]


# --------------------------------------------------------------------------- #
# Beamformer (ATA)
# --------------------------------------------------------------------------- #

def beamform(x: np.ndarray, phasors: np.ndarray, incoherent: bool = False,
             incoherent_sqrt: bool = False) -> np.ndarray:
    """y[b, f, t, p] = sum_a x[a, f, t, p] * w[b, a, f, 0, p]  (no conjugate).

    Follows ``src/modules/beamformer/beamformer.cu:53-62`` and the test oracle
    ``tests/modules/beamformer/ata.py:58-60``.  With ``incoherent`` an extra beam
    at index B holds ``sum_a |x * w[0]|^2`` (optionally square-rooted) in the real
    part and 0 in the imaginary part, as ``beamformer.cu:64-78`` computes it
    (beam 0's phasor; the test at ``ata.py:61-63`` coincides when B = 1).
    Output shape [B(+1), F, T, P] (``include/blade/modules/beamformer/ata.hh:16-24``).
    """
    x = np.asarray(x, dtype=np.complex128)
    w = np.asarray(phasors, dtype=np.complex128)
    A, F, T, P = x.shape
    B = w.shape[0]
    assert w.shape == (B, A, F, 1, P)
    xf = np.transpose(x, (1, 3, 0, 2))                 # [F, P, A, T]
    wf = np.transpose(w[:, :, :, 0, :], (2, 3, 0, 1))  # [F, P, B, A]
    yf = wf @ xf                                       # [F, P, B, T]
    y = np.transpose(yf, (2, 0, 3, 1))                 # [B, F, T, P]
    if not incoherent:
        return y
    ph = x * w[0, :, :, :, :]                          # [A, F, T, P] (broadcast over T)
    inc = (ph.real * ph.real + ph.imag * ph.imag).sum(axis=0)
    if incoherent_sqrt:
        inc = np.sqrt(inc)
    return np.concatenate([y, inc[None].astype(np.complex128)], axis=0)


def beamform_meerkat(x: np.ndarray, phasors: np.ndarray, beams: int, incoherent: bool = False) -> np.ndarray:
    """MeerKAT beamformer: y[b, f, t, p] = sum_a x[a, f, t, p] * w[b*A + a].

    Follows ``src/modules/beamformer/beamformer.cu:81-117``: the kernel reads the
    phasor buffer as a flat [B, A] array (index ``iy`` runs over beams then
    antennas), one weight per (beam, antenna) for every channel and polarisation,
    i.e. the first B*A values of the [B, A, F, 1, P] phasor tensor it is given.
    The output has B(+1) beams (``include/blade/modules/beamformer/meerkat.hh:17-24``);
    the kernel never writes the incoherent beam, which is returned as zeros here.
    """
    x = np.asarray(x, dtype=np.complex128)
    A, F, T, P = x.shape
    B = int(beams)
    w = np.asarray(phasors, dtype=np.complex128).reshape(-1)[: B * A].reshape(B, A)
    y = np.einsum("ba,aftp->bftp", w, x)
    if incoherent:
        y = np.concatenate([y, np.zeros((1, F, T, P), dtype=np.complex128)], axis=0)
    return y


# --------------------------------------------------------------------------- #
# Channelizer
# --------------------------------------------------------------------------- #

def channelize(x: np.ndarray, rate: int) -> np.ndarray:
    """[A, F, T, P] -> [A, F*C, T/C, P], C = rate.

    out[a, f*C + k, s, p] = fftshift(FFT_C(x[a, f, s*C:(s+1)*C, p]))[k], no
    normalisation.  Follows the reference test oracle
    ``tests/modules/channelizer/advanced.py:49-65`` (general rate) and the module
    ``src/modules/channelizer/base.cc:59-138`` + ``channelizer.cu:5-19``, where the
    (-1)^t pre-multiply realises the fftshift for even C.  rate == 1 is the
    identity (``base.cc:124-126``).
    """
    x = np.asarray(x, dtype=np.complex128)
    A, F, T, P = x.shape
    C = int(rate)
    if C == 1:
        return x.copy()
    assert T % C == 0
    S = T // C
    blocks = x.reshape(A, F, S, C, P)
    spec = np.fft.fftshift(np.fft.fft(blocks, axis=3), axes=3)   # [A, F, S, C, P]
    return np.transpose(spec, (0, 1, 3, 2, 4)).reshape(A, F * C, S, P)


# --------------------------------------------------------------------------- #
# Polarizer
# --------------------------------------------------------------------------- #

def polarize(x: np.ndarray) -> np.ndarray:
    """(X, Y) -> (X + iY, X - iY) along the last (polarisation) axis, no 1/sqrt(2).

    Follows ``src/modules/polarizer/polarizer.cu:17-23`` and the test oracle
    ``tests/modules/polarizer/polarizer.py:47-49``.
    """
    x = np.asarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    out[..., 0] = x[..., 0] + 1j * x[..., 1]
    out[..., 1] = x[..., 0] - 1j * x[..., 1]
    return out


# --------------------------------------------------------------------------- #
# Detector
# --------------------------------------------------------------------------- #

def detect(x: np.ndarray, integration: int, npols: int) -> np.ndarray:
    """[A, F, T, 2] complex -> [A, F, T/I, npols] real.

    npols = 4: (sum |X|^2, sum |Y|^2, sum Re X conj(Y), sum Im X conj(Y)) per
    window of I consecutive samples (``src/modules/detector/detector.cu:7-32``,
    test ``tests/modules/detector/cross_pol.py:58-71``).
    npols = 1: Stokes-I, sum |X|^2 + |Y|^2 (``detector.cu:34-51``, test
    ``tests/modules/detector/single_pol.py:56-67``).
    """
    x = np.asarray(x, dtype=np.complex128)
    A, F, T, P = x.shape
    assert P == 2 and T % integration == 0
    X = x[..., 0].reshape(A, F, T // integration, integration)
    Y = x[..., 1].reshape(A, F, T // integration, integration)
    if npols == 1:
        s = (X.real ** 2 + X.imag ** 2 + Y.real ** 2 + Y.imag ** 2).sum(axis=-1)
        return s[..., None]
    if npols == 4:
        xx = (X.real ** 2 + X.imag ** 2).sum(axis=-1)
        yy = (Y.real ** 2 + Y.imag ** 2).sum(axis=-1)
        c = (X * np.conj(Y)).sum(axis=-1)
        return np.stack([xx, yy, c.real, c.imag], axis=-1)
    raise ValueError("number_of_output_polarizations must be 1 or 4")


# --------------------------------------------------------------------------- #
# Gather / Permutation / Duplicate (bit-exact byte movement)
# --------------------------------------------------------------------------- #

def gather(inputs, axis: int) -> np.ndarray:
    """Concatenate successive blocks along ``axis``.

    Follows ``src/modules/gather/base.cc:71-109`` (block ``step`` lands at offset
    ``step * shape[axis]``) and the test oracle ``tests/modules/gather/gather.py:54-55``.
    """
    return np.concatenate(list(inputs), axis=axis)


def permute(x: np.ndarray, indexes) -> np.ndarray:
    """out.shape[i] = in.shape[indexes[i]] (``include/blade/modules/permutation.hh:71-77``),
    out[coords permuted] = in[coords] (``src/modules/permutation/permutation.cu:12-18``);
    test oracle ``tests/modules/permutation/permutation.py:49`` (``np.transpose``)."""
    return np.ascontiguousarray(np.transpose(x, tuple(indexes)))


def duplicate(x: np.ndarray) -> np.ndarray:
    """Device-to-device copy (``src/modules/duplicate/base.cc:35-37``)."""
    return np.array(x, copy=True)


# --------------------------------------------------------------------------- #
# Chains (bundles and the benchmark workloads)
# --------------------------------------------------------------------------- #

def beamform_channelize_detect(x_ci8: np.ndarray, phasors: np.ndarray, rate: int,
                               integration: int, npols: int = 1) -> np.ndarray:
    """Cast(CI8->CF32) -> Beamformer::ATA -> Channelizer(rate) -> Detector.

    The chain of ``include/blade/bundles/ata/mode_b.hh:99-199`` without the
    pre-beamformer stages, and the Stokes-I reduction of the test oracle
    ``tests/bundles/ata/mode_b.py:377-390``.
    """
    x = ci8_to_complex(x_ci8)
    y = beamform(x, phasors)
    y = channelize(y, rate)
    return detect(y, integration, npols)


def spectrometer(x_ci8: np.ndarray, rate: int, integration: int, polarizer: bool = True,
                 npols: int = 1) -> np.ndarray:
    """Cast(CI8->CF32) -> Channelizer(rate) -> Polarizer -> Detector.

    The ModeH chain of ``include/blade/bundles/generic/mode_h.hh:55-106`` and the
    test oracle ``tests/bundles/generic/mode_h.py:56-74``.
    """
    x = ci8_to_complex(x_ci8)
    y = channelize(x, rate)
    if polarizer:
        y = polarize(y)
    return detect(y, integration, npols)


def mode_b(x: np.ndarray, phasors: np.ndarray, rate: int, circular: bool = False, incoherent: bool = False,
           detector: bool = True, integration: int = 1, npols: int = 1) -> np.ndarray:
    """Cast -> Channelizer(rate) -> Polarizer -> Beamformer::ATA -> [Detector].

    The ATA ModeB chain of ``include/blade/bundles/ata/mode_b.hh:99-199`` (the
    phasors are per channelized channel, [B, A, F*rate, 1, P]; the incoherent beam
    is square-rooted when the detector is enabled, ``mode_b.hh:146-147``) and the
    Stokes-I reduction of its test oracle ``tests/bundles/ata/mode_b.py:377-390``.
    ``x`` is CI8 ([..., 2] int8) or complex.
    """
    x = ci8_to_complex(x) if np.asarray(x).dtype == np.int8 else np.asarray(x, dtype=np.complex128)
    y = channelize(x, rate)
    if circular:
        y = polarize(y)
    z = beamform(y, phasors, incoherent=incoherent, incoherent_sqrt=detector)
    if not detector:
        return z
    return detect(z, integration, npols)


# --------------------------------------------------------------------------- #
# Adjoint of beamform + Stokes-I detect (no reference counterpart)
# --------------------------------------------------------------------------- #

def stokes_loss(x: np.ndarray, w: np.ndarray) -> float:
    """L = -sum S, S = Stokes-I of beamform(x, w); integration windows do not change the sum."""
    y = beamform(x, w)
    return -float(np.sum(y.real ** 2 + y.imag ** 2))


def stokes_loss_grad(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    """dL/d conj(w) for L = -sum_{b,f,t,p} |y[b,f,t,p]|^2, y = beamform(x, w).

    With y = sum_a x w, d|y|^2 / d conj(w_a) = y conj(x_a), so
    G[b, a, f, 0, p] = -sum_t y[b, f, t, p] conj(x[a, f, t, p]).
    The gradient with respect to the real parameters (Re w, Im w) is
    (2 Re G, 2 Im G).  Integration windows do not change the sum.
    """
    x = np.asarray(x, dtype=np.complex128)
    w = np.asarray(w, dtype=np.complex128)
    y = beamform(x, w)                                        # [B, F, T, P]
    g = -np.einsum("bftp,aftp->bafp", y, np.conj(x))
    return g[:, :, :, None, :]


def relative_l2(a: np.ndarray, ref: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) else np.float64)
    ref = np.asarray(ref, dtype=a.dtype)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((a - ref).ravel()) / (den if den > 0 else 1.0))


# --------------------------------------------------------------------------- #
# Geometric delays (the astrometric half of Modules::Phasor::ATA)
# --------------------------------------------------------------------------- #
# The reference computes these with ERFA (src/modules/phasor/ata.cc:88-167) and
# pins them only against astropy at rtol 0.5 (tests/modules/phasor/advanced.py:
# 106-143, 183-195: w = baseline . source direction in ITRS, delay = (w_beam -
# w_boresight) / c).  Neither ERFA nor astropy is available, so this restates the
# published low-precision formulas the library uses (Meeus, Astronomical
# Algorithms, 2nd ed.: eq. 12.4 sidereal time, ch. 21 IAU 1976 precession, ch. 22
# leading IAU 1980 nutation terms, ch. 23 annual aberration); the tests pin each
# part against Meeus' worked examples.  Parity with ERFA stays unpinned.

_AS = np.pi / (180.0 * 3600.0)
_DEG = np.pi / 180.0
C_LIGHT = 299792458.0


def _r1(t):
    c, s = np.cos(t), np.sin(t)
    return np.array([[1, 0, 0], [0, c, s], [0, -s, c]])


def _r2(t):
    c, s = np.cos(t), np.sin(t)
    return np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]])


def _r3(t):
    c, s = np.cos(t), np.sin(t)
    return np.array([[c, s, 0], [-s, c, 0], [0, 0, 1]])


def gmst_deg(jd_ut1: float) -> float:
    """Greenwich mean sidereal time in degrees (Meeus eq. 12.4, IAU 1982)."""
    du = jd_ut1 - 2451545.0
    tu = du / 36525.0
    return (280.46061837 + 360.98564736629 * du + 0.000387933 * tu * tu - tu ** 3 / 38710000.0) % 360.0


def nutation(t: float):
    """(dpsi, deps, eps0) in radians for Julian centuries t of TT from J2000.0:
    the four leading IAU 1980 terms (Meeus ch. 22, 0.5" / 0.1")."""
    om = (125.04452 - 1934.136261 * t) * _DEG
    ls = (280.4665 + 36000.7698 * t) * _DEG
    lm = (218.3165 + 481267.8813 * t) * _DEG
    dpsi = (-17.20 * np.sin(om) - 1.32 * np.sin(2 * ls) - 0.23 * np.sin(2 * lm) + 0.21 * np.sin(2 * om)) * _AS
    deps = (9.20 * np.cos(om) + 0.57 * np.cos(2 * ls) + 0.10 * np.cos(2 * lm) - 0.09 * np.cos(2 * om)) * _AS
    eps0 = (84381.448 - 46.8150 * t - 0.00059 * t * t + 0.001813 * t ** 3) * _AS
    return dpsi, deps, eps0


def precession_matrix(t: float) -> np.ndarray:
    """IAU 1976 precession from J2000.0 to t Julian centuries (Meeus eq. 21.3)."""
    zeta = (2306.2181 * t + 0.30188 * t * t + 0.017998 * t ** 3) * _AS
    z = (2306.2181 * t + 1.09468 * t * t + 0.018203 * t ** 3) * _AS
    theta = (2004.3109 * t - 0.42665 * t * t - 0.041833 * t ** 3) * _AS
    return _r3(-z) @ _r2(theta) @ _r3(-zeta)


def source_itrs(ra: float, dec: float, jd_utc: float, dut1: float) -> np.ndarray:
    """Unit vector of ICRS (ra, dec) in the terrestrial frame (polar motion
    neglected): R3(GAST) N P applied to the annually aberrated direction."""
    t = (jd_utc + 69.184 / 86400.0 - 2451545.0) / 36525.0
    dpsi, deps, eps0 = nutation(t)
    eps = eps0 + deps
    l0 = (280.46646 + 36000.76983 * t + 0.0003032 * t * t) * _DEG
    ma = (357.52911 + 35999.05029 * t - 0.0001537 * t * t) * _DEG
    cen = ((1.914602 - 0.004817 * t - 0.000014 * t * t) * np.sin(ma) + (0.019993 - 0.000101 * t) * np.sin(2 * ma)
           + 0.000289 * np.sin(3 * ma)) * _DEG
    lsun = l0 + cen
    kappa = 20.49552 * _AS
    p = np.array([np.cos(dec) * np.cos(ra), np.cos(dec) * np.sin(ra), np.sin(dec)])
    p = p + kappa * np.array([np.sin(lsun), -np.cos(lsun) * np.cos(eps), -np.cos(lsun) * np.sin(eps)])
    p = p / np.linalg.norm(p)
    gast = gmst_deg(jd_utc + dut1 / 86400.0) * _DEG + dpsi * np.cos(eps)
    n = _r1(-eps) @ _r3(-dpsi) @ _r1(eps0)
    return _r3(gast) @ n @ precession_matrix(t) @ p


def geometric_delays(positions, reference: int, boresight, beams, jd_utc: float, dut1: float) -> np.ndarray:
    """delays[b, a] = ((r_a - r_ref) . (s_b - s_boresight)) / c (ata.cc:39-47)."""
    r = np.asarray(positions, dtype=np.float64)
    bl = r - r[reference]
    s0 = source_itrs(boresight[0], boresight[1], jd_utc, dut1)
    out = np.empty((len(beams), len(r)))
    for b, (ra, dec) in enumerate(beams):
        out[b] = bl @ (source_itrs(ra, dec, jd_utc, dut1) - s0) / C_LIGHT
    return out


def delays_via_hour_angle(positions, reference: int, lon: float, boresight, beams, jd_utc: float, dut1: float):
    """The same delays by the reference's route (ata.cc:17-47): array-centred XYZ
    (ECEF rotated by the reference longitude), W of the UVW frame of each source's
    apparent hour angle and declination (Thompson, Moran & Swenson eq. 4.1)."""
    r = np.asarray(positions, dtype=np.float64) - np.asarray(positions, dtype=np.float64)[reference]
    xyz = r @ _r3(lon).T  # X toward the local meridian, Y east, Z north

    def w_of(ra, dec):
        s = source_itrs(ra, dec, jd_utc, dut1)
        ha = lon - np.arctan2(s[1], s[0])  # local apparent hour angle
        d = np.arcsin(s[2])
        return np.cos(d) * np.cos(ha) * xyz[:, 0] - np.cos(d) * np.sin(ha) * xyz[:, 1] + np.sin(d) * xyz[:, 2]

    w0 = w_of(*boresight)
    return np.stack([(w_of(ra, dec) - w0) / C_LIGHT for ra, dec in beams])
