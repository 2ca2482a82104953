"""GPU parity of every module kernel against the FP64 oracle, through the C ABI.

Bit-exact for Cast, Gather, Permutation, Duplicate and Polarizer (CF16 half
arithmetic); relative L2 <= 1e-5 for the FP32 arithmetic (beamformer,
channelizer, detector, phasors)."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from oracle import formulas as O
from blade_b200 import _lib, synthetic as S
from tests.gpu_util import c64, call, crand, dev, host, ptr, rel_l2, stream

pytestmark = pytest.mark.gpu
TOL = 1e-5  # relative L2 for FP32 arithmetic


# ----------------------------------------------------------------------------- cast
CASTS = [
    (_lib.CI8, _lib.CF32, np.int8, np.float32, True),
    (_lib.CI8, _lib.CF16, np.int8, np.float16, True),
    (_lib.I8, _lib.F32, np.int8, np.float32, False),
    (_lib.F16, _lib.F32, np.float16, np.float32, False),
    (_lib.F32, _lib.F16, np.float32, np.float16, False),
    (_lib.F32, _lib.I32, np.float32, np.int32, False),
    (_lib.CF32, _lib.CF16, np.float32, np.float16, True),
    (_lib.CF16, _lib.CF32, np.float16, np.float32, True),
]


@pytest.mark.parametrize("it,ot,nt,no,cplx", CASTS)
@pytest.mark.parametrize("n", [0, 1, 7, 4096, 100003])
def test_cast_bit_exact(cuda, it, ot, nt, no, cplx, n):
    rng = np.random.default_rng(n + it * 10 + ot)
    ns = n * (2 if cplx else 1)
    if np.issubdtype(nt, np.integer):
        x = rng.integers(-128, 128, size=ns).astype(nt)
    else:
        x = (rng.standard_normal(ns) * 1000).astype(nt)
    xd = dev(x) if ns else torch.empty(0, dtype=torch.int8, device="cuda")
    yd = torch.zeros(max(ns, 1), dtype=getattr(torch, np.dtype(no).name), device="cuda")
    call("blade_cast", it, ot, ptr(xd), ptr(yd), n, stream())
    y = host(yd)[:ns]
    np.testing.assert_array_equal(y, O.cast_scalars(x, no))


def test_cast_unaligned_tail(cuda):
    x = np.arange(-64, 64, dtype=np.int8)
    xd = dev(x)
    yd = torch.zeros(128, dtype=torch.float32, device="cuda")
    call("blade_cast", _lib.I8, _lib.F32, xd.data_ptr() + 3, yd.data_ptr() + 12, 101, stream())
    np.testing.assert_array_equal(host(yd)[3:104], x[3:104].astype(np.float32))


# ------------------------------------------------------------------------ beamformer
BF_CASES = [
    # (A, F, T, P, B, incoherent, sqrt)
    (20, 96, 256, 2, 8, False, False),     # ATA small workload
    (2, 192, 512, 2, 1, True, True),       # tests/modules/beamformer/ata.py shapes
    (28, 12, 1024, 2, 16, True, False),
    (64, 4, 512, 2, 64, False, False),     # A = B = 64 (the reference kernel cannot build this)
    (3, 5, 77, 1, 5, True, True),          # ragged, single polarisation
    (1, 1, 1, 2, 1, False, False),         # minimal
    (5, 3, 130, 2, 37, False, False),      # beams spanning two beam tiles
]


@pytest.mark.parametrize("A,F,T,P,B,inc,sq", BF_CASES)
def test_beamformer_f32(cuda, A, F, T, P, B, inc, sq):
    rng = np.random.default_rng(A * 1000 + B)
    x = crand(rng, (A, F, T, P))
    w = crand(rng, (B, A, F, 1, P))
    xd, wd = c64(x), c64(w)
    yd = torch.zeros((B + int(inc), F, T, P), dtype=torch.complex64, device="cuda")
    call("blade_beamform_f32", ptr(xd), ptr(wd), ptr(yd), B, A, F, T, P, int(inc), int(sq), stream())
    y = host(yd)
    ref = O.beamform(x, w, inc, sq)
    assert rel_l2(y[:B], ref[:B]) < TOL
    if inc:
        assert rel_l2(y[B], ref[B]) < TOL
        assert np.all(y[B].imag == 0)


@pytest.mark.parametrize("A,F,T,P,B,inc", [(16, 4, 512, 2, 8, True), (64, 3, 1024, 2, 64, False),
                                           (3, 5, 77, 1, 5, True), (7, 2, 64, 2, 2, False)])
def test_beamformer_meerkat(cuda, A, F, T, P, B, inc):
    # src/modules/beamformer/beamformer.cu:81-117: weight w[b*A + a] of a [B, A, F, 1, P] tensor
    rng = np.random.default_rng(A * 7 + B)
    x = crand(rng, (A, F, T, P))
    w = crand(rng, (B, A, F, 1, P))
    xd, wd = c64(x), c64(w)
    yd = torch.full((B + int(inc), F, T, P), 7.0, dtype=torch.complex64, device="cuda")
    call("blade_beamform_meerkat_f32", ptr(xd), ptr(wd), ptr(yd), B, A, F, T, P, int(inc), stream())
    y = host(yd)
    ref = O.beamform_meerkat(x, w, B, inc)
    assert rel_l2(y[:B], ref[:B]) < TOL
    if inc:
        assert np.all(y[B] == 0)


def test_beamformer_meerkat_module(cuda):
    A, F, T, P, B = 8, 4, 256, 2, 3
    rng = np.random.default_rng(5)
    x, w = crand(rng, (A, F, T, P)), crand(rng, (B, A, F, 1, P))
    buf = bl.array_tensor((A, F, T, P), dtype=bl.cf32, device=bl.cuda)
    ph = bl.phasor_tensor((B, A, F, 1, P), dtype=bl.cf32, device=bl.cuda)
    buf.as_torch().copy_(c64(x))
    ph.as_torch().copy_(c64(w))
    mod = bl.module(bl.beamformer, {"enable_incoherent_beam": False}, (buf, ph), telescope=bl.meerkat)
    assert isinstance(mod, bl.BeamformerMeerKAT)
    mod.process()
    torch.cuda.synchronize()
    assert rel_l2(mod.get_output().as_torch().cpu().numpy(), O.beamform_meerkat(x, w, B)) < TOL


# ------------------------------------------------------------------------ channelizer
CH_CASES = [
    # (A, F, T, P, rate)  -- first three are the reference's meson cases
    (5, 100, 200, 1, 200),
    (8, 128, 1024, 2, 1024),
    (8, 128, 1024, 1, 1024),
    (8, 16, 1024, 1, 512),      # reference should_fail (rate != T): supported here
    (4, 6, 64, 2, 4),
    (2, 3, 96, 2, 6),
    (2, 5, 4096, 2, 4096),
    (1, 2, 16384, 2, 8192),     # rate 8192, two spectra per row
    (1, 2, 131072, 2, 65536),   # the spectrometer NFFT
    (3, 4, 20, 2, 2),
    # rates 2, 4, 8, 16 run one spectrum per thread in registers: both pol counts
    (3, 5, 96, 1, 4),
    (2, 3, 256, 2, 8),
    (2, 3, 256, 1, 8),
    (2, 3, 512, 2, 16),
    (2, 3, 512, 1, 16),
    (2, 2, 64, 1, 2),
    (2, 3, 24576, 1, 8192),     # rate 8192: one transform per CTA unit, three spectra per row
    (2, 3, 24576, 2, 8192),     # rate 8192, two polarisations, three spectra per row
]


@pytest.mark.parametrize("A,F,T,P,rate", CH_CASES)
def test_channelizer(cuda, A, F, T, P, rate):
    rng = np.random.default_rng(rate + T)
    x = crand(rng, (A, F, T, P))
    xd = c64(x)
    yd = torch.zeros((A, F * rate, T // rate, P), dtype=torch.complex64, device="cuda")
    wsb = _lib.load().blade_channelize_workspace_size(A, F, T, P, rate)
    ws = torch.empty(max(int(wsb), 1), dtype=torch.uint8, device="cuda")
    call("blade_channelize", ptr(xd), ptr(yd), ptr(ws) if wsb else None, A, F, T, P, rate, stream())
    assert rel_l2(host(yd), O.channelize(x, rate)) < TOL


@pytest.mark.parametrize("A,F,T,P", [(3, 7, 256, 2), (3, 5, 8192, 2), (2, 3, 8192, 1), (2, 2, 4, 2)])
def test_channelizer_in_place_rate_equals_T(cuda, A, F, T, P):
    # rate == T in place, as the reference module runs it (its benchmark: rate 8192)
    rng = np.random.default_rng(77 + T + P)
    x = crand(rng, (A, F, T, P))
    xd = c64(x)
    call("blade_channelize", ptr(xd), ptr(xd), None, A, F, T, P, T, stream())
    assert rel_l2(host(xd).reshape(A, F * T, 1, P), O.channelize(x, T)) < TOL


@pytest.mark.parametrize("A,F,nspec", [(2, 3, 3), (4, 40, 1)])
def test_rate8192_two_polarisations_match_one(cuda, A, F, nspec):
    # At rate 8192 each CTA unit is one polarisation of one spectrum: the unit of a
    # two-polarisation input computes exactly what the one-polarisation input of that
    # polarisation does (bit for bit).  160 x 2 units (the second case) make each CTA
    # loop, prefetching its next unit's spectrum into L2.
    T = 8192 * nspec
    rng = np.random.default_rng(8192 + A * F * nspec)
    x = crand(rng, (A, F, T, 2))
    y = torch.zeros((A, F * 8192, nspec, 2), dtype=torch.complex64, device="cuda")
    call("blade_channelize", ptr(c64(x)), ptr(y), None, A, F, T, 2, 8192, stream())
    for p in range(2):
        xp = c64(np.ascontiguousarray(x[..., p:p + 1]))
        yp = torch.zeros((A, F * 8192, nspec, 1), dtype=torch.complex64, device="cuda")
        call("blade_channelize", ptr(xp), ptr(yp), None, A, F, T, 1, 8192, stream())
        assert torch.equal(y[..., p:p + 1], yp)
    assert rel_l2(host(y), O.channelize(x, 8192)) < TOL


# ------------------------------------------------------------------------ polarizer
def test_polarizer_cf32(cuda):
    rng = np.random.default_rng(5)
    x = crand(rng, (2, 19, 875, 2))
    xd = c64(x)
    call("blade_polarize", _lib.CF32, ptr(xd), ptr(xd), 2 * 19 * 875, stream())
    y = host(xd)
    np.testing.assert_array_equal(y[..., 0], (x[..., 0] + 1j * x[..., 1]).astype(np.complex64))
    np.testing.assert_array_equal(y[..., 1], (x[..., 0] - 1j * x[..., 1]).astype(np.complex64))


@pytest.mark.parametrize("n", [1, 2, 1001])
def test_polarizer_cf16_bit_exact(cuda, n):
    rng = np.random.default_rng(n)
    x = (rng.standard_normal((n, 2, 2)) * 100).astype(np.float16)  # [sample][pol][re, im]
    xd = dev(x)
    call("blade_polarize", _lib.CF16, ptr(xd), ptr(xd), n, stream())
    y = host(xd)
    xr, xi, yr, yi = x[:, 0, 0], x[:, 0, 1], x[:, 1, 0], x[:, 1, 1]
    np.testing.assert_array_equal(y[:, 0, 0], xr - yi)
    np.testing.assert_array_equal(y[:, 0, 1], xi + yr)
    np.testing.assert_array_equal(y[:, 1, 0], xr + yi)
    np.testing.assert_array_equal(y[:, 1, 1], xi - yr)


# ------------------------------------------------------------------------ detector
@pytest.mark.parametrize("npol", [1, 4])
@pytest.mark.parametrize("A,F,T,I", [(2, 192, 8750, 10), (2, 8, 512, 1), (3, 4, 4096, 64), (1, 2, 8192, 2048),
                                     (2, 3, 24, 24)])
def test_detector(cuda, npol, A, F, T, I):
    rng = np.random.default_rng(T + I)
    x = crand(rng, (A, F, T, 2))
    xd = c64(x)
    yd = torch.zeros((A, F, T // I, npol), dtype=torch.float32, device="cuda")
    call("blade_detect", ptr(xd), ptr(yd), A, F, T, 2, I, npol, stream())
    y = host(yd)
    assert rel_l2(y, O.detect(x, I, npol)) < TOL
    # deterministic: identical bits on a second run
    y2d = torch.zeros_like(yd)
    call("blade_detect", ptr(xd), ptr(y2d), A, F, T, 2, I, npol, stream())
    np.testing.assert_array_equal(host(y2d), y)


# ------------------------------------------------------------------------ gather
GATHER_CASES = [(2, 192, 512, 2, 2, 16), (27, 1024, 3, 2, 2, 16), (3, 7, 3, 1, 0, 5), (1, 2, 5, 6, 1, 6),
                (11, 1, 13, 9, 2, 7), (9, 2, 1, 3, 3, 8), (9, 2, 5555, 3, 2, 8)]


@pytest.mark.parametrize("A,F,T,P,axis,m", GATHER_CASES)
@pytest.mark.parametrize("dtype", ["cf32", "ci8"])
def test_gather_bit_exact(cuda, A, F, T, P, axis, m, dtype):
    rng = np.random.default_rng(A + F + T)
    if dtype == "cf32":
        blocks = [crand(rng, (A, F, T, P)) for _ in range(m)]
        es = 8
    else:
        blocks = [rng.integers(-128, 128, size=(A, F, T, P, 2)).astype(np.int8) for _ in range(m)]
        es = 2
    out_shape = list(blocks[0].shape)
    out_shape[axis] *= m
    od = torch.zeros(out_shape, dtype=torch.complex64 if dtype == "cf32" else torch.int8, device="cuda")
    shape = _lib.u64_array([A, F, T, P])
    for step, b in enumerate(blocks):
        bd = dev(b)
        call("blade_gather", es, ptr(bd), ptr(od), shape, axis, m, step, stream())
        torch.cuda.synchronize()
    np.testing.assert_array_equal(host(od), O.gather(blocks, axis))


# ------------------------------------------------------------------------ permutation
import itertools  # noqa: E402

PERMS = list(itertools.permutations(range(4)))


@pytest.mark.parametrize("perm", PERMS)
def test_permutation_all_orders_bit_exact(cuda, perm):
    rng = np.random.default_rng(sum(p * 10 ** i for i, p in enumerate(perm)))
    x = crand(rng, (3, 5, 37, 2))
    xd = c64(x)
    out = O.permute(x, perm)
    yd = torch.zeros(out.shape, dtype=torch.complex64, device="cuda")
    call("blade_permute", 8, ptr(xd), ptr(yd), _lib.u64_array(x.shape), _lib.u64_array(perm), stream())
    np.testing.assert_array_equal(host(yd), out)


@pytest.mark.parametrize("perm", [(0, 1, 2, 3), (0, 2, 1, 3), (3, 2, 1, 0), (2, 0, 3, 1)])
@pytest.mark.parametrize("es", [2, 4, 8])
def test_permutation_reference_cases(cuda, perm, es):
    # tests/modules/permutation/meson.build:3-37 on (2, 192, 1024, 2) (T shrunk from 8192).
    rng = np.random.default_rng(es)
    shape = (2, 192, 1024, 2)
    raw = rng.integers(0, 256, size=shape + (es,)).astype(np.uint8)
    xd = dev(raw)
    out = np.ascontiguousarray(np.transpose(raw, tuple(perm) + (4,)))
    yd = torch.zeros(out.shape, dtype=torch.uint8, device="cuda")
    call("blade_permute", es, ptr(xd), ptr(yd), _lib.u64_array(shape), _lib.u64_array(perm), stream())
    np.testing.assert_array_equal(host(yd), out)


# ------------------------------------------------------------------------ duplicate
@pytest.mark.parametrize("nbytes", [1, 15, 16, 1 << 20, (1 << 20) + 3])
def test_duplicate_bit_exact(cuda, nbytes):
    rng = np.random.default_rng(nbytes)
    x = rng.integers(0, 256, size=nbytes).astype(np.uint8)
    xd = dev(x)
    yd = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    call("blade_duplicate", ptr(xd), ptr(yd), nbytes, stream())
    np.testing.assert_array_equal(host(yd), x)


# ------------------------------------------------------------------------ phasors
def test_phasors_from_delays(cuda):
    rng = np.random.default_rng(13)
    B, A, F, P = 4, 20, 192, 2
    tau = rng.uniform(-5e-6, 5e-6, size=(B, A))
    cal = crand(rng, (A, F, 1, P), np.complex128)
    rf, bw, tot, start = 6500.125e6, 0.5e6, 1.024e9, 352
    ref = O.phasors_from_delays(tau, cal, rf, bw, tot, start)
    td, cd = dev(tau), dev(cal)
    od = torch.zeros((B, A, F, 1, P), dtype=torch.complex64, device="cuda")
    call("blade_phasor_from_delays", ptr(td), ptr(cd), ptr(od), B, A, F, P, rf, bw, tot, start, stream())
    assert rel_l2(host(od), ref) < 1e-6
    # unit calibration, the synthetic-workload frequency plan (f = 6 GHz + 0.5 MHz k)
    od2 = torch.zeros_like(od)
    call("blade_phasor_from_delays", ptr(td), None, ptr(od2), B, A, F, P, S.F0_HZ, S.DF_HZ, 0.0, 0, stream())
    got = host(od2)
    f = S.F0_HZ + S.DF_HZ * np.arange(F)
    exp = np.exp(-2j * np.pi * tau[:, :, None] * f[None, None, :])
    assert rel_l2(got[:, :, :, 0, 0], exp) < 1e-6
