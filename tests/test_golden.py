"""Golden fixtures: outputs of the reference's own CUDA kernels (built from the
reference sources, oracle/ref_kernels) on deterministic inputs, committed in
tests/golden/reference_kernels.npz by tests/golden/make_golden.py.

CPU: pins the FP64 oracle to the reference kernels.  GPU: our kernels against
the same fixtures.  Cast, Polarizer, Gather and Permutation are compared bit for
bit; the FP32 kernels within the relative-L2 bound (the reference's detector sums
with atomicAdd in arbitrary order, and cuFFT's rounding differs from the Stockham
FFT's)."""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import golden_inputs as G  # noqa: E402

from oracle import formulas as O  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "reference_kernels.npz")
TOL = 1e-5


@pytest.fixture(scope="module")
def gold():
    if not os.path.exists(FIXTURE):
        pytest.skip("golden fixture missing: run tests/golden/make_golden.py on a GPU")
    return dict(np.load(FIXTURE))


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


# ----------------------------------------------------------------------------- CPU: oracle vs reference kernels
def test_oracle_cast_matches_reference_kernel(gold):
    x = G.cast_input()
    np.testing.assert_array_equal(O.cast_scalars(x.reshape(-1), np.float32), gold["cast_ci8_cf32"])


def test_oracle_beamformer_matches_reference_kernel(gold):
    x, w = G.bf_inputs()
    assert rel(O.beamform(x, w), gold["beamformer"]) < TOL
    ref = O.beamform(x, w, True, True)
    assert rel(ref, gold["beamformer_inc_sqrt"]) < TOL


def test_oracle_detector_matches_reference_kernel(gold):
    x = G.det_input()
    assert rel(O.detect(x, G.DET["I"], 1), gold["detector_1pol"]) < TOL
    assert rel(O.detect(x, G.DET["I"], 4), gold["detector_4pol"]) < TOL


def test_oracle_channelizer_matches_reference_kernel(gold):
    x = G.ch_input()
    assert rel(O.channelize(x, G.CH["T"]), gold["channelizer_rate_T"]) < TOL


def need(gold, *keys):
    missing = [k for k in keys if k not in gold]
    if missing:
        pytest.skip(f"golden fixture lacks {missing}: rerun tests/golden/make_golden.py on a GPU")


def cf16_to_complex(h):
    return h[..., 0].astype(np.float64) + 1j * h[..., 1].astype(np.float64)


def complex_to_cf16(y):
    return np.stack([y.real, y.imag], axis=-1).astype(np.float16)


def test_oracle_polarizer_matches_reference_kernel(gold):
    need(gold, "polarizer_cf32", "polarizer_cf16")
    # FP64 sums of two FP32 (FP16) values are exact here, so rounding them once
    # gives the correctly rounded FP32 (FP16) sums the kernel must produce
    np.testing.assert_array_equal(O.polarize(G.pol_input_cf32()).astype(np.complex64), gold["polarizer_cf32"])
    np.testing.assert_array_equal(complex_to_cf16(O.polarize(cf16_to_complex(G.pol_input_cf16()))),
                                  gold["polarizer_cf16"])


def test_oracle_gather_matches_reference_kernel(gold):
    need(gold, *[f"gather_case{c}" for c in range(len(G.GATHER_CASES))])
    for c, (_, axis, _) in enumerate(G.GATHER_CASES):
        np.testing.assert_array_equal(O.gather(G.gather_inputs(c), axis), gold[f"gather_case{c}"])


def test_oracle_permutation_matches_reference_kernel(gold):
    keys = ["permute_" + "".join(map(str, idx)) for idx in G.PERMS]
    need(gold, *keys)
    x = G.perm_input()
    for idx, key in zip(G.PERMS, keys):
        np.testing.assert_array_equal(O.permute(x, idx), gold[key])


# ----------------------------------------------------------------------------- GPU: our kernels vs reference kernels
@pytest.mark.gpu
def test_byte_kernels_match_reference_kernels(cuda, gold):
    """Polarizer (CF32, CF16), Gather (CHRONOUS, every step) and Permutation against
    the reference's own kernels, bit for bit."""
    import torch

    from blade_b200 import _lib
    from tests.gpu_util import call, dev, host, ptr, stream

    perm_keys = ["permute_" + "".join(map(str, idx)) for idx in G.PERMS]
    need(gold, "polarizer_cf32", "polarizer_cf16", *perm_keys,
         *[f"gather_case{c}" for c in range(len(G.GATHER_CASES))])
    n = int(np.prod(G.POL_SHAPE[:3]))  # dual-polarisation samples
    for key, x, code in (("polarizer_cf32", G.pol_input_cf32(), _lib.CF32),
                         ("polarizer_cf16", G.pol_input_cf16(), _lib.CF16)):
        xd = dev(x)
        call("blade_polarize", code, ptr(xd), ptr(xd), n, stream())
        np.testing.assert_array_equal(host(xd), gold[key])

    for c, (shape, axis, mult) in enumerate(G.GATHER_CASES):
        oshape = list(shape)
        oshape[axis] *= mult
        od = torch.zeros(oshape, dtype=torch.complex64, device="cuda")
        for step, x in enumerate(G.gather_inputs(c)):
            xd = dev(x)
            call("blade_gather", 8, ptr(xd), ptr(od), _lib.u64_array(shape), axis, mult, step, stream())
            torch.cuda.synchronize()
        np.testing.assert_array_equal(host(od), gold[f"gather_case{c}"])

    x = G.perm_input()
    xd = dev(x)
    for idx, key in zip(G.PERMS, perm_keys):
        od = torch.zeros([G.PERM_SHAPE[i] for i in idx], dtype=torch.complex64, device="cuda")
        call("blade_permute", 8, ptr(xd), ptr(od), _lib.u64_array(G.PERM_SHAPE), _lib.u64_array(idx), stream())
        np.testing.assert_array_equal(host(od), gold[key])


# ----------------------------------------------------------------------------- GPU: our kernels vs reference kernels (FP32)
@pytest.mark.gpu
def test_kernels_match_reference_kernels(cuda, gold):
    import torch

    from blade_b200 import _lib
    from tests.gpu_util import c64, call, dev, host, ptr, stream

    x = G.cast_input()
    xd = dev(x)
    yd = torch.zeros(x.size, dtype=torch.float32, device="cuda")
    call("blade_cast", _lib.CI8, _lib.CF32, ptr(xd), ptr(yd), x.size // 2, stream())
    np.testing.assert_array_equal(host(yd), gold["cast_ci8_cf32"])

    x, w = G.bf_inputs()
    A, F, T, B = G.BF["A"], G.BF["F"], G.BF["T"], G.BF["B"]
    xd, wd = c64(x), c64(w)
    od = torch.zeros((B + 1, F, T, 2), dtype=torch.complex64, device="cuda")
    call("blade_beamform_f32", ptr(xd), ptr(wd), ptr(od), B, A, F, T, 2, 1, 1, stream())
    assert rel(host(od), gold["beamformer_inc_sqrt"]) < TOL

    x = G.det_input()
    A, F, T, I = G.DET["A"], G.DET["F"], G.DET["T"], G.DET["I"]
    xd = c64(x)
    for npol, key in ((1, "detector_1pol"), (4, "detector_4pol")):
        od = torch.zeros((A, F, T // I, npol), dtype=torch.float32, device="cuda")
        call("blade_detect", ptr(xd), ptr(od), A, F, T, 2, I, npol, stream())
        assert rel(host(od), gold[key]) < TOL

    x = G.ch_input()
    A, F, T = G.CH["A"], G.CH["F"], G.CH["T"]
    xd = c64(x)
    call("blade_channelize", ptr(xd), ptr(xd), None, A, F, T, 2, T, stream())
    assert rel(host(xd).reshape(A, F * T, 1, 2), gold["channelizer_rate_T"]) < TOL
