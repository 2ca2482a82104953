"""CPU: the FP64 oracle against the literal loop restatements and against the
reference formulas it restates (tests/modules/*/*.py of the reference)."""

import numpy as np
import pytest

from oracle import formulas as O
from oracle import loops as L


def crand(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("inc,sq", [(False, False), (True, False), (True, True)])
def test_beamform_matches_loops(inc, sq):
    rng = np.random.default_rng(1)
    x = crand(rng, (3, 4, 5, 2))
    w = crand(rng, (2, 3, 4, 1, 2))
    np.testing.assert_allclose(O.beamform(x, w, inc, sq), L.beamform(x, w, inc, sq), rtol=1e-12, atol=1e-12)


def test_beamform_reference_test_formula():
    # tests/modules/beamformer/ata.py:56-63 with one beam (beam 0 == beam -1).
    rng = np.random.default_rng(2)
    x = crand(rng, (2, 6, 8, 2))
    w = crand(rng, (1, 2, 6, 1, 2))
    ref = np.zeros((2, 6, 8, 2), dtype=np.complex128)
    ref[0] = (x * w[0][..., :]).sum(axis=0)
    ph = x * w[-1][..., :]
    ref[-1] = np.sqrt((ph.real * ph.real + ph.imag * ph.imag).sum(axis=0))
    np.testing.assert_allclose(O.beamform(x, w, True, True), ref, rtol=1e-12)


@pytest.mark.parametrize("npol", [1, 4])
@pytest.mark.parametrize("integ", [1, 2, 5])
def test_detect_matches_loops(npol, integ):
    rng = np.random.default_rng(3)
    x = crand(rng, (2, 3, 10, 2))
    np.testing.assert_allclose(O.detect(x, integ, npol), L.detect(x, integ, npol), rtol=1e-12, atol=1e-12)


def test_detect_reference_cross_pol_formula():
    # tests/modules/detector/cross_pol.py:58-71
    rng = np.random.default_rng(4)
    x = crand(rng, (2, 3, 20, 2))
    I = 10
    out = O.detect(x, I, 4)
    for b in range(2):
        for c in range(3):
            for s in range(2):
                X = x[b, c, s * I:(s + 1) * I, 0]
                Y = x[b, c, s * I:(s + 1) * I, 1]
                cross = X * np.conj(Y)
                np.testing.assert_allclose(out[b, c, s], [np.sum((X * np.conj(X)).real), np.sum((Y * np.conj(Y)).real),
                                                          np.sum(cross.real), np.sum(cross.imag)], rtol=1e-12)


@pytest.mark.parametrize("rate", [2, 4, 6, 8, 10])
def test_channelize_matches_loops(rate):
    rng = np.random.default_rng(5)
    x = crand(rng, (2, 3, 2 * rate, 2))
    np.testing.assert_allclose(O.channelize(x, rate), L.channelize(x, rate), rtol=1e-10, atol=1e-10)


def test_channelize_reference_test_formula():
    # tests/modules/channelizer/advanced.py:49-65 (general rate)
    rng = np.random.default_rng(6)
    A, F, T, P, C = 2, 3, 16, 2, 4
    x = crand(rng, (A, F, T, P))
    ref = np.zeros((A, F * C, T // C, P), dtype=np.complex128)
    for a in range(A):
        for f in range(F):
            for p in range(P):
                for s in range(T // C):
                    ref[a, f * C:(f + 1) * C, s, p] = np.fft.fftshift(np.fft.fft(x[a, f, s * C:(s + 1) * C, p]))
    np.testing.assert_allclose(O.channelize(x, C), ref, rtol=1e-12, atol=1e-12)


def test_polarize():
    rng = np.random.default_rng(7)
    x = crand(rng, (2, 3, 4, 2))
    out = O.polarize(x)
    np.testing.assert_allclose(out[..., 0], x[..., 0] + 1j * x[..., 1])
    np.testing.assert_allclose(out[..., 1], x[..., 0] - 1j * x[..., 1])


# Reference gather cases, tests/modules/gather/meson.build:4-68 (shrunk where large).
GATHER_CASES = [(2, 6, 16, 2, 2, 4), (3, 7, 3, 1, 0, 5), (1, 2, 5, 6, 1, 6), (11, 1, 13, 9, 2, 7), (9, 2, 1, 3, 3, 8),
                (9, 2, 55, 3, 2, 8)]


@pytest.mark.parametrize("A,F,T,P,axis,m", GATHER_CASES)
def test_gather_matches_loops(A, F, T, P, axis, m):
    rng = np.random.default_rng(8)
    blocks = [crand(rng, (A, F, T, P)) for _ in range(m)]
    shape = [A, F, T, P]
    shape[axis] *= m
    out = np.zeros(shape, dtype=np.complex128)
    for step, b in enumerate(blocks):
        L.gather_step(out, b, axis, step)
    np.testing.assert_array_equal(O.gather(blocks, axis), out)


@pytest.mark.parametrize("perm", [(0, 1, 2, 3), (0, 2, 1, 3), (3, 2, 1, 0), (2, 0, 3, 1)])
def test_permute_matches_loops(perm):
    rng = np.random.default_rng(9)
    x = crand(rng, (2, 3, 4, 2))
    np.testing.assert_array_equal(O.permute(x, perm), L.permute(x, perm))


def test_phasors_from_delays_matches_mode_b_formula():
    # tests/bundles/ata/mode_b.py:302-313 (create_delay_phasors * get_fringe_rate) times calibration.
    rng = np.random.default_rng(10)
    B, A, F, P = 2, 3, 5, 2
    tau = rng.uniform(-5e-6, 5e-6, size=(B, A))
    cal = crand(rng, (A, F, 1, P))
    rf, bw, tot, start = 6500.125e6, 0.5e6, 1.024e9, 352
    out = O.phasors_from_delays(tau, cal, rf, bw, tot, start)
    freqs = np.arange(start, start + F) * bw
    for b in range(B):
        for a in range(A):
            ph = np.exp(-1j * 2 * np.pi * tau[b, a] * freqs) * np.exp(-1j * 2 * np.pi * tau[b, a] * (rf - tot / 2.0))
            for p in range(P):
                np.testing.assert_allclose(out[b, a, :, 0, p], ph * cal[a, :, 0, p], rtol=1e-9)


def test_cast_semantics():
    x = np.array([-2.7, -0.5, 0.5, 2.7, 127.9], dtype=np.float32)
    np.testing.assert_array_equal(O.cast_scalars(x, np.int32), [-2, 0, 0, 2, 127])
    h = O.cast_scalars(np.array([1.0 + 2 ** -11], dtype=np.float32), np.float16)
    assert h[0] == np.float16(1.0)  # round half to even


def test_grad_matches_finite_differences():
    rng = np.random.default_rng(11)
    x = crand(rng, (3, 2, 6, 2))
    w = crand(rng, (2, 3, 2, 1, 2))
    g = O.stokes_loss_grad(x, w)
    h = 1e-6
    for idx in [(0, 0, 0, 0, 0), (1, 2, 1, 0, 1), (0, 1, 1, 0, 0)]:
        e = np.zeros_like(w)
        e[idx] = h
        dre = (O.stokes_loss(x, w + e) - O.stokes_loss(x, w - e)) / (2 * h)
        dim = (O.stokes_loss(x, w + 1j * e) - O.stokes_loss(x, w - 1j * e)) / (2 * h)
        np.testing.assert_allclose(dre, 2 * g[idx].real, rtol=1e-6)
        np.testing.assert_allclose(dim, 2 * g[idx].imag, rtol=1e-6)


def test_chain_rate4_equals_stepwise():
    from blade_b200 import synthetic as S

    rng = np.random.default_rng(12)
    x = S.ci8_voltages(rng, (3, 2, 32, 2))
    _, w = S.phasors(rng, 2, 3, 2)
    y = O.beamform_channelize_detect(x, w, 4, 2)
    step = O.detect(O.channelize(O.beamform(O.ci8_to_complex(x), w), 4), 2, 1)
    np.testing.assert_allclose(y, step, rtol=1e-12)


def test_mode_b_matches_reference_test_loops():
    # tests/bundles/ata/mode_b.py:377-390: per beam, the antenna sum of input x phasors,
    # then |x|^2 + |y|^2 per sample (rate 1, integration 1, no polarizer).
    rng = np.random.default_rng(13)
    A, F, T, P, B = 4, 3, 8, 2, 2
    x = crand(rng, (A, F, T, P))
    w = crand(rng, (B, A, F, 1, P))
    out = np.zeros((B, F, T, 1))
    for ib in range(B):
        phased = (x.astype(np.complex128) * w[ib][..., :].astype(np.complex128)).sum(axis=0)
        for ic in range(F):
            for it in range(T):
                xx, yy = phased[ic, it, 0], phased[ic, it, 1]
                out[ib, ic, it, 0] = xx.real * xx.real + xx.imag * xx.imag + yy.real * yy.real + yy.imag * yy.imag
    np.testing.assert_allclose(O.mode_b(x, w, 1), out, rtol=1e-12)


def test_mode_b_incoherent_beam_is_square_rooted_before_the_detector():
    rng = np.random.default_rng(14)
    x = crand(rng, (3, 2, 16, 2))
    w = crand(rng, (2, 3, 4, 1, 2))
    out = O.mode_b(x, w, 2, circular=True, incoherent=True, detector=True, integration=2)
    y = O.polarize(O.channelize(x, 2))
    inc = (np.abs(y * w[0]) ** 2).sum(axis=0)                # [F*R, T/R, P]
    ref = (inc.reshape(4, 4, 2, 2)).sum(axis=(2, 3))         # sqrt then |.|^2 gives the sum back
    np.testing.assert_allclose(out[2, :, :, 0], ref, rtol=1e-12)
    stepwise = O.detect(O.beamform(y, w), 2, 1)
    np.testing.assert_allclose(out[:2], stepwise, rtol=1e-12)


def test_beamform_meerkat_reads_flat_beam_antenna_weights():
    # src/modules/beamformer/beamformer.cu:103-114: iy runs 0, 1, ... over (beam, antenna)
    rng = np.random.default_rng(15)
    A, F, T, P, B = 3, 2, 4, 2, 2
    x = crand(rng, (A, F, T, P))
    w = crand(rng, (B, A, F, 1, P))
    flat = w.reshape(-1)
    out = O.beamform_meerkat(x, w, B, incoherent=True)
    assert out.shape == (B + 1, F, T, P)
    for b in range(B):
        for f in range(F):
            for t in range(T):
                for p in range(P):
                    ref = sum(x[a, f, t, p] * flat[b * A + a] for a in range(A))
                    np.testing.assert_allclose(out[b, f, t, p], ref, rtol=1e-12)
    assert np.all(out[B] == 0)
