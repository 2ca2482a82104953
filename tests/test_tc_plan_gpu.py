"""The tensor-core chain's phasor image ("plan", blade_beamform_tc_prepare) byte
for byte against a numpy restatement of its layout: each CF32 phasor split into
FP16 hi = rn(w) and lo = rn(w - hi) per component, laid out per (chunk, channel,
polarisation) as K-major 128-byte-swizzled blocks (16-byte chunk c of row r at
chunk c ^ (r & 7) of the row, 8-row groups of 1 KB):
  * KA = 64 without stacking (more than 32 beams): per hi/lo, three blocks of NB
    rows x 64 antennas, [-Wi | Wr | Wi];
  * KA = 32 without stacking: per hi/lo, one block of 2 NB rows x 64 K, row nb =
    [Wr | -Wi], row NB + nb = [Wi | Wr];
  * stacked (NB <= 32): (2 KA / 64) column blocks of 4 NB rows, rows nb, NB + nb,
    2 NB + nb, 3 NB + nb = hi [Wr | -Wi], hi [Wi | Wr], lo [Wr | -Wi], lo [Wi | Wr].
Padded antennas and beams are zero."""

import numpy as np
import pytest
import torch

from blade_b200 import _lib
from tests.gpu_util import c64, call, ptr, stream

pytestmark = pytest.mark.gpu


def _split(w):
    """FP16 hi and lo of each FP32 component (the FP32 subtraction is exact)."""
    w32 = w.astype(np.complex64)
    re, im = w32.real.astype(np.float32), w32.imag.astype(np.float32)
    rh, ih = re.astype(np.float16), im.astype(np.float16)
    rl = (re - rh.astype(np.float32)).astype(np.float16)
    il = (im - ih.astype(np.float32)).astype(np.float16)
    return rh, ih, rl, il


def _put(img, base, rows, row, k, vals):
    """Eight FP16 values of K elements k .. k + 7 of `row` in a swizzled operand."""
    blk, c = k // 64, (k % 64) // 8
    off = base + blk * rows * 128 + (row // 8) * 1024 + (row % 8) * 128 + ((c ^ (row % 8)) * 16)
    img[off:off + 16] = np.ascontiguousarray(vals, dtype=np.float16).view(np.uint8)


def expected_plan(w, B, A, F):
    bc = min(B, 64)
    NB = (bc + 15) // 16 * 16
    KA = 32 if A <= 32 else 64
    stacked = NB <= 32
    nch = (B + 63) // 64
    img_bytes = (2 * KA // 64) * 1024 * NB if stacked else (1536 if KA == 64 else 1024) * NB
    ph_bytes = (3 if KA == 64 else 2) * NB * 128
    pol_stacked = (2 * KA // 64) * 4 * NB * 128
    plan = np.zeros(nch * F * img_bytes, dtype=np.uint8)
    wp = np.zeros((nch * 64, KA, F, 2), dtype=np.complex64)
    wp[:B, :A] = w[:, :, :, 0, :]
    rh, ih, rl, il = _split(wp)
    for c in range(nch):
        for f in range(F):
            for p in range(2):
                for nb in range(NB):
                    b = c * 64 + nb
                    for j in range(KA // 8):
                        s = slice(8 * j, 8 * j + 8)
                        h_re, h_im, l_re, l_im = rh[b, s, f, p], ih[b, s, f, p], rl[b, s, f, p], il[b, s, f, p]
                        k0 = 8 * j
                        if stacked:
                            base = (c * F + f) * img_bytes + p * pol_stacked
                            rows = 4 * NB
                            _put(plan, base, rows, nb, k0, h_re)
                            _put(plan, base, rows, nb, KA + k0, -h_im)
                            _put(plan, base, rows, NB + nb, k0, h_im)
                            _put(plan, base, rows, NB + nb, KA + k0, h_re)
                            _put(plan, base, rows, 2 * NB + nb, k0, l_re)
                            _put(plan, base, rows, 2 * NB + nb, KA + k0, -l_im)
                            _put(plan, base, rows, 3 * NB + nb, k0, l_im)
                            _put(plan, base, rows, 3 * NB + nb, KA + k0, l_re)
                            continue
                        base = (c * F + f) * img_bytes + p * 2 * ph_bytes
                        for h, (re, im) in enumerate(((h_re, h_im), (l_re, l_im))):
                            blk = base + h * ph_bytes
                            if KA == 64:
                                _put(plan, blk, NB, nb, k0, -im)
                                _put(plan, blk + NB * 128, NB, nb, k0, re)
                                _put(plan, blk + 2 * NB * 128, NB, nb, k0, im)
                            else:
                                _put(plan, blk, 2 * NB, nb, k0, re)
                                _put(plan, blk, 2 * NB, nb, 32 + k0, -im)
                                _put(plan, blk, 2 * NB, NB + nb, k0, im)
                                _put(plan, blk, 2 * NB, NB + nb, 32 + k0, re)
    return plan


@pytest.mark.parametrize("B,A,F", [(64, 64, 5), (100, 50, 3), (49, 61, 6), (40, 20, 3), (16, 28, 4), (8, 40, 2)])
def test_plan_bytes_match_the_layout(cuda, B, A, F):
    rng = np.random.default_rng(B * 1000 + A)
    w = (rng.standard_normal((B, A, F, 1, 2)) + 1j * rng.standard_normal((B, A, F, 1, 2))).astype(np.complex64)
    lib = _lib.load()
    plan = torch.full((int(lib.blade_beamform_tc_plan_size(B, A, F, 2)),), 0x5A, dtype=torch.uint8, device="cuda")
    call("blade_beamform_tc_prepare", ptr(c64(w)), ptr(plan), B, A, F, 2, stream())
    got = plan.cpu().numpy()
    exp = expected_plan(w, B, A, F)
    assert got.shape == exp.shape
    np.testing.assert_array_equal(got, exp)
