"""GPU: ATA ModeB in the reference's order on tensor cores — the pre-beamformer
Cast -> Channelizer -> [Polarizer] into exact FP16 (blade_prechannelize_cf16,
include/blade/bundles/ata/mode_b.hh:99-139) and the tensor-core Beamformer ->
Detector on the fine channels (blade_beamform_detect_tc_cf16) — against the FP64
oracle (oracle/formulas.py mode_b: the chain of mode_b.hh and the Stokes-I of
tests/bundles/ata/mode_b.py:377-390)."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from oracle import formulas as O
from blade_b200 import _lib
from tests.gpu_util import call, dev, host, ptr, rel_l2, stream

pytestmark = pytest.mark.gpu
TOL = 1e-5


def ci8(A, F, T, seed):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.standard_normal((A, F, T, 2, 2)) * 8), -127, 127).astype(np.int8)


def phasors(B, A, F, seed):
    rng = np.random.default_rng(seed)
    ph = np.exp(2j * np.pi * rng.random((B, A, F, 1, 1)))
    return np.repeat(ph, 2, axis=4).astype(np.complex64)


def pre(x, R, circular):
    A, F, T = x.shape[:3]
    out = torch.empty((A, F * R, T // R, 2, 2), dtype=torch.float16, device="cuda")
    call("blade_prechannelize_cf16", ptr(x), ptr(out), A, F, T, 2, R, circular, stream())
    return out


@pytest.mark.parametrize("R", [1, 2, 4])
@pytest.mark.parametrize("circular", [0, 1])
def test_prechannelize_is_exact(cuda, R, circular):
    A, F, T = 3, 5, 64
    xh = ci8(A, F, T, 10 + R + circular)
    got = host(pre(dev(xh), R, circular)).astype(np.float64)
    ref = O.channelize(O.ci8_to_complex(xh), R)
    if circular:
        ref = O.polarize(ref)
    np.testing.assert_array_equal(got[..., 0] + 1j * got[..., 1], ref)  # integers <= 1024: exact in FP16


def test_prechannelize_rejects_bad_arguments(cuda):
    x = dev(ci8(1, 1, 64, 0))
    out = torch.empty(64 * 4, dtype=torch.float16, device="cuda")
    with pytest.raises(RuntimeError):
        call("blade_prechannelize_cf16", ptr(x), ptr(out), 1, 1, 64, 2, 8, 0, stream())  # rate > 4
    with pytest.raises(RuntimeError):
        call("blade_prechannelize_cf16", ptr(x), ptr(out), 1, 1, 63, 2, 2, 0, stream())  # T % rate


@pytest.mark.parametrize("A,F,T,B,R,I,circ", [
    (28, 4, 2048, 16, 4, 4, 0),   # ATA production shape per channel, stacked hi/lo image
    (28, 3, 1024, 16, 4, 1, 1),
    (20, 2, 512, 40, 2, 2, 0),    # NB > 32: separate hi/lo MMAs, KA = 32
    (64, 2, 512, 64, 2, 8, 1),    # KA = 64, NB = 64: the single-issuer ring
])
def test_tensor_core_fine_channels_match_oracle(cuda, A, F, T, B, R, I, circ):
    xh, wh = ci8(A, F, T, A + B + R), phasors(B, A, F * R, I)
    x, w = dev(xh), dev(wh)
    y = pre(x, R, circ)
    plan = torch.empty(int(_lib.load().blade_beamform_tc_plan_size(B, A, F * R, 2)), dtype=torch.uint8, device="cuda")
    out = torch.empty((B, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    call("blade_beamform_tc_prepare", ptr(w), ptr(plan), B, A, F * R, 2, stream())
    call("blade_beamform_detect_tc_cf16", ptr(y), ptr(plan), ptr(out), B, A, F * R, T // R, 2, I, stream())
    ref = O.mode_b(xh, wh, R, bool(circ), False, True, I, 1)
    assert rel_l2(host(out), ref) < TOL
    # the split and the chain in one call (chain launched as the split's programmatic
    # dependent): the same bits, from a plan that first holds other phasors
    w2 = dev(phasors(B, A, F * R, I + 100))
    call("blade_beamform_tc_prepare", ptr(w2), ptr(plan), B, A, F * R, 2, stream())
    out2 = torch.full_like(out, float("nan"))
    call("blade_beamform_prepare_detect_tc_cf16", ptr(w), ptr(plan), ptr(y), ptr(out2), B, A, F * R, T // R, 2, I,
         stream())
    np.testing.assert_array_equal(host(out2), host(out))


def test_modeb_module_takes_the_tensor_core_path(cuda):
    A, F, T, B, R, I = 12, 4, 1024, 3, 4, 2
    xh, wh = ci8(A, F, T, 77), phasors(B, A, F * R, 78)
    buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cuda)
    buf.as_torch().copy_(dev(xh))
    ph = bl.phasor_tensor((B, A, F * R, 1, 2), dtype=bl.cf32, device=bl.cuda)
    ph.as_torch().copy_(dev(wh))
    cfg = {"input_shape": (A, F, T, 2), "output_shape": (B, F * R, T // (R * I), 1),
           "pre_beamformer_channelizer_rate": R, "pre_beamformer_polarizer_convert_to_circular": True,
           "detector_enable": True, "detector_integration_size": I, "detector_number_of_output_polarizations": 1}
    mod = bl.module(bl.modeb, cfg, {"buffer": buf, "phasors": ph}, it=bl.ci8, ot=bl.f32, telescope=bl.ata)
    assert mod.tensor_cores and not mod.fused
    for _ in range(2):  # the second call reuses the stage's buffers
        mod.process()
    torch.cuda.synchronize()
    got = mod.get_output().as_torch().cpu().numpy()
    assert rel_l2(got, O.mode_b(xh, wh, R, True, False, True, I, 1)) < TOL


@pytest.mark.parametrize("I", [1, 4, 32])
def test_incoherent_detect_matches_oracle(cuda, I):
    A, F, T, B, R = 10, 3, 512, 2, 4
    xh, wh = ci8(A, F, T, 40 + I), phasors(B, A, F * R, 41)
    wh = wh * np.linspace(0.5, 1.5, A)[None, :, None, None, None].astype(np.float32)  # unequal antenna gains
    x, w = dev(xh), dev(wh)
    y = pre(x, R, 1)
    out = torch.empty((F * R, T // (R * I)), dtype=torch.float32, device="cuda")
    call("blade_incoherent_detect_cf16", ptr(y), ptr(w), ptr(out), A, F * R, T // R, 2, I, stream())
    ref = O.mode_b(xh, wh, R, True, True, True, I, 1)[B, :, :, 0]
    assert rel_l2(host(out), ref) < TOL


def test_modeb_module_tensor_cores_with_incoherent_beam(cuda):
    A, F, T, B, R, I = 8, 4, 1024, 2, 2, 4
    xh, wh = ci8(A, F, T, 90), phasors(B, A, F * R, 91)
    buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cuda)
    buf.as_torch().copy_(dev(xh))
    ph = bl.phasor_tensor((B, A, F * R, 1, 2), dtype=bl.cf32, device=bl.cuda)
    ph.as_torch().copy_(dev(wh))
    cfg = {"input_shape": (A, F, T, 2), "output_shape": (B + 1, F * R, T // (R * I), 1),
           "pre_beamformer_channelizer_rate": R, "beamformer_incoherent_beam": True, "detector_enable": True,
           "detector_integration_size": I, "detector_number_of_output_polarizations": 1}
    mod = bl.module(bl.modeb, cfg, {"buffer": buf, "phasors": ph}, it=bl.ci8, ot=bl.f32, telescope=bl.ata)
    assert mod.tensor_cores
    mod.process()
    torch.cuda.synchronize()
    got = mod.get_output().as_torch().cpu().numpy()
    ref = O.mode_b(xh, wh, R, False, True, True, I, 1)
    assert rel_l2(got[:B], ref[:B]) < TOL
    assert rel_l2(got[B], ref[B]) < TOL
