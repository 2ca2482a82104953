"""GPU: the fused spectrometer (blade_spectrometer, the ModeH bundle of
include/blade/bundles/generic/mode_h.hh:55-106 in two kernels) against the module
chain Cast -> Channelizer -> [Polarizer] -> Detector on the same device, against
the FP64 oracle (tests/bundles/generic/mode_h.py:56-74 restated in
oracle/formulas.py), and through bl.module(bl.modeh, ...)."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from oracle import formulas as O
from blade_b200 import _lib
from tests.gpu_util import call, dev, host, ptr, rel_l2, stream

pytestmark = pytest.mark.gpu
TOL = 1e-5
R = 65536


def ci8_voltages(A, F, T, seed):
    rng = np.random.default_rng(seed)
    return np.clip(np.rint(rng.standard_normal((A, F, T, 2, 2)) * 8), -127, 127).astype(np.int8)


def fused(x, in_type, A, F, T, I, OP, circular, out_type=_lib.F32):
    ws = torch.empty(int(_lib.load().blade_spectrometer_workspace_size(A, F, T, 2, R)), dtype=torch.uint8,
                     device="cuda")
    out = torch.empty((A, F * R, T // (R * I), OP), dtype=torch.float32 if out_type == _lib.F32 else torch.float16,
                      device="cuda")
    call("blade_spectrometer", in_type, ptr(x), out_type, ptr(out), ptr(ws), A, F, T, 2, R, I, OP, circular,
         stream())
    return out


def chain(x_ci8, A, F, T, I, OP, circular):
    n = A * F * T * 2
    xf = torch.empty((A, F, T, 2), dtype=torch.complex64, device="cuda")
    call("blade_cast", _lib.CI8, _lib.CF32, ptr(x_ci8), ptr(xf), n, stream())
    yc = torch.empty((A, F * R, T // R, 2), dtype=torch.complex64, device="cuda")
    ws = torch.empty(int(_lib.load().blade_channelize_workspace_size(A, F, T, 2, R)), dtype=torch.uint8,
                     device="cuda")
    call("blade_channelize", ptr(xf), ptr(yc), ptr(ws), A, F, T, 2, R, stream())
    if circular:
        call("blade_polarize", _lib.CF32, ptr(yc), ptr(yc), A * F * T, stream())
    out = torch.empty((A, F * R, T // (R * I), OP), dtype=torch.float32, device="cuda")
    call("blade_detect", ptr(yc), ptr(out), A, F * R, T // R, 2, I, OP, stream())
    return out, xf


@pytest.mark.parametrize("OP", [1, 4])
@pytest.mark.parametrize("circular", [0, 1])
@pytest.mark.parametrize("I", [1, 2])
def test_fused_matches_module_chain(cuda, OP, circular, I):
    A, F, T = 1, 2, 2 * R
    x = dev(ci8_voltages(A, F, T, 71 + OP + 2 * circular + 4 * I))
    ref, xf = chain(x, A, F, T, I, OP, circular)
    got = fused(x, _lib.CI8, A, F, T, I, OP, circular)
    assert rel_l2(host(got), host(ref)) < TOL
    # CF32 input gives the same products
    got_f = fused(xf, _lib.CF32, A, F, T, I, OP, circular)
    assert rel_l2(host(got_f), host(got)) < 1e-6


@pytest.mark.parametrize("OP,circular", [(1, 1), (4, 0)])
def test_fused_matches_oracle(cuda, OP, circular):
    A, F, T, I = 1, 1, 2 * R, 2
    xh = ci8_voltages(A, F, T, 5 + OP)
    got = fused(dev(xh), _lib.CI8, A, F, T, I, OP, circular)
    ref = O.spectrometer(xh, R, I, polarizer=bool(circular), npols=OP)
    assert rel_l2(host(got), ref) < TOL


def test_f16_output_is_the_rounded_f32_output(cuda):
    A, F, T, I = 1, 1, 4 * R, 4
    x = dev(ci8_voltages(A, F, T, 9))
    o32 = fused(x, _lib.CI8, A, F, T, I, 1, 1)
    o16 = fused(x, _lib.CI8, A, F, T, I, 1, 1, out_type=_lib.F16)
    assert torch.equal(o32.half(), o16)


def test_modeh_module(cuda):
    A, F, T = 1, 2, R
    xh = ci8_voltages(A, F, T, 13)
    buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cuda)
    buf.as_torch().copy_(dev(xh))
    mod = bl.module(bl.modeh, {"input_shape": (A, F, T, 2), "output_shape": (A, F * T, 1, 1),
                               "polarizer_convert_to_circular": True, "detector_integration_size": 1,
                               "detector_number_of_output_polarizations": 1},
                    {"buffer": buf}, it=bl.ci8, ot=bl.f32)
    mod.process()
    torch.cuda.synchronize()
    got = mod.get_output().as_torch().cpu().numpy()
    ref = O.spectrometer(xh, T, 1, polarizer=True, npols=1)
    assert rel_l2(got, ref) < TOL


def test_modeh_rejects_wrong_output_shape(cuda):
    A, F, T = 1, 1, R
    buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cuda)
    with pytest.raises(RuntimeError):
        bl.module(bl.modeh, {"input_shape": (A, F, T, 2), "output_shape": (A, F * T, 2, 1),
                             "polarizer_convert_to_circular": False, "detector_integration_size": 1,
                             "detector_number_of_output_polarizations": 1}, {"buffer": buf})
