"""GPU: the launch-shape autotuner.

For each family, a tuning call on the caller's shape must time every candidate,
find every candidate's output bit-identical to the default's (params[5] == 0),
and make later launches of that shape use the stored choice: the query reports
it, and the tuned launch reproduces the default launch bit for bit (and the FP64
oracle within the chain bound)."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from blade_b200 import _lib, synthetic as S
from oracle import formulas as O
from tests.gpu_util import c64, call, dev, host, ptr, rel_l2, stream

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def fresh_cache():
    bl.autotune.clear()
    yield
    bl.autotune.clear()


TC_SHAPES = [
    ("ata-production", 28, 12, 8192, 16, 4, 4),
    ("dense-64x64", 64, 6, 8192, 64, 1, 8),
    ("ata-small", 20, 96, 256, 8, 1, 4),
    ("ragged-beams", 13, 3, 512, 37, 4, 2),
]


@pytest.mark.parametrize("name,A,F,T,B,R,I", TC_SHAPES)
def test_tensor_core_autotune(cuda, name, A, F, T, B, R, I):
    rng = np.random.default_rng(7)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    _, w = S.phasors(rng, B, A, F)
    xd, wd = dev(x), c64(w.astype(np.complex64))
    lib = _lib.load()
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    shape = (B, F * R, T // (R * I), 1)
    key = (B, A, F, T, 2, R, I, 4)

    def run():
        o = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
        call("blade_beamform_prepare_detect_tc", ptr(wd), ptr(plan), ptr(xd), ptr(o), B, A, F, T, 2, R, I, stream())
        return host(o)

    before = bl.autotune.query(bl.autotune.TC, key)
    assert not before["tuned"]
    y0 = run()
    info = bl.autotune.tensor_core(B, A, F, T, R, I)
    print(f"{name}: default {before['params'][:4]} -> tuned {info['params'][:4]} "
          f"({info['params'][4]} candidates, {info['us']:.1f} us)")
    assert info["tuned"] and info["params"][4] >= 2 and info["params"][5] == 0
    assert bl.device_status() == 0
    y1 = run()
    np.testing.assert_array_equal(y1, y0)
    assert rel_l2(y1, O.beamform_channelize_detect(x, w, R, I)) < 1e-5


F32_SHAPES = [
    ("ata-production-ci8", _lib.CI8, 28, 8, 2048, 16, 4, 4),
    ("ata-small-ci8", _lib.CI8, 20, 96, 256, 8, 1, 4),
    ("calibration-cf32", _lib.CF32, 28, 8, 512, 1, 1, 1),
]


@pytest.mark.parametrize("name,it,A,F,T,B,R,I", F32_SHAPES)
def test_fp32_autotune(cuda, name, it, A, F, T, B, R, I):
    rng = np.random.default_rng(8)
    if it == _lib.CI8:
        x = S.ci8_voltages(rng, (A, F, T, 2))
        xd = dev(x)
    else:
        x = (rng.standard_normal((A, F, T, 2)) + 1j * rng.standard_normal((A, F, T, 2))).astype(np.complex64)
        xd = c64(x)
    _, w = S.phasors(rng, B, A, F)
    wd = c64(w.astype(np.complex64))
    shape = (B, F * R, T // (R * I), 1)

    def run():
        o = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
        call("blade_beamform_detect_f32", it, ptr(xd), ptr(wd), ptr(o), B, A, F, T, 2, R, I, stream())
        return host(o)

    y0 = run()
    info = bl.autotune.fp32(B, A, F, T, R, I, in_type=it)
    print(f"{name}: TG {info['params'][0]} ({info['params'][4]} candidates, {info['us']:.1f} us)")
    assert info["tuned"] and info["params"][4] >= 1 and info["params"][5] == 0
    np.testing.assert_array_equal(run(), y0)


def test_spectrometer_autotune(cuda):
    A, F, T, R, I = 1, 2, 1 << 20, 65536, 8
    rng = np.random.default_rng(9)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    xd = dev(x)
    lib = _lib.load()
    ws = torch.empty(int(lib.blade_spectrometer_workspace_size(A, F, T, 2, R)), dtype=torch.uint8, device="cuda")

    def run():
        o = torch.full((A, F * R, T // (R * I), 1), float("nan"), dtype=torch.float32, device="cuda")
        call("blade_spectrometer", _lib.CI8, ptr(xd), _lib.F32, ptr(o), ptr(ws), A, F, T, 2, R, I, 1, 1, stream())
        return host(o)

    y0 = run()
    info = bl.autotune.spectrometer(A, F, T, R, I)
    print(f"spectrometer: CTAs per SM {info['params'][:2]} ({info['params'][4]} candidates, {info['us']:.1f} us)")
    assert info["tuned"] and info["params"][4] == 9 and info["params"][5] == 0
    np.testing.assert_array_equal(run(), y0)


def test_module_autotune_flag(cuda):
    A, F, T, B, R, I = 28, 4, 2048, 16, 4, 4
    rng = np.random.default_rng(10)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    _, w = S.phasors(rng, B, A, F)
    buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cuda)
    buf.as_torch().copy_(torch.from_numpy(x))
    ph = bl.phasor_tensor((B, A, F, 1, 2), dtype=bl.cf32, device=bl.cuda)
    ph.as_torch().copy_(torch.from_numpy(w.astype(np.complex64)))
    mod = bl.module(bl.beamform_detect, {"rate": R, "integration_size": I, "autotune": True}, (buf, ph),
                    telescope=bl.ata)
    assert bl.autotune.query(bl.autotune.TC, (B, A, F, T, 2, R, I, 4))["tuned"]
    mod.process(0, bl.stream())
    got = host(mod.get_output().as_torch())
    assert rel_l2(got, O.beamform_channelize_detect(x, w, R, I)) < 1e-5
