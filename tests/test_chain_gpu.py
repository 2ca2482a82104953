"""GPU parity of the fused beamform -> channelize -> detect chains (FP32 CUDA
cores and FP16-split tcgen05 tensor cores) and of the adjoint, against the FP64
oracle, on the workload shapes (channel count reduced so the oracle stays fast).

The tensor-core path's Stokes-I error bound is 1e-5 relative L2 against FP64;
the FP32 path must meet the same bound."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from blade_b200 import _lib, synthetic as S
from oracle import formulas as O
from tests.gpu_util import c64, call, dev, host, ptr, rel_l2, stream

pytestmark = pytest.mark.gpu
TOL = 1e-5

# (name, A, F, T, B, rate, integ) -- workloads 1-3 with F reduced for the oracle
CHAINS = [
    ("ata-small", 20, 96, 256, 8, 1, 4),
    ("ata-production", 28, 12, 8192, 16, 4, 4),
    ("dense-64x64", 64, 6, 8192, 64, 1, 8),
    ("rate2", 28, 4, 1024, 16, 2, 8),
    ("ragged-beams", 13, 3, 512, 37, 4, 2),
    ("many-beams", 9, 2, 256, 100, 1, 1),
    ("window32", 16, 2, 1024, 16, 1, 32),
    # rate 4: few antennas (padded K), a full 32-antenna K, windows of 1, 8 and 32
    ("tmem-operand-5ant", 5, 3, 256, 3, 4, 1),
    ("tmem-operand-32ant", 32, 2, 1024, 16, 4, 32),
    ("tmem-operand-i8", 17, 5, 2048, 9, 4, 8),
    # rate 1 with a large phasor image (converters load the voltages directly): ragged
    # antennas and an odd number of tiles per CTA, 48 beams (padded rows), two beam chunks
    ("direct-ragged", 50, 40, 1152, 64, 1, 4),
    ("direct-48-beams", 64, 4, 2048, 48, 1, 16),
    ("direct-two-chunks", 64, 3, 1024, 100, 1, 8),
    ("direct-stacked-32-beams", 64, 4, 1024, 32, 1, 2),
    # accumulator with outputs along TMEM lanes (full 64-beam chunks, windows of 16):
    # an odd number of tiles per channel; two chunks with 40 beams in the second and
    # a 32-antenna K
    ("lanes-i16", 64, 5, 1152, 64, 1, 16),
    ("lanes-i16-two-chunks", 24, 3, 2048, 104, 1, 16),
]


def make(A, F, T, B, seed):
    rng = np.random.default_rng(seed)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    _, w = S.phasors(rng, B, A, F)
    return x, w.astype(np.complex64)


@pytest.mark.parametrize("name,A,F,T,B,R,I", CHAINS)
def test_fused_f32_chain(cuda, name, A, F, T, B, R, I):
    x, w = make(A, F, T, B, 1)
    ref = O.beamform_channelize_detect(x, w, R, I)
    xd, wd = dev(x), c64(w)
    od = torch.zeros((B, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    call("blade_beamform_detect_f32", _lib.CI8, ptr(xd), ptr(wd), ptr(od), B, A, F, T, 2, R, I, stream())
    assert rel_l2(host(od), ref) < TOL


@pytest.mark.parametrize("name,A,F,T,B,R,I", CHAINS)
def test_tensor_core_chain(cuda, name, A, F, T, B, R, I):
    x, w = make(A, F, T, B, 2)
    ref = O.beamform_channelize_detect(x, w, R, I)
    lib = _lib.load()
    assert lib.blade_beamform_detect_tc_supported(B, A, F, T, 2, R, I) == 1
    xd, wd = dev(x), c64(w)
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    od = torch.full((B, F * R, T // (R * I), 1), float("nan"), dtype=torch.float32, device="cuda")
    call("blade_beamform_tc_prepare", ptr(wd), ptr(plan), B, A, F, 2, stream())
    call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(od), B, A, F, T, 2, R, I, stream())
    y = host(od)
    assert bl.device_status() == 0
    assert np.isfinite(y).all()
    err = rel_l2(y, ref)
    print(f"{name}: Stokes-I relative L2 vs FP64 = {err:.3e}")
    assert err < TOL
    # deterministic
    od2 = torch.zeros_like(od)
    call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(od2), B, A, F, T, 2, R, I, stream())
    np.testing.assert_array_equal(host(od2), y)


@pytest.mark.parametrize("name,A,F,T,B,R,I", [CHAINS[1], CHAINS[4], CHAINS[5], CHAINS[10]])
def test_prepare_detect_tc_matches_two_calls(cuda, name, A, F, T, B, R, I):
    # the chain launched as a programmatic dependent of the split must read the
    # split's new image, never the plan's previous contents: each call below
    # rewrites the plan with different phasors
    x, w1 = make(A, F, T, B, 4)
    _, w2 = make(A, F, T, B, 5)
    lib = _lib.load()
    xd, w1d, w2d = dev(x), c64(w1), c64(w2)
    plan = torch.full((int(lib.blade_beamform_tc_plan_size(B, A, F, 2)),), 0x7F, dtype=torch.uint8, device="cuda")
    shape = (B, F * R, T // (R * I), 1)
    expect = []
    for wd in (w1d, w2d):
        o = torch.zeros(shape, dtype=torch.float32, device="cuda")
        call("blade_beamform_tc_prepare", ptr(wd), ptr(plan), B, A, F, 2, stream())
        call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(o), B, A, F, T, 2, R, I, stream())
        expect.append(host(o))
    plan.fill_(0x7F)
    for _ in range(3):
        for wd, e in zip((w1d, w2d), expect):
            o = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
            call("blade_beamform_prepare_detect_tc", ptr(wd), ptr(plan), ptr(xd), ptr(o), B, A, F, T, 2, R, I,
                 stream())
            np.testing.assert_array_equal(host(o), e)
    assert bl.device_status() == 0
    # captured into a CUDA graph (the programmatic edge is recorded), replayed alternately
    side = torch.cuda.Stream()
    outs = [torch.zeros(shape, dtype=torch.float32, device="cuda") for _ in range(2)]
    graphs = []
    with torch.cuda.stream(side):
        for wd, o in zip((w1d, w2d), outs):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=side):
                call("blade_beamform_prepare_detect_tc", ptr(wd), ptr(plan), ptr(xd), ptr(o), B, A, F, T, 2, R, I,
                     side.cuda_stream)
            graphs.append(g)
    for _ in range(3):
        for g, o, e in zip(graphs, outs, expect):
            o.fill_(float("nan"))
            g.replay()
            np.testing.assert_array_equal(host(o), e)
    assert bl.device_status() == 0


@pytest.mark.parametrize("I", [8, 16])
def test_tensor_core_chain_repeated_launches(cuda, I):
    # Hundreds of back-to-back launches of a full 64-beam chunk (the accumulator with
    # outputs along TMEM lanes): every CTA's range ends once per launch, where the
    # epilogue halves hand the last tile's partial sums over, so an ordering fault
    # there shows up as an expired bounded wait (a non-zero status word, ~2 s
    # launches) or as an output that differs from the first launch.
    A, F, T, B, R = 64, 16, 8192, 64, 1
    x, w = make(A, F, T, B, 6)
    lib = _lib.load()
    xd, wd = dev(x), c64(w)
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    call("blade_beamform_tc_prepare", ptr(wd), ptr(plan), B, A, F, 2, stream())
    outs = [torch.full((B, F * R, T // (R * I), 1), float("nan"), dtype=torch.float32, device="cuda")
            for _ in range(2)]
    first = None
    for k in range(400):
        o = outs[k % 2]
        call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(o), B, A, F, T, 2, R, I, stream())
        if k < 2:
            torch.cuda.synchronize()
            if k == 0:
                first = o.clone()
        elif k % 50 == 49:
            assert torch.equal(o, first)
            assert torch.equal(outs[(k + 1) % 2], first)
    torch.cuda.synchronize()
    assert bl.device_status() == 0
    assert rel_l2(host(first), O.beamform_channelize_detect(x, w, R, I)) < TOL


@pytest.mark.parametrize("I", [8, 16])
def test_tensor_core_chain_output_offset_by_one_float(cuda, I):
    # A full 64-beam chunk with the output 4 bytes past a 16-byte boundary takes the
    # lane-shuffle epilogue (the lane-major one stores 16-byte vectors); both meet the
    # FP64 bound and agree with each other.
    A, F, T, B, R = 64, 3, 2048, 64, 1
    x, w = make(A, F, T, B, 7)
    ref = O.beamform_channelize_detect(x, w, R, I)
    lib = _lib.load()
    xd, wd = dev(x), c64(w)
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    call("blade_beamform_tc_prepare", ptr(wd), ptr(plan), B, A, F, 2, stream())
    n = B * F * R * (T // (R * I))
    buf = torch.full((n + 4,), float("nan"), dtype=torch.float32, device="cuda")
    aligned, offset = buf[:n], buf[1:n + 1]
    assert aligned.data_ptr() % 16 == 0 and offset.data_ptr() % 16 == 4
    call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(offset), B, A, F, T, 2, R, I, stream())
    y_off = host(offset).reshape(ref.shape)
    call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(aligned), B, A, F, T, 2, R, I, stream())
    y_al = host(aligned).reshape(ref.shape)
    assert bl.device_status() == 0
    assert rel_l2(y_off, ref) < TOL and rel_l2(y_al, ref) < TOL
    assert rel_l2(y_off, y_al) < 1e-6


def test_tensor_core_matches_fp32_path(cuda):
    A, F, T, B, R, I = 28, 8, 2048, 16, 4, 4
    x, w = make(A, F, T, B, 3)
    xd, wd = dev(x), c64(w)
    lib = _lib.load()
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    o1 = torch.zeros((B, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    o2 = torch.zeros_like(o1)
    call("blade_beamform_tc_prepare", ptr(wd), ptr(plan), B, A, F, 2, stream())
    call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(o1), B, A, F, T, 2, R, I, stream())
    call("blade_beamform_detect_f32", _lib.CI8, ptr(xd), ptr(wd), ptr(o2), B, A, F, T, 2, R, I, stream())
    assert rel_l2(host(o1), host(o2)) < 2 * TOL


def test_unfused_module_chain_matches_fused(cuda):
    # Cast -> Beamformer -> Channelizer -> Detector as four modules (the reference's
    # ModeB order) equals the fused kernels.
    A, F, T, B, R, I = 20, 6, 1024, 8, 4, 4
    x, w = make(A, F, T, B, 4)
    xd = bl.array_tensor((A, F, T, 2), dtype=bl.ci8)
    xd.as_torch().copy_(dev(x))
    wd = bl.phasor_tensor((B, A, F, 1, 2), dtype=bl.cf32)
    wd.as_torch().copy_(c64(w))
    cast = bl.module(bl.cast, {}, xd, it=bl.ci8, ot=bl.cf32)
    bf = bl.module(bl.beamformer, {}, (cast.get_output(), wd), telescope=bl.ata)
    ch = bl.module(bl.channelizer, {"rate": R}, bf.get_output())
    det = bl.module(bl.detector, {"integration_size": I, "number_of_output_polarizations": 1}, ch.get_output())
    for m in (cast, bf, ch, det):
        assert m.process(0) == bl.result.success
    fused = bl.module(bl.beamform_detect, {"rate": R, "integration_size": I}, (xd, wd), telescope=bl.ata)
    fused.process(0)
    torch.cuda.synchronize()
    ref = O.beamform_channelize_detect(x, w, R, I)
    assert rel_l2(det.get_output().as_torch().cpu().numpy(), ref) < TOL
    assert rel_l2(fused.get_output().as_torch().cpu().numpy(), ref) < TOL
    assert fused.precision == "fp16_split"


# ------------------------------------------------------------------------ adjoint
@pytest.mark.parametrize("A,F,T,B", [(28, 6, 2048, 1), (7, 3, 300, 3), (16, 2, 512, 20)])
def test_adjoint_gradient_vs_fp64(cuda, A, F, T, B):
    rng = np.random.default_rng(A + B)
    x, _ = S.calibration_voltages(rng, A, F, T)
    w = (rng.standard_normal((B, A, F, 1, 2)) + 1j * rng.standard_normal((B, A, F, 1, 2))) / np.sqrt(A)
    xd, wd = c64(x), c64(w)
    gd = torch.zeros((B, A, F, 1, 2), dtype=torch.complex64, device="cuda")
    ld = torch.zeros(1, dtype=torch.float64, device="cuda")
    call("blade_beamform_detect_adjoint", ptr(xd), ptr(wd), ptr(gd), ptr(ld), B, A, F, T, 2, stream())
    x32, w32 = x.astype(np.complex64), w.astype(np.complex64)
    g_ref = O.stokes_loss_grad(x32, w32)
    assert rel_l2(host(gd), g_ref) < TOL
    assert abs(host(ld)[0] - O.stokes_loss(x32, w32)) / abs(O.stokes_loss(x32, w32)) < TOL


@pytest.mark.parametrize("A,F,T,B,P", [(9, 4, 640, 2, 1), (40, 2, 256, 40, 2)])
def test_adjoint_general_path_vs_fp64(cuda, A, F, T, B, P):
    # one polarisation, and B x A above the main path's pair limit, take the
    # one-CTA-per-(f, p) kernel; same gradient and scalar loss
    rng = np.random.default_rng(A * B + P)
    x = (rng.standard_normal((A, F, T, P)) + 1j * rng.standard_normal((A, F, T, P))).astype(np.complex64)
    w = ((rng.standard_normal((B, A, F, 1, P)) + 1j * rng.standard_normal((B, A, F, 1, P))) / np.sqrt(A)).astype(
        np.complex64)
    gd = torch.zeros((B, A, F, 1, P), dtype=torch.complex64, device="cuda")
    ld = torch.zeros(1, dtype=torch.float64, device="cuda")
    xd, wd = c64(x), c64(w)  # keep the device copies alive until the kernels have run
    call("blade_beamform_detect_adjoint", ptr(xd), ptr(wd), ptr(gd), ptr(ld), B, A, F, T, P, stream())
    assert rel_l2(host(gd), O.stokes_loss_grad(x, w)) < TOL
    assert abs(host(ld)[0] - O.stokes_loss(x, w)) / abs(O.stokes_loss(x, w)) < TOL


def test_bounded_wait_expiry_is_reported_and_the_context_survives(cuda):
    # A wait that nothing completes gives up after its budget (2e6 cycles, about a
    # millisecond), records its code in the status word and returns; the status is
    # read once and cleared, and the tensor-core chain then runs normally.
    assert bl.device_status() == 0
    call("blade_wait_selftest", 2_000_000, stream())
    torch.cuda.synchronize()
    assert bl.device_status() == 0x20
    assert bl.device_status() == 0
    A, F, T, B, R, I = 28, 2, 1024, 16, 4, 4
    x, w = make(A, F, T, B, 11)
    xd, wd = dev(x), c64(w)
    plan = torch.empty(int(_lib.load().blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    od = torch.zeros((B, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    call("blade_beamform_prepare_detect_tc", ptr(wd), ptr(plan), ptr(xd), ptr(od), B, A, F, T, 2, R, I, stream())
    assert rel_l2(host(od), O.beamform_channelize_detect(x, w, R, I)) < TOL
    assert bl.device_status() == 0


def test_wait_selftest_rejects_bad_budgets(cuda):
    with pytest.raises(_lib.BladeError):
        call("blade_wait_selftest", 0, stream())
    with pytest.raises(_lib.BladeError):
        call("blade_wait_selftest", 10**11, stream())
