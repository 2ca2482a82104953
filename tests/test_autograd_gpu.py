"""GPU: the adjoint (tensor-core and CUDA-core paths) as a torch.autograd.Function,
checked against an FP64 reference gradient and FP64 central finite differences,
and used for gain/phase calibration on the calibration workload (A = 28, B = 1,
F = 192, T = 2048, P = 2, v_a = g_a exp(i phi_a) s + n_a at per-antenna SNR 0 dB;
the gain calibration through the tensor-core adjoint)."""

import math

import numpy as np
import pytest
import torch

from blade_b200 import synthetic as S
from blade_b200.autograd import calibrate_gains, calibrate_phases, stokes_loss
from oracle import formulas as O

pytestmark = pytest.mark.gpu


def _case(A, F, T, B, seed):
    rng = np.random.default_rng(seed)
    x, g = S.calibration_voltages(rng, A, F, T)
    w = (rng.standard_normal((B, A, F, 1, 2)) + 1j * rng.standard_normal((B, A, F, 1, 2))) / np.sqrt(A)
    return x.astype(np.complex64), w.astype(np.complex64), g


@pytest.mark.parametrize("path", ["tensor_cores", "fp32", "auto"])
def test_autograd_gradient_matches_fp64_reference(cuda, path):
    x, w, _ = _case(28, 8, 2048, 1, 5)
    xt = torch.from_numpy(x).cuda()
    wt = torch.from_numpy(w).cuda().requires_grad_(True)
    loss = stokes_loss(xt, wt, path)
    loss.backward()
    ref_loss = O.stokes_loss(x, w)
    assert abs(loss.item() - ref_loss) / abs(ref_loss) < 1e-5
    g_ref = 2 * O.stokes_loss_grad(x, w)  # torch convention: dL/dRe w + i dL/dIm w
    got = wt.grad.cpu().numpy()
    assert np.linalg.norm(got - g_ref) / np.linalg.norm(g_ref) < 1e-5


@pytest.mark.parametrize("path", ["tensor_cores", "fp32"])
def test_autograd_matches_fp64_central_differences(cuda, path):
    A, F, T, B = 6, 2, 256, 2
    x, w, _ = _case(A, F, T, B, 6)
    xt = torch.from_numpy(x).cuda()
    wt = torch.from_numpy(w).cuda().requires_grad_(True)
    stokes_loss(xt, wt, path).backward()
    grad = wt.grad.cpu().numpy()
    x64, w64 = x.astype(np.complex128), w.astype(np.complex128)
    h = 1e-5
    rng = np.random.default_rng(0)
    for _ in range(12):
        idx = tuple(int(rng.integers(0, n)) for n in w.shape)
        e = np.zeros_like(w64)
        e[idx] = h
        d_re = (O.stokes_loss(x64, w64 + e) - O.stokes_loss(x64, w64 - e)) / (2 * h)
        d_im = (O.stokes_loss(x64, w64 + 1j * e) - O.stokes_loss(x64, w64 - 1j * e)) / (2 * h)
        fd = complex(d_re, d_im)
        assert abs(grad[idx] - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(grad).max()), (idx, grad[idx], fd)


def test_phase_calibration_recovers_phases(cuda):
    A, F, T = 28, 192, 2048
    rng = np.random.default_rng(S.SEEDS[5])
    x, g = S.calibration_voltages(rng, A, F, T)
    xt = torch.from_numpy(x.astype(np.complex64)).cuda()
    del x
    theta = calibrate_phases(xt, steps=300, lr=0.05).cpu().numpy()
    phi = np.angle(g)
    truth = np.remainder(phi - phi[0] + np.pi, 2 * np.pi) - np.pi
    err = np.degrees(np.abs(np.remainder(theta - truth + np.pi, 2 * np.pi) - np.pi))
    print(f"phase calibration: max error {err.max():.3f} deg, median {np.median(err):.3f} deg")
    assert err.max() < 1.0


def test_gain_calibration_recovers_gains_and_phases(cuda):
    A, F, T = 28, 192, 2048
    rng = np.random.default_rng(S.SEEDS[5])
    x, g = S.calibration_voltages(rng, A, F, T)
    xt = torch.from_numpy(x.astype(np.complex64)).cuda()
    del x
    gains, theta = calibrate_gains(xt, steps=300, lr=0.05, path="tensor_cores")
    gains, theta = gains.cpu().numpy(), theta.cpu().numpy()
    g_rel = np.abs(g) / np.abs(g[0])
    gerr = np.abs(gains - g_rel) / g_rel
    phi = np.angle(g)
    truth = np.remainder(phi - phi[0] + np.pi, 2 * np.pi) - np.pi
    perr = np.degrees(np.abs(np.remainder(theta - truth + np.pi, 2 * np.pi) - np.pi))
    print(f"gain calibration: max gain ratio error {gerr.max():.4f}, max phase error {perr.max():.3f} deg")
    assert gerr.max() < 0.02
    assert perr.max() < 1.0


@pytest.mark.parametrize("A,F,T,B", [(28, 8, 2048, 1), (28, 4, 1024, 16), (32, 3, 128, 32), (5, 2, 384, 3),
                                     (17, 300, 256, 2), (40, 2, 256, 2),
                                     # one beam (registers only): 1 and 32 antennas, ragged samples and chunks
                                     (1, 3, 100, 1), (32, 2, 700, 1), (13, 5, 1536, 1), (40, 2, 256, 1)])
def test_adjoint_paths_match_fp64(cuda, A, F, T, B):
    # _tc: tensor cores (P = 2, A <= 32, B <= 32, T % 128 == 0); _f32: CUDA cores;
    # the plain entry picks tensor cores from 8 beams up where they apply
    from blade_b200 import _lib

    x, w, _ = _case(A, F, T, B, 11)
    xt, wt = torch.from_numpy(x).cuda(), torch.from_numpy(w).cuda()
    g_ref = O.stokes_loss_grad(x, w)
    l_ref = O.stokes_loss(x, w)
    s = torch.cuda.current_stream().cuda_stream
    names = ["blade_beamform_detect_adjoint", "blade_beamform_detect_adjoint_f32"]
    if A <= 32 and B <= 32 and T % 128 == 0:
        names.append("blade_beamform_detect_adjoint_tc")
    for name in names:
        grad = torch.full_like(wt, float("nan"))
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        _lib.call(name, xt.data_ptr(), wt.data_ptr(), grad.data_ptr(), loss.data_ptr(), B, A, F, T, 2, s)
        g = grad.cpu().numpy()
        err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
        print(f"{name} A={A} F={F} T={T} B={B}: gradient rel L2 {err:.2e}, loss rel {abs(loss.item() - l_ref) / abs(l_ref):.2e}")
        assert np.isfinite(g).all()
        assert err < 1e-5
        assert abs(loss.item() - l_ref) / abs(l_ref) < 1e-6
    import blade_b200 as bl

    assert bl.device_status() == 0
