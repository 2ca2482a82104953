"""Differentiable beamform + Stokes-I detect (no reference counterpart).

``stokes_loss(x, w)`` returns L = -sum_{b,f,t,p} |y[b,f,t,p]|^2 with
y = beamform(x, w) (the reference's ATA beamformer arithmetic,
src/modules/beamformer/beamformer.cu:53-62, followed by the Stokes-I detector,
src/modules/detector/detector.cu:34-51; integration windows do not change the
sum).  Forward and backward are one launch of the hand-written adjoint kernel
(blade_beamform_detect_adjoint), which recomputes the beam voltages tile by tile
and never stores them.  PyTorch's complex-gradient convention
(grad = dL/dRe w + i dL/dIm w = 2 dL/d conj(w)) is applied in ``backward``.

``calibrate_phases`` runs gradient ascent on the summed Stokes-I of a boresight
beam over per-antenna phases; ``calibrate_gains`` over unit-norm complex weights,
which recovers both the relative gain magnitudes and the phases: the gain/phase
calibration use of the adjoint.
"""

from __future__ import annotations

import math

import torch

from . import _lib


_ENTRY = {"auto": "blade_beamform_detect_adjoint", "tensor_cores": "blade_beamform_detect_adjoint_tc",
          "fp32": "blade_beamform_detect_adjoint_f32"}


def _adjoint(x: torch.Tensor, w: torch.Tensor, path: str = "auto"):
    if not (x.is_cuda and w.is_cuda):
        raise RuntimeError("stokes_loss needs CUDA tensors")
    if x.dtype != torch.complex64 or w.dtype != torch.complex64:
        raise RuntimeError("stokes_loss takes complex64 voltages [A,F,T,P] and weights [B,A,F,1,P]")
    x = x.contiguous()
    w = w.contiguous()
    A, F, T, P = x.shape
    B = w.shape[0]
    if tuple(w.shape) != (B, A, F, 1, P):
        raise RuntimeError(f"weights shape {tuple(w.shape)} does not match voltages {tuple(x.shape)}")
    grad = torch.empty_like(w)
    loss = torch.empty(1, dtype=torch.float64, device=x.device)
    if path not in _ENTRY:
        raise ValueError(f"path must be one of {sorted(_ENTRY)}")
    _lib.call(_ENTRY[path], x.data_ptr(), w.data_ptr(), grad.data_ptr(), loss.data_ptr(), B, A, F, T, P,
              torch.cuda.current_stream().cuda_stream)
    return loss[0], grad


class StokesLoss(torch.autograd.Function):
    """L(w) = -sum Stokes-I(beamform(x, w)); gradient w.r.t. the complex weights."""

    @staticmethod
    def forward(ctx, x: torch.Tensor, w: torch.Tensor, path: str = "auto"):
        loss, g = _adjoint(x.detach(), w.detach(), path)
        ctx.save_for_backward(g)
        return loss

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        # g = dL/d conj(w); torch wants dL/dRe w + i dL/dIm w = 2 g (L is real).
        return None, (2.0 * grad_out.to(torch.float32)) * g, None


def stokes_loss(x: torch.Tensor, w: torch.Tensor, path: str = "auto") -> torch.Tensor:
    """path: "auto" (tensor cores from 8 beams up where the shape allows, else CUDA
    cores), "tensor_cores" (blade_beamform_detect_adjoint_tc) or "fp32"."""
    return StokesLoss.apply(x, w, path)


def calibrate_phases(x: torch.Tensor, steps: int = 200, lr: float = 0.05, ref: int = 0, path: str = "auto"):
    """Per-antenna phase calibration of a boresight beam by gradient ascent on its
    summed Stokes-I: w[0, a, f, 0, p] = exp(-i theta_a) / sqrt(A), maximise
    sum |y|^2 over theta (Adam).  Returns theta relative to antenna ``ref``,
    wrapped to (-pi, pi]; for voltages g_a exp(i phi_a) s + n_a it converges to
    phi_a - phi_ref."""
    A, F, T, P = x.shape
    theta = torch.zeros(A, dtype=torch.float32, device=x.device, requires_grad=True)
    opt = torch.optim.Adam([theta], lr=lr)
    scale = 1.0 / float(A * F * T * P)
    for _ in range(steps):
        opt.zero_grad()
        w = torch.exp(-1j * theta.to(torch.complex64)) / math.sqrt(A)
        w = w.view(1, A, 1, 1, 1).expand(1, A, F, 1, P).contiguous()
        loss = stokes_loss(x, w, path) * scale  # minimising -S maximises S
        loss.backward()
        opt.step()
    with torch.no_grad():
        rel = theta - theta[ref]
        return torch.remainder(rel + math.pi, 2 * math.pi) - math.pi


def calibrate_gains(x: torch.Tensor, steps: int = 300, lr: float = 0.05, ref: int = 0, path: str = "auto"):
    """Per-antenna gain and phase calibration of a boresight beam by gradient ascent
    on its summed Stokes-I over complex weights of unit norm, w = u / |u| with
    w[0, a, f, 0, p] = w_a (Adam on u).  For voltages v_a = g_a exp(i phi_a) s + n_a
    with equal noise powers the power sum_{f,t,p} |sum_a v_a w_a|^2 is a Rayleigh
    quotient whose maximiser is proportional to conj(g_a exp(i phi_a)), so
    |w_a| / |w_ref| -> |g_a| / |g_ref| and -arg(w_a / w_ref) -> phi_a - phi_ref.
    Returns (gain ratios |g_a| / |g_ref|, phases relative to antenna ``ref``
    wrapped to (-pi, pi])."""
    A, F, T, P = x.shape
    u = torch.ones(A, dtype=torch.complex64, device=x.device, requires_grad=True)
    opt = torch.optim.Adam([u], lr=lr)
    scale = 1.0 / float(F * T * P)
    for _ in range(steps):
        opt.zero_grad()
        wa = u / torch.linalg.vector_norm(u)
        w = wa.view(1, A, 1, 1, 1).expand(1, A, F, 1, P).contiguous()
        loss = stokes_loss(x, w, path) * scale
        loss.backward()
        opt.step()
    with torch.no_grad():
        wa = u / torch.linalg.vector_norm(u)
        gains = wa.abs() / wa[ref].abs()
        rel = -(torch.angle(wa) - torch.angle(wa[ref]))
        return gains, torch.remainder(rel + math.pi, 2 * math.pi) - math.pi
