"""Seeded synthetic inputs with the value distributions of the five workloads.

* CI8 voltages: real and imaginary parts i.i.d. N(0, sigma = 8), rounded and
  clipped to +-127, stored as int8 [..., 2] (the reference's CI8 layout).
* Phasors: w[b, a, f, 0, p] = exp(-i 2 pi f_k tau_ba), f_k = 6.0 GHz + 0.5 MHz k,
  tau_ba ~ U[-5 us, 5 us]; both polarisations share the value; computed in FP64.
* Calibration voltages: v_a(t) = g_a exp(i phi_a) s(t) + n_a(t), s and n complex
  Gaussian at per-antenna SNR 0 dB, |g_a| ~ U[0.5, 1.5], phi_a ~ U[-pi, pi].

There is no public dataset for this path; these generators stand in for
recorded voltages with the shapes and distributions of the workloads.
"""

from __future__ import annotations

import numpy as np

F0_HZ = 6.0e9
DF_HZ = 0.5e6
TAU_MAX_S = 5e-6


def ci8_voltages(rng: np.random.Generator, shape, sigma: float = 8.0) -> np.ndarray:
    """int8 array of shape (*shape, 2)."""
    v = rng.normal(0.0, sigma, size=tuple(shape) + (2,))
    return np.clip(np.rint(v), -127, 127).astype(np.int8)


def delays(rng: np.random.Generator, B: int, A: int) -> np.ndarray:
    return rng.uniform(-TAU_MAX_S, TAU_MAX_S, size=(B, A))


def phasors_from_delays(tau: np.ndarray, F: int, P: int = 2) -> np.ndarray:
    """complex128 [B, A, F, 1, P], FP64 argument reduction of f * tau in turns."""
    f = F0_HZ + DF_HZ * np.arange(F, dtype=np.float64)
    turns = tau[:, :, None] * f[None, None, :]
    turns = turns - np.rint(turns)
    ph = np.exp(-2j * np.pi * turns)
    return np.repeat(ph[:, :, :, None, None], P, axis=4)


def phasors(rng: np.random.Generator, B: int, A: int, F: int, P: int = 2):
    """(delays [B, A], phasors complex128 [B, A, F, 1, P])."""
    tau = delays(rng, B, A)
    return tau, phasors_from_delays(tau, F, P)


def calibration_voltages(rng: np.random.Generator, A: int, F: int, T: int, P: int = 2):
    """(x complex128 [A, F, T, P], gains complex128 [A]) for the calibration workload."""
    g = rng.uniform(0.5, 1.5, size=A) * np.exp(1j * rng.uniform(-np.pi, np.pi, size=A))
    cn = lambda *s: (rng.normal(size=s) + 1j * rng.normal(size=s)) / np.sqrt(2.0)  # noqa: E731
    s = cn(1, F, T, P)
    n = cn(A, F, T, P)
    x = g[:, None, None, None] * s + n
    return x, g


# Seeds per workload (A F T P B are in WORKLOADS).
SEEDS = {1: 1001, 2: 1002, 3: 1003, 4: 1004, 5: 1005}

WORKLOADS = {
    1: dict(name="ata-small", A=20, F=96, T=256, P=2, B=8, rate=1, integ=4),
    2: dict(name="ata-production", A=28, F=192, T=8192, P=2, B=16, rate=4, integ=4),
    3: dict(name="dense-64x64", A=64, F=256, T=8192, P=2, B=64, rate=1, integ=8),
    4: dict(name="hires-spectrometer", A=1, F=64, T=1 << 20, P=2, B=0, rate=65536, integ=8),
    5: dict(name="calibration-adjoint", A=28, F=192, T=2048, P=2, B=1, rate=1, integ=1),
}
