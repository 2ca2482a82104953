"""Deterministic inputs of the golden fixtures (shapes match
oracle/ref_kernels/golden_shapes.h).

Values come from a 32-bit linear congruential generator in plain integer
arithmetic, so the inputs can be regenerated bit for bit on any machine without
storing them; only the reference kernels' outputs are committed.
"""

import numpy as np

CAST_SHAPE = (2, 4, 64, 2)          # CI8 [A, F, T, P]
BF = dict(A=20, F=4, T=256, B=8)     # Beamformer::ATA, P = 2, TBLOCK = 256
DET = dict(A=2, F=4, T=512, I=4)     # Detector, P = 2
CH = dict(A=2, F=4, T=256)           # Channelizer rate == T, P = 2


def lcg(n: int, seed: int) -> np.ndarray:
    """n uint32 values of x_{k+1} = 1664525 x_k + 1013904223 (mod 2^32)."""
    out = np.empty(n, dtype=np.uint64)
    x = np.uint64(seed & 0xFFFFFFFF)
    a, c, m = np.uint64(1664525), np.uint64(1013904223), np.uint64(0xFFFFFFFF)
    for i in range(n):
        x = (a * x + c) & m
        out[i] = x
    return out.astype(np.uint32)


def ints(n: int, seed: int, lo: int = -127, hi: int = 127) -> np.ndarray:
    v = lcg(n, seed).astype(np.int64)
    return (lo + (v >> 8) % (hi - lo + 1)).astype(np.int64)


def cast_input() -> np.ndarray:
    n = int(np.prod(CAST_SHAPE)) * 2
    return ints(n, 11, -128, 127).astype(np.int8).reshape(CAST_SHAPE + (2,))


def complex_ints(shape, seed, amp=100) -> np.ndarray:
    n = int(np.prod(shape))
    v = ints(2 * n, seed, -amp, amp).astype(np.float32).reshape(tuple(shape) + (2,))
    return (v[..., 0] + 1j * v[..., 1]).astype(np.complex64)


def unit_phasors(B, A, F, seed) -> np.ndarray:
    u = lcg(B * A, seed).astype(np.float64) / 2.0 ** 32
    tau = (u * 2 - 1).reshape(B, A) * 5e-6
    f = 6.0e9 + 0.5e6 * np.arange(F)
    turns = tau[:, :, None] * f[None, None, :]
    turns -= np.rint(turns)
    ph = np.exp(-2j * np.pi * turns)
    return np.repeat(ph[:, :, :, None, None], 2, axis=4).astype(np.complex64)


def bf_inputs():
    x = complex_ints((BF["A"], BF["F"], BF["T"], 2), 21)
    w = unit_phasors(BF["B"], BF["A"], BF["F"], 22)
    return x, w


def det_input():
    return complex_ints((DET["A"], DET["F"], DET["T"], 2), 31)


def ch_input():
    return complex_ints((CH["A"], CH["F"], CH["T"], 2), 41)


# Byte-movement and polarizer fixtures (the reference's device-only kernels,
# oracle/_ref/ref_*.cubin).  Polarizer inputs have 24-bit fractions, so its sums
# round and bit equality is a real check of the arithmetic.
POL_SHAPE = (2, 4, 64, 2)                      # Polarizer [A, F, T, P], CF32 and CF16
GATHER_CASES = [((2, 3, 8, 2), 2, 4),          # (input shape, axis, multiplier); all widths
                ((2, 3, 8, 2), 1, 3),          # below the reference's 512-element copy
                ((3, 2, 4, 2), 0, 2)]          # threshold, so its accumulate kernel runs
PERM_SHAPE = (2, 3, 5, 2)
PERMS = [(0, 2, 1, 3), (0, 2, 3, 1), (3, 2, 1, 0)]


def complex_frac(shape, seed) -> np.ndarray:
    """complex64 with re, im = k / 2^23 - 1 for 24-bit k (exact in FP32)."""
    n = int(np.prod(shape))
    k = (lcg(2 * n, seed) >> np.uint32(8)).astype(np.float64)
    v = (k / 2.0 ** 23 - 1.0).astype(np.float32).reshape(tuple(shape) + (2,))
    return (v[..., 0] + 1j * v[..., 1]).astype(np.complex64)


def pol_input_cf32() -> np.ndarray:
    return complex_frac(POL_SHAPE, 51)


def pol_input_cf16() -> np.ndarray:
    """float16 [..., 2] (re, im) pairs: the CF16 layout."""
    x = complex_frac(POL_SHAPE, 52)
    return np.stack([x.real, x.imag], axis=-1).astype(np.float16)


def gather_inputs(case: int):
    shape, _, mult = GATHER_CASES[case]
    return [complex_frac(shape, 60 + 10 * case + k) for k in range(mult)]


def perm_input() -> np.ndarray:
    return complex_frac(PERM_SHAPE, 71)
