"""Literal loop-order restatements of the reference kernels, for small cases.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  These walk the same
index arithmetic as the reference CUDA kernels, one output element at a time, and
are used to cross-check the vectorised ``oracle.formulas`` on tiny shapes.
"""

from __future__ import annotations

import cmath
import math

import numpy as np


def beamform(x, w, incoherent=False, incoherent_sqrt=False):
    """``src/modules/beamformer/beamformer.cu:13-79``: per (ch, t) thread, phasor
    cache [b][a][p], accumulate ``acc[p] += x[a][p] * phr[b][a][p]`` over a."""
    A, F, T, P = x.shape
    B = w.shape[0]
    out = np.zeros((B + (1 if incoherent else 0), F, T, P), dtype=np.complex128)
    for ch in range(F):
        for t in range(T):
            for b in range(B):
                for p in range(P):
                    acc = 0j
                    for a in range(A):
                        acc += complex(x[a, ch, t, p]) * complex(w[b, a, ch, 0, p])
                    out[b, ch, t, p] = acc
            if incoherent:
                for p in range(P):
                    acc = 0.0
                    for a in range(A):
                        v = complex(x[a, ch, t, p]) * complex(w[0, a, ch, 0, p])
                        acc += v.real * v.real + v.imag * v.imag
                    out[B, ch, t, p] = math.sqrt(acc) if incoherent_sqrt else acc
    return out


def detect(x, integration, npols):
    """``src/modules/detector/detector.cu:7-51``: sample tid = ((a F + f) T + t),
    output index tid / INTG, products accumulated per window."""
    A, F, T, P = x.shape
    N = A * F * T
    flat = x.reshape(N, P)
    out = np.zeros((N // integration, npols), dtype=np.float64)
    for tid in range(N):
        X = complex(flat[tid, 0])
        Y = complex(flat[tid, 1])
        o = tid // integration
        if npols == 4:
            out[o, 0] += (X * X.conjugate()).real
            out[o, 1] += (Y * Y.conjugate()).real
            z = X * Y.conjugate()
            out[o, 2] += z.real
            out[o, 3] += z.imag
        else:
            out[o, 0] += X.real * X.real + X.imag * X.imag + Y.real * Y.real + Y.imag * Y.imag
    return out.reshape(A, F, T // integration, npols)


def channelize(x, rate):
    """``src/modules/channelizer/channelizer.cu:5-19`` (negate odd t) followed by a
    forward DFT of length ``rate`` per (a, f, spectrum, p), laid out as the test
    oracle ``tests/modules/channelizer/advanced.py:60-65`` places it."""
    A, F, T, P = x.shape
    C = rate
    S = T // C
    out = np.zeros((A, F * C, S, P), dtype=np.complex128)
    for a in range(A):
        for f in range(F):
            for p in range(P):
                for s in range(S):
                    seg = [complex(x[a, f, s * C + j, p]) * (-1 if (s * C + j) % 2 else 1)
                           for j in range(C)]
                    for k in range(C):
                        acc = 0j
                        for j in range(C):
                            acc += seg[j] * cmath.exp(-2j * math.pi * j * k / C)
                        out[a, f * C + k, s, p] = acc
    return out


def gather_step(out, inp, axis, step):
    """``src/modules/gather/gather.cu:6-18``: output[shapeToOffset(coords, axis,
    step * in.shape[axis])] = input[tid]."""
    shp = inp.shape
    for idx in np.ndindex(*shp):
        o = list(idx)
        o[axis] += step * shp[axis]
        out[tuple(o)] = inp[idx]
    return out


def permute(x, indexes):
    """``src/modules/permutation/permutation.cu:6-20``."""
    out_shape = tuple(x.shape[i] for i in indexes)
    out = np.zeros(out_shape, dtype=x.dtype)
    for idx in np.ndindex(*x.shape):
        out[tuple(idx[i] for i in indexes)] = x[idx]
    return out
