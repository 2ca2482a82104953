"""GPU: the allocation-free tensor-core entry point.

blade_beamform_detect_tc_noalloc serves streaming callers that size all of their
device memory once at start-up and then must not allocate inside their
fixed-cadence loop (cudaMalloc / cudaFree synchronise the device and take
unbounded time).  It keeps the phasor image in a fixed 8 MiB device array in the
library instead of caller-allocated memory.  These tests call it through the
C ABI and check that it gives, bit for bit, the output of the allocating entry
point it stands for (blade_beamform_prepare_detect_tc with a caller-allocated
image: the same two kernels on the same inputs): on two calls in a row, and on
two calls queued back to back on one stream with no synchronisation between
them (the second call's phasor split rewrites the shared array while the first
call's chain may still be reading it, which stream order must make safe); that
no bounded in-kernel wait expired; and that an image above the 8 MiB limit is
rejected.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one; it also passes alone in a fresh process.
"""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from blade_b200 import _lib, synthetic as S
from tests.gpu_util import c64, dev, host, ptr, stream

pytestmark = pytest.mark.gpu

A, F, T, B, R, I = 28, 192, 1024, 16, 4, 4   # ATA production shape, shorter block
SHAPE = (B, F * R, T // (R * I), 1)


def _inputs(seed):
    rng = np.random.default_rng(seed)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    _, w = S.phasors(rng, B, A, F)
    return dev(x), c64(w)


def _allocating(xd, wd):
    """The allocating entry point with a caller-allocated phasor image."""
    lib = _lib.load()
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
    ref = torch.full(SHAPE, float("nan"), dtype=torch.float32, device="cuda")
    _lib.call("blade_beamform_prepare_detect_tc", ptr(wd), ptr(plan), ptr(xd), ptr(ref), B, A, F, T, 2, R, I,
              stream())
    out = host(ref)
    assert bl.device_status() == 0
    return out


def _noalloc(xd, wd, out):
    _lib.call("blade_beamform_detect_tc_noalloc", ptr(xd), ptr(wd), ptr(out), B, A, F, T, 2, R, I, stream())


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    lib = _lib.load()
    assert lib.blade_beamform_tc_plan_size(B, A, F, 2) <= 8 << 20
    for call in range(2):
        xd, wd = _inputs(100 + call)
        ref = _allocating(xd, wd)
        got = torch.full(SHAPE, float("nan"), dtype=torch.float32, device="cuda")
        _noalloc(xd, wd, got)
        g = host(got)
        assert bl.device_status() == 0
        assert np.isfinite(g).all()
        np.testing.assert_array_equal(g, ref)


def test_noalloc_back_to_back_on_one_stream(cuda):
    (x0, w0), (x1, w1) = _inputs(200), _inputs(201)
    ref0, ref1 = _allocating(x0, w0), _allocating(x1, w1)
    o0 = torch.full(SHAPE, float("nan"), dtype=torch.float32, device="cuda")
    o1 = torch.full(SHAPE, float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    _noalloc(x0, w0, o0)   # no synchronisation between the two calls
    _noalloc(x1, w1, o1)
    g0, g1 = host(o0), host(o1)
    assert bl.device_status() == 0
    np.testing.assert_array_equal(g0, ref0)
    np.testing.assert_array_equal(g1, ref1)


def test_noalloc_rejects_image_above_limit(cuda):
    lib = _lib.load()
    Bb, Ab, Fb, Tb = 64, 64, 256, 256
    assert lib.blade_beamform_tc_plan_size(Bb, Ab, Fb, 2) > 8 << 20
    x = torch.zeros((Ab, Fb, Tb, 2, 2), dtype=torch.int8, device="cuda")
    w = torch.zeros((Bb, Ab, Fb, 1, 2), dtype=torch.complex64, device="cuda")
    o = torch.zeros((Bb, Fb, Tb // 8, 1), dtype=torch.float32, device="cuda")
    st = lib.blade_beamform_detect_tc_noalloc(ptr(x), ptr(w), ptr(o), Bb, Ab, Fb, Tb, 2, 1, 8, stream())
    assert st == _lib.ERROR
    assert "static workspace" in _lib.last_error()
