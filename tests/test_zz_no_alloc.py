"""GPU: the allocation-free tensor-core entry point.

blade_beamform_detect_tc_noalloc serves streaming callers that size all of their
device memory once at start-up and then must not allocate inside their
fixed-cadence loop (cudaMalloc / cudaFree synchronise the device and take
unbounded time).  It keeps the phasor image in a fixed 8 MiB device array in the
library instead of caller-allocated memory.  These tests call it through the
C ABI and check that two calls in a row give the output of the allocating entry
points (blade_beamform_tc_prepare + blade_beamform_detect_tc) on the same
inputs, and that an image above the 8 MiB limit is rejected.

The file name sorts last so that a run stopping at the first failure has run
every other test before this one; it also passes alone in a fresh process.
"""

import numpy as np
import pytest
import torch

from blade_b200 import _lib, synthetic as S
from tests.gpu_util import c64, dev, host, ptr, rel_l2, stream

pytestmark = pytest.mark.gpu


def _inputs(A, F, T, B, seed):
    rng = np.random.default_rng(seed)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    _, w = S.phasors(rng, B, A, F)
    return dev(x), c64(w)


def test_noalloc_matches_allocating_entry_points_twice(cuda):
    A, F, T, B, R, I = 28, 192, 1024, 16, 4, 4   # ATA production shape, shorter block
    lib = _lib.load()
    assert lib.blade_beamform_tc_plan_size(B, A, F, 2) <= 8 << 20
    shape = (B, F * R, T // (R * I), 1)
    for call in range(2):
        xd, wd = _inputs(A, F, T, B, 100 + call)
        plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, 2)), dtype=torch.uint8, device="cuda")
        ref = torch.zeros(shape, dtype=torch.float32, device="cuda")
        _lib.call("blade_beamform_tc_prepare", ptr(wd), ptr(plan), B, A, F, 2, stream())
        _lib.call("blade_beamform_detect_tc", ptr(xd), ptr(plan), ptr(ref), B, A, F, T, 2, R, I, stream())
        got = torch.full(shape, float("nan"), dtype=torch.float32, device="cuda")
        _lib.call("blade_beamform_detect_tc_noalloc", ptr(xd), ptr(wd), ptr(got), B, A, F, T, 2, R, I, stream())
        g, r = host(got), host(ref)
        assert np.isfinite(g).all()
        assert rel_l2(g, r) < 1e-5


def test_noalloc_rejects_image_above_limit(cuda):
    lib = _lib.load()
    B, A, F, T = 64, 64, 256, 256
    assert lib.blade_beamform_tc_plan_size(B, A, F, 2) > 8 << 20
    x = torch.zeros((A, F, T, 2, 2), dtype=torch.int8, device="cuda")
    w = torch.zeros((B, A, F, 1, 2), dtype=torch.complex64, device="cuda")
    o = torch.zeros((B, F, T // 8, 1), dtype=torch.float32, device="cuda")
    st = lib.blade_beamform_detect_tc_noalloc(ptr(x), ptr(w), ptr(o), B, A, F, T, 2, 1, 8, stream())
    assert st == _lib.ERROR
    assert "static workspace" in _lib.last_error()
