"""CPU: host-side logic of the Python surface (module dispatch, Pipeline CHRONOUS
stepping, Runner queue states) with fake modules, no GPU."""

import pytest

import blade_b200 as bl
from blade_b200.constants import Taint
from blade_b200.modules import Module
from blade_b200.runtime import Runner


class Fake(Module):
    def __init__(self, log, name, ratio=1):
        super().__init__()
        self.log, self._n, self.ratio = log, name, ratio
        self.taint = Taint.CONSUMER | Taint.PRODUCER | (Taint.CHRONOUS if ratio > 1 else Taint.NONE)

    def get_compute_ratio(self):
        return self.ratio

    def process(self, step=0, stream=None):
        self.log.append((self._n, step))
        return bl.result.success


def test_module_dispatch_errors():
    with pytest.raises(ValueError):
        bl.module("beamformer", {}, None)
    with pytest.raises(AttributeError, match="telescopes"):
        bl.module(bl.beamformer, {}, None, telescope=bl.vla)
    with pytest.raises(AttributeError, match="generic telescopes"):
        bl.module(bl.detector, {}, None, telescope=bl.ata)
    with pytest.raises(AttributeError, match="input types"):
        bl.module(bl.detector, {}, None, it=bl.ci8)
    with pytest.raises(AttributeError, match="output types"):
        bl.module(bl.beamformer, {}, None, it=bl.cf32, ot=bl.f16, telescope=bl.ata)
    with pytest.raises(ValueError, match="Config"):
        bl.module(bl.detector, [1, 2], None)


def test_pipeline_chronous_stepping():
    # src/pipeline.cc:89-141: modules after a ratio-R module run on its last sub-step.
    log = []
    r = Runner()
    r.add_module(Fake(log, "a"))
    r.add_module(Fake(log, "gather", ratio=3))
    r.add_module(Fake(log, "b"))
    assert r.compute_steps_per_cycle() == 3
    outs = []
    for _ in range(6):
        outs.append(r.will_output())
        assert r.compute(0) == bl.result.success
    assert outs == [False, False, True, False, False, True]
    # Modules before the first CHRONOUS module see step % ratio, as in the reference.
    assert log[:4] == [("a", 0), ("gather", 0), ("a", 1), ("gather", 1)]
    assert log[4:7] == [("a", 2), ("gather", 2), ("b", 0)]
    assert r.compute_lifetime_cycles() == 2


def test_runner_queue_states():
    # src/runner.cc:17-68
    log = []
    r = Runner()
    r.add_module(Fake(log, "a"))
    got = []
    assert r.dequeue(lambda i, o, d: got.append((i, o, d))) == bl.result.runner_queue_empty
    assert r.enqueue(lambda: None, lambda: None, 1, 10) == bl.result.success
    assert r.enqueue(lambda: None, lambda: None, 2, 20) == bl.result.success
    assert r.enqueue(lambda: None, lambda: None, 3, 30) == bl.result.runner_queue_full
    assert r.dequeue(lambda i, o, d: got.append((i, o, d))) == bl.result.success
    assert r.dequeue(lambda i, o, d: got.append((i, o, d))) == bl.result.success
    assert got == [(1, 10, True), (2, 20, True)]
    assert r.head_index == 0


def test_runner_callback_failure_propagates():
    r = Runner()
    r.add_module(Fake([], "a"))
    assert r.enqueue(lambda: bl.result.error, lambda: None, 0, 0) == bl.result.error


def test_commit_blocks_new_modules():
    r = Runner()
    r.add_module(Fake([], "a"))
    r.compute(0)
    with pytest.raises(RuntimeError, match="commited"):
        r.add_module(Fake([], "b"))


def test_result_soft_bit():
    # Soft errors carry bit 4 (include/blade/macros.hh:31-48).
    for r in (bl.result.runner_queue_full, bl.result.runner_queue_empty, bl.result.runner_queue_none_available,
              bl.result.pipeline_exhausted):
        assert int(r) & (1 << 4)
    for r in (bl.result.error, bl.result.cuda_error, bl.result.assertion_error):
        assert not int(r) & (1 << 4)


def test_modeb_tensor_core_dispatch():
    # which ModeB configurations take the tensor-core path (host logic, no GPU)
    from blade_b200.modules import _ModeBTensorCore as M

    assert M.applies("ci8", 28, 192, 8192, 2, 16, 4, 4, True, 1)
    assert M.applies("ci8", 64, 4, 1024, 2, 200, 2, 32, True, 1)      # several 64-beam chunks
    assert not M.applies("cf32", 28, 192, 8192, 2, 16, 4, 4, True, 1)  # CF32 voltages: module chain
    assert not M.applies("ci8", 28, 192, 8192, 2, 16, 8, 4, True, 1)   # rate 8: module chain
    assert not M.applies("ci8", 28, 192, 8192, 2, 16, 4, 4, False, 1)  # no detector: beams out
    assert not M.applies("ci8", 28, 192, 8192, 2, 16, 4, 4, True, 4)   # four products
    assert not M.applies("ci8", 28, 192, 256, 2, 16, 4, 1, True, 1)    # 64 spectra: not a 128-row tile
    assert not M.applies("ci8", 65, 4, 1024, 2, 16, 4, 1, True, 1)     # more than 64 antennas
