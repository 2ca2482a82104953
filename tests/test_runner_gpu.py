"""GPU: the Python surface used the way the reference's own tests use it
(tests/modules/*/*.py: a @bl.runner Pipeline with transfer_in / transfer_out),
plus the asynchronous Runner queue and CUDA-graph replay."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from oracle import formulas as O
from tests.gpu_util import rel_l2

pytestmark = pytest.mark.gpu


@bl.runner
class BeamformerPipeline:
    def __init__(self, input_shape, phasor_shape, output_shape, config):
        self.input.buf = bl.array_tensor(input_shape, dtype=bl.cf32)
        self.input.phasors = bl.phasor_tensor(phasor_shape, dtype=bl.cf32)
        self.output.buf = bl.array_tensor(output_shape, dtype=bl.cf32)
        inp = (self.input.buf, self.input.phasors)
        self.module.beamformer = bl.module(bl.beamformer, config, inp, telescope=bl.ata)

    def transfer_in(self, buf, phasors):
        self.copy(self.input.buf, buf)
        self.copy(self.input.phasors, phasors)

    def transfer_out(self, buf):
        self.copy(self.output.buf, self.module.beamformer.get_output())
        self.copy(buf, self.output.buf)


def test_beamformer_pipeline_like_reference(cuda):
    # tests/modules/beamformer/ata.py
    input_shape, phasor_shape, output_shape = (2, 192, 512, 2), (1, 2, 192, 1, 2), (2, 192, 512, 2)
    config = {"enable_incoherent_beam": True, "enable_incoherent_beam_sqrt": True}
    host_input = bl.array_tensor(input_shape, dtype=bl.cf32, device=bl.cpu)
    host_phasors = bl.phasor_tensor(phasor_shape, dtype=bl.cf32, device=bl.cpu)
    host_output = bl.array_tensor(output_shape, dtype=bl.cf32, device=bl.cpu)
    rng = np.random.default_rng(0)
    np.copyto(host_input.as_numpy(), rng.random(input_shape) + 1j * rng.random(input_shape))
    np.copyto(host_phasors.as_numpy(), rng.random(phasor_shape) + 1j * rng.random(phasor_shape))
    pipeline = BeamformerPipeline(input_shape, phasor_shape, output_shape, config)
    assert pipeline(host_input, host_phasors, host_output)
    ref = O.beamform(host_input.as_numpy(), host_phasors.as_numpy(), True, True)
    out = host_output.as_numpy()
    assert rel_l2(out[:-1], ref[:-1]) < 1e-5
    assert rel_l2(out[-1], ref[-1]) < 1e-5


@bl.runner
class GatherPipeline:
    def __init__(self, in_shape, out_shape, config):
        self.input.buf = bl.array_tensor(in_shape, dtype=bl.cf32)
        self.output.buf = bl.array_tensor(out_shape, dtype=bl.cf32)
        self.module.gather = bl.module(bl.gather, config, self.input.buf)

    def transfer_in(self, buf):
        self.copy(self.input.buf, buf)

    def transfer_out(self, buf):
        self.copy(self.output.buf, self.module.gather.get_output())
        self.copy(buf, self.output.buf)


@pytest.mark.parametrize("A,F,T,P,axis,m", [(2, 64, 256, 2, 2, 16), (3, 7, 3, 1, 0, 5), (9, 2, 1, 3, 3, 8)])
def test_gather_pipeline_like_reference(cuda, A, F, T, P, axis, m):
    # tests/modules/gather/gather.py: loop until the pipeline outputs.
    in_shape = (A, F, T, P)
    out_shape = list(in_shape)
    out_shape[axis] *= m
    host_input = bl.array_tensor(in_shape, dtype=bl.cf32, device=bl.cpu)
    host_output = bl.array_tensor(tuple(out_shape), dtype=bl.cf32, device=bl.cpu)
    rng = np.random.default_rng(1)
    np.copyto(host_input.as_numpy(), rng.random(in_shape) + 1j * rng.random(in_shape))
    pipeline = GatherPipeline(in_shape, tuple(out_shape), {"axis": axis, "multiplier": m})
    n = 0
    while True:
        n += 1
        if pipeline(host_input, host_output):
            break
    assert n == m
    np.testing.assert_array_equal(host_output.as_numpy(),
                                  np.concatenate([host_input.as_numpy()] * m, axis=axis))


@bl.runner
class ChainPipeline:
    """Cast -> Beamformer -> Channelizer -> Detector (+ Polarizer) in the reference's
    module-by-module form."""

    def __init__(self, A, F, T, B, R, I, pol):
        self.input.buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8)
        self.input.phasors = bl.phasor_tensor((B, A, F, 1, 2), dtype=bl.cf32)
        self.output.buf = bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32)
        self.module.cast = bl.module(bl.cast, {}, self.input.buf, it=bl.ci8, ot=bl.cf32)
        self.module.bf = bl.module(bl.beamformer, {}, (self.module.cast.get_output(), self.input.phasors),
                                   telescope=bl.ata)
        self.module.ch = bl.module(bl.channelizer, {"rate": R}, self.module.bf.get_output())
        src = self.module.ch.get_output()
        if pol:
            self.module.pol = bl.module(bl.polarizer, {"inputPolarization": bl.pol.xy,
                                                       "outputPolarization": bl.pol.lr}, src)
            src = self.module.pol.get_output()
        self.module.det = bl.module(bl.detector, {"integration_size": I, "number_of_output_polarizations": 1}, src)

    def transfer_in(self, buf, phasors):
        self.copy(self.input.buf, buf)
        self.copy(self.input.phasors, phasors)

    def transfer_out(self, buf):
        self.copy(self.output.buf, self.module.det.get_output())
        self.copy(buf, self.output.buf)


@pytest.mark.parametrize("pol", [False, True])
def test_module_chain_pipeline(cuda, pol):
    from blade_b200 import synthetic as S

    A, F, T, B, R, I = 16, 8, 1024, 8, 4, 4
    rng = np.random.default_rng(2)
    x = S.ci8_voltages(rng, (A, F, T, 2))
    _, w = S.phasors(rng, B, A, F)
    hx = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cpu)
    hx.as_numpy()[...] = x
    hw = bl.phasor_tensor((B, A, F, 1, 2), dtype=bl.cf32, device=bl.cpu)
    hw.as_numpy()[...] = w
    ho = bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32, device=bl.cpu)
    p = ChainPipeline(A, F, T, B, R, I, pol)
    assert p(hx, hw, ho)
    y = O.channelize(O.beamform(O.ci8_to_complex(x), w), R)
    if pol:
        y = O.polarize(y)
    assert rel_l2(ho.as_numpy(), O.detect(y, I, 1)) < 1e-5


@bl.runner(graph=True)
class FusedPipeline:
    def __init__(self, A, F, T, B, R, I, precision):
        self.input.buf = bl.array_tensor((A, F, T, 2), dtype=bl.ci8)
        self.input.phasors = bl.phasor_tensor((B, A, F, 1, 2), dtype=bl.cf32)
        self.output.buf = bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32)
        self.module.bd = bl.module(bl.beamform_detect, {"rate": R, "integration_size": I, "precision": precision},
                                   (self.input.buf, self.input.phasors), telescope=bl.ata)

    def transfer_in(self, buf, phasors):
        self.copy(self.input.buf, buf)
        self.copy(self.input.phasors, phasors)

    def transfer_out(self, buf):
        self.copy(self.output.buf, self.module.bd.get_output())
        self.copy(buf, self.output.buf)


@pytest.mark.parametrize("precision", ["fp16_split", "fp32"])
def test_async_runner_with_cuda_graphs(cuda, precision):
    """enqueue/dequeue over the two slots for several blocks; the steady state of
    each slot is captured in a CUDA graph after its first eager run."""
    from blade_b200 import synthetic as S

    A, F, T, B, R, I = 28, 8, 1024, 16, 4, 4
    p = FusedPipeline(A, F, T, B, R, I, precision)
    rng = np.random.default_rng(3)
    blocks = []
    for k in range(6):
        x = S.ci8_voltages(rng, (A, F, T, 2))
        _, w = S.phasors(rng, B, A, F)
        hx = bl.array_tensor((A, F, T, 2), dtype=bl.ci8, device=bl.cpu)
        hx.as_numpy()[...] = x
        hw = bl.phasor_tensor((B, A, F, 1, 2), dtype=bl.cf32, device=bl.cpu)
        hw.as_numpy()[...] = w
        ho = bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32, device=bl.cpu)
        blocks.append((x, w.astype(np.complex64), hx, hw, ho))
    done = []
    k = 0
    while len(done) < len(blocks):
        if k < len(blocks):
            _, _, hx, hw, ho = blocks[k]

            def cin(hx=hx, hw=hw):
                p.copy(p.input.buf, hx)
                p.copy(p.input.phasors, hw)

            def cout(ho=ho):
                p.copy(p.output.buf, p.module.bd.get_output())
                p.copy(ho, p.output.buf)

            if p.enqueue(cin, cout, k, k) == bl.result.success:
                k += 1
        p.dequeue(lambda i, o, d: done.append(i))
    assert done == list(range(len(blocks)))
    assert len(p.runner._graphs) == 2
    for x, w, _, _, ho in blocks:
        assert rel_l2(ho.as_numpy(), O.beamform_channelize_detect(x, w, R, I)) < 1e-5
