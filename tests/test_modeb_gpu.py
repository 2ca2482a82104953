"""GPU: the ATA ModeB bundle (bl.modeb, include/blade/bundles/ata/mode_b.hh:17-225)
against the FP64 oracle of its chain (oracle/formulas.py mode_b: Cast ->
Channelizer -> Polarizer -> Beamformer::ATA -> [Detector], the Stokes-I
reduction of tests/bundles/ata/mode_b.py:377-390), through the module API, a
@bl.runner pipeline shaped like the reference's test, and the delays input."""

import numpy as np
import pytest
import torch

import blade_b200 as bl
from oracle import formulas as O
from tests.gpu_util import rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def voltages(it, shape, seed):
    rng = np.random.default_rng(seed)
    if it == "ci8":
        return np.clip(np.rint(rng.standard_normal(tuple(shape) + (2,)) * 8), -127, 127).astype(np.int8)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def unit_phasors(B, A, F, P, seed):
    rng = np.random.default_rng(seed)
    ph = np.exp(2j * np.pi * rng.random((B, A, F, 1, 1)))
    return np.repeat(ph, P, axis=4).astype(np.complex64)


def device_input(it, x):
    buf = bl.array_tensor(x.shape[:4], dtype=bl.ci8 if it == "ci8" else bl.cf32, device=bl.cuda)
    buf.as_torch().copy_(torch.from_numpy(np.ascontiguousarray(x)).cuda())
    return buf


def device_phasors(w):
    ph = bl.phasor_tensor(w.shape, dtype=bl.cf32, device=bl.cuda)
    ph.as_torch().copy_(torch.from_numpy(w).cuda())
    return ph


def run(mod):
    mod.process()
    torch.cuda.synchronize()
    return mod.get_output().as_torch().cpu().numpy()


def config(shape, out_shape, R=1, circular=False, incoherent=False, detector=True, I=1, OP=1):
    return {"input_shape": shape, "output_shape": out_shape, "pre_beamformer_channelizer_rate": R,
            "pre_beamformer_polarizer_convert_to_circular": circular, "beamformer_incoherent_beam": incoherent,
            "detector_enable": detector, "detector_integration_size": I,
            "detector_number_of_output_polarizations": OP}


@pytest.mark.parametrize("it", ["ci8", "cf32"])
@pytest.mark.parametrize("I", [1, 4])
def test_rate1_stokes_i_runs_fused(cuda, it, I):
    A, F, T, P, B = 20, 8, 1024, 2, 2
    x = voltages(it, (A, F, T, P), 11 + I)
    w = unit_phasors(B, A, F, P, 3)
    mod = bl.module(bl.modeb, config((A, F, T, P), (B, F, T // I, 1), I=I),
                    {"buffer": device_input(it, x), "phasors": device_phasors(w)},
                    it=getattr(bl, it), ot=bl.f32, telescope=bl.ata)
    assert mod.fused
    got = run(mod)
    assert rel_l2(got, O.mode_b(x, w, 1, integration=I)) < TOL


@pytest.mark.parametrize("it,R,circular,incoherent,OP,I", [
    ("ci8", 4, True, True, 1, 2),
    ("cf32", 2, False, True, 4, 1),
    ("ci8", 4, False, False, 1, 1),
    ("cf32", 8, True, False, 4, 2),
])
def test_module_chain_matches_oracle(cuda, it, R, circular, incoherent, OP, I):
    A, F, T, P, B = 12, 4, 512, 2, 3
    x = voltages(it, (A, F, T, P), 100 + R)
    w = unit_phasors(B, A, F * R, P, 7)
    nb = B + (1 if incoherent else 0)
    mod = bl.module(bl.modeb, config((A, F, T, P), (nb, F * R, T // (R * I), OP), R, circular, incoherent, True, I, OP),
                    {"buffer": device_input(it, x), "phasors": device_phasors(w)},
                    it=getattr(bl, it), ot=bl.f32, telescope=bl.ata)
    assert not mod.fused
    got = run(mod)
    ref = O.mode_b(x, w, R, circular, incoherent, True, I, OP)
    assert rel_l2(got[:B], ref[:B]) < TOL
    if incoherent:
        assert rel_l2(got[B], ref[B]) < TOL


def test_complex_output_without_detector(cuda):
    A, F, T, P, B, R = 8, 4, 256, 2, 2, 2
    x = voltages("ci8", (A, F, T, P), 5)
    w = unit_phasors(B, A, F * R, P, 9)
    mod = bl.module(bl.modeb, config((A, F, T, P), (B + 1, F * R, T // R, P), R, False, True, False),
                    {"buffer": device_input("ci8", x), "phasors": device_phasors(w)},
                    it=bl.ci8, ot=bl.cf32, telescope=bl.ata)
    got = run(mod)
    ref = O.mode_b(x, w, R, incoherent=True, detector=False)
    assert rel_l2(got[:B], ref[:B]) < TOL
    assert rel_l2(got[B], ref[B]) < TOL  # incoherent beam, not square-rooted without the detector


def test_delays_input_through_the_phasor_stage(cuda):
    A, F, T, P, B, R = 10, 3, 256, 2, 2, 4
    rng = np.random.default_rng(21)
    x = voltages("ci8", (A, F, T, P), 21)
    tau = rng.uniform(-5e-6, 5e-6, (B, A))
    cal = (rng.random((A, F * R, 1, P)) + 1j * rng.random((A, F * R, 1, P))).astype(np.complex128)
    f0, df, bw, start = 6.0e9, 0.5e6 / R, 0.5e6 * F, 3
    d = bl.delay_tensor((B, A), dtype=bl.f64, device=bl.cuda)
    d.as_torch().copy_(torch.from_numpy(tau).cuda())
    cfg = config((A, F, T, P), (B, F * R, T // R, 1), R)
    cfg.update(phasor_observation_frequency_hz=f0, phasor_channel_bandwidth_hz=df, phasor_total_bandwidth_hz=bw,
               phasor_frequency_start_index=start, phasor_antenna_calibrations=cal)
    mod = bl.module(bl.modeb, cfg, {"buffer": device_input("ci8", x), "delays": d}, it=bl.ci8, ot=bl.f32,
                    telescope=bl.ata)
    got = run(mod)
    w = O.phasors_from_delays(tau, cal, f0, df, bw, start)
    assert rel_l2(mod.get_phasors().as_torch().cpu().numpy(), w) < 1e-6
    assert rel_l2(got, O.mode_b(x, w, R)) < TOL


@bl.runner
class ModeBPipeline:
    # the shape of tests/bundles/ata/mode_b.py:12-30
    def __init__(self, in_shape, phasor_shape, out_shape, config):
        self.input.buffer = bl.array_tensor(in_shape, dtype=bl.cf32)
        self.input.phasors = bl.phasor_tensor(phasor_shape, dtype=bl.cf32)
        self.output.buffer = bl.array_tensor(out_shape, dtype=bl.f32)
        self.module.modeb = bl.module(bl.modeb, config, (self.input.buffer, self.input.phasors),
                                      it=bl.cf32, ot=bl.f32, telescope=bl.ata)

    def transfer_in(self, buffer, phasors):
        self.copy(self.input.buffer, buffer)
        self.copy(self.input.phasors, phasors)

    def transfer_out(self, buffer):
        self.copy(self.output.buffer, self.module.modeb.get_output())
        self.copy(buffer, self.output.buffer)


@pytest.mark.parametrize("R", [1, 4])
def test_runner_pipeline_like_reference(cuda, R):
    in_shape, B = (20, 8, 512, 2), 2
    A, F, T, P = in_shape
    pha_shape, out_shape = (B, A, F * R, 1, P), (B, F * R, T // R, 1)
    host_in = bl.array_tensor(in_shape, dtype=bl.cf32, device=bl.cpu)
    host_ph = bl.phasor_tensor(pha_shape, dtype=bl.cf32, device=bl.cpu)
    host_out = bl.array_tensor(out_shape, dtype=bl.f32, device=bl.cpu)
    rng = np.random.default_rng(R)
    np.copyto(host_in.as_numpy(), rng.random(in_shape) + 1j * rng.random(in_shape))
    np.copyto(host_ph.as_numpy(), unit_phasors(B, A, F * R, P, 17))
    pipeline = ModeBPipeline(in_shape, pha_shape, out_shape, config(in_shape, out_shape, R))
    assert pipeline(host_in, host_ph, host_out)
    ref = O.mode_b(host_in.as_numpy(), host_ph.as_numpy(), R)
    assert rel_l2(host_out.as_numpy(), ref) < TOL


def test_rejects_inconsistent_configuration(cuda):
    A, F, T, P, B = 4, 2, 256, 2, 1
    x = device_input("ci8", voltages("ci8", (A, F, T, P), 1))
    ph = device_phasors(unit_phasors(B, A, F, P, 1))
    with pytest.raises(RuntimeError):  # output shape mismatch
        bl.module(bl.modeb, config((A, F, T, P), (B, F, T, 4)), {"buffer": x, "phasors": ph}, it=bl.ci8, ot=bl.f32,
                  telescope=bl.ata)
    with pytest.raises(RuntimeError):  # phasors sized for the coarse channels with rate 4
        bl.module(bl.modeb, config((A, F, T, P), (B, F * 4, T // 4, 1), 4), {"buffer": x, "phasors": ph},
                  it=bl.ci8, ot=bl.f32, telescope=bl.ata)
    with pytest.raises(RuntimeError):  # F32 output needs the detector
        bl.module(bl.modeb, config((A, F, T, P), (B, F, T, P), detector=False), {"buffer": x, "phasors": ph},
                  it=bl.ci8, ot=bl.f32, telescope=bl.ata)
