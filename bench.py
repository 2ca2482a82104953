"""Benchmark of the beamform -> channelize -> detect hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (ATA production chain, seeded synthetic data): A = 28 antennas,
F = 192 channels, T = 8192 samples, P = 2 polarisations, B = 16 beams, CI8
voltages (sigma 8, clipped to +-127), phasors exp(-i 2 pi f tau) with
f = 6.0 GHz + 0.5 MHz k, tau ~ U[-5 us, 5 us]; Cast -> Beamformer ->
Channelizer (rate 4) -> Detector (Stokes-I, integration 4).

One step = one pass of the chain over one block: phasor hi/lo split + the fused
tcgen05 kernel.  value = 4 B A F T P / t in TMAC/s (whole job); the JSON line
also carries the ingest rate, the plain FP32 CUDA-core path on the same block,
the dense 64 x 64 workload (A = B = 64, F = 256, T = 8192, I = 8) for both
paths, the roofline of the dominant kernel, the CPU baseline (the reference's
numpy formulas, FP64, on a bounded channel sample) and the end-to-end rate
through the public Runner API with host buffers.  Three further legs cover the
other measured workloads: the high-resolution spectrometer (A = 1, F = 64,
T = 2^20, Cast -> Channelizer(65536) -> Polarizer -> Detector I = 8), the small
block's launch latency eager against one CUDA graph (A = 20, F = 96, T = 256,
B = 8; also as one fused FP32 launch and as the tensor-core pair), the forward +
adjoint step of the Stokes loss (A = 28, B = 1, F = 192, T = 2048, CF32) and the
ATA ModeB bundle in the reference's order on the production block
(pre-beamformer channelizer, per-fine-channel phasors; the tensor-core path with
and without the incoherent beam, and the module chain);
--skip-extra leaves them out.

Multi-GPU (torchrun): weak scaling, every rank owns its own 192-channel band
(frequency sharding, no data-path collective); time = max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORK = dict(A=28, F=192, T=8192, P=2, B=16, R=4, I=4)
DENSE = dict(A=64, F=256, T=8192, P=2, B=64, R=1, I=8)
METRIC = "Beamform+detect TMAC/s & ingest GB/s: FP16-split TC vs FP32 at <=1e-5 rel err"


def tmac(w):
    return 4.0 * w["B"] * w["A"] * w["F"] * w["T"] * w["P"]


def ingest_bytes(w):
    return w["A"] * w["F"] * w["T"] * w["P"] * 2


def algorithmic_bytes(w):
    # CI8 in + CF32 phasors + F32 Stokes-I out (the fused-chain minimum).
    out = w["B"] * w["F"] * w["R"] * (w["T"] // (w["R"] * w["I"])) * 4
    return ingest_bytes(w) + w["B"] * w["A"] * w["F"] * w["P"] * 8 + out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "bf_tc_kernel_ata_production.md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms in the background."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, index: int):
        self.rows, self.proc = [], None
        try:
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            self.index = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        except Exception:
            self.index = str(index)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        load = [r for r in self.rows if len(r) >= 9 and r[8].isdigit() and int(r[8]) > 0] or self.rows
        sm = [float(r[0]) for r in load if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in load if len(r) > 1 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in load if len(r) >= 8 for i in range(4) if r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(load)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------------------- data
def make_inputs(w, seed, device=True):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((w["A"], w["F"], w["T"], w["P"], 2), generator=g, dtype=torch.float32) * 8.0
    x = x.round_().clamp_(-127, 127).to(torch.int8)
    tau = (torch.rand((w["B"], w["A"]), generator=g, dtype=torch.float64) * 2 - 1) * 5e-6
    if device:
        return x.cuda(), tau.cuda()
    return x, tau


def phasors_on_device(tau, w, stream):
    from blade_b200 import _lib
    from blade_b200.synthetic import DF_HZ, F0_HZ

    ph = torch.empty((w["B"], w["A"], w["F"], 1, w["P"]), dtype=torch.complex64, device="cuda")
    _lib.call("blade_phasor_from_delays", tau.data_ptr(), None, ph.data_ptr(), w["B"], w["A"], w["F"], w["P"],
              F0_HZ, DF_HZ, 0.0, 0, stream)
    return ph


# --------------------------------------------------------------------------- timing
def time_path(w, x, ph, path, steps, warmup, world):
    """Returns (ms per step, ms per launch of the main kernel, output tensor, launches per step)."""
    from blade_b200 import _lib

    lib = _lib.load()
    s = torch.cuda.current_stream()
    sh = s.cuda_stream
    B, A, F, T, P, R, I = (w[k] for k in ("B", "A", "F", "T", "P", "R", "I"))
    out = torch.empty((B, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    plan = None
    if path == "tc":
        plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, P)), dtype=torch.uint8, device="cuda")

    def step(ev=None):
        if path == "tc" and ev is None:  # the split and the chain, the chain a programmatic dependent
            _lib.call("blade_beamform_prepare_detect_tc", ph.data_ptr(), plan.data_ptr(), x.data_ptr(),
                      out.data_ptr(), B, A, F, T, P, R, I, sh)
        elif path == "tc":  # the same two kernels as separate calls, events around the chain
            _lib.call("blade_beamform_tc_prepare", ph.data_ptr(), plan.data_ptr(), B, A, F, P, sh)
            if ev is not None:
                ev[0].record(s)
            _lib.call("blade_beamform_detect_tc", x.data_ptr(), plan.data_ptr(), out.data_ptr(), B, A, F, T, P, R, I,
                      sh)
            if ev is not None:
                ev[1].record(s)
        else:
            if ev is not None:
                ev[0].record(s)
            _lib.call("blade_beamform_detect_f32", _lib.CI8, x.data_ptr(), ph.data_ptr(), out.data_ptr(), B, A, F, T,
                      P, R, I, sh)
            if ev is not None:
                ev[1].record(s)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    # the step as a user enqueues it, nothing between the launches
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s)
    for k in range(steps):
        step()
    t1.record(s)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    total = t0.elapsed_time(t1)
    # then the main kernel's own duration: events on its stream around each launch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    u0, u1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    u0.record(s)
    for k in range(steps):
        step(evs[k])
    u1.record(s)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    kern = sum(a.elapsed_time(b) for a, b in evs) / steps
    time_path.separate_ms = max_over_ranks(u0.elapsed_time(u1) / steps, world)
    launches = 1 + (B + 63) // 64 if path == "tc" else 1
    return max_over_ranks(total / steps, world), kern, out, launches


def e2e_runner(w, steps, warmup, world):
    """End to end through the public Runner API: per step H2D of the block's CI8
    voltages and phasors from pinned host memory, the fused chain, D2H of the
    Stokes-I result; the two Runner slots overlap copies and compute."""
    import blade_b200 as bl

    B, A, F, T, P, R, I = (w[k] for k in ("B", "A", "F", "T", "P", "R", "I"))

    @bl.runner(graph=True)
    class Chain:
        def __init__(self):
            self.input.buf = bl.array_tensor((A, F, T, P), dtype=bl.ci8)
            self.input.phasors = bl.phasor_tensor((B, A, F, 1, P), dtype=bl.cf32)
            self.output.buf = bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32)
            self.module.bd = bl.module(bl.beamform_detect, {"rate": R, "integration_size": I},
                                       (self.input.buf, self.input.phasors), telescope=bl.ata)

    p = Chain()
    x, tau = make_inputs(w, 2002, device=False)
    hx = [bl.array_tensor((A, F, T, P), dtype=bl.ci8, device=bl.cpu) for _ in range(2)]
    hw = [bl.phasor_tensor((B, A, F, 1, P), dtype=bl.cf32, device=bl.cpu) for _ in range(2)]
    ho = [bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32, device=bl.cpu) for _ in range(2)]
    ph = phasors_on_device(tau.cuda(), w, torch.cuda.current_stream().cuda_stream)
    for k in range(2):
        hx[k].as_torch().copy_(x)
        hw[k].as_torch().copy_(ph.cpu())
    torch.cuda.synchronize()
    h2d = hx[0].nbytes + hw[0].nbytes
    d2h = ho[0].nbytes

    def run(n):
        done, k = 0, 0
        while done < n:
            if k < n:
                j = k % 2

                def cin(j=j):
                    p.copy(p.input.buf, hx[j])
                    p.copy(p.input.phasors, hw[j])

                def cout(j=j):
                    p.copy(p.output.buf, p.module.bd.get_output())
                    p.copy(ho[j], p.output.buf)

                if p.enqueue(cin, cout, k, k) == bl.result.success:
                    k += 1
                    continue
            if p.dequeue(lambda i, o, d: None) == bl.result.success:
                done += 1

    run(max(warmup, 3))
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    s0, s1 = p.runner.stream(0), p.runner.stream(1)
    start = torch.cuda.Event(enable_timing=True)
    start.record(s0)
    s1.wait_event(start)
    run(steps)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s0)
    e1.record(s1)
    torch.cuda.synchronize()
    ms = max(start.elapsed_time(e0), start.elapsed_time(e1)) / steps
    barrier(world)
    p.runner.release_graphs()
    return max_over_ranks(ms, world), h2d, d2h


SPECTRO = dict(A=1, F=64, T=1 << 20, P=2, R=65536, I=8)
SMALL = dict(A=20, F=96, T=256, P=2, B=8, R=1, I=4)
ADJ = dict(A=28, F=192, T=2048, P=2, B=1)


def spectrometer(steps, warmup):
    """High-resolution spectrometer on one dual-polarisation stream, module by module:
    Cast<CI8,CF32> -> Channelizer(rate 65536) -> Polarizer -> Detector(Stokes-I, I=8)
    (A=1, F=64, T=2^20, P=2).  Per-kernel device times and GB/s against each kernel's
    own bytes, and the chain's rate against the fused minimum (CI8 in + Stokes-I out)."""
    from blade_b200 import _lib

    lib = _lib.load()
    A, F, T, P, R, I = (SPECTRO[k] for k in ("A", "F", "T", "P", "R", "I"))
    s = torch.cuda.current_stream()
    sh = s.cuda_stream
    g = torch.Generator(device="cuda").manual_seed(1004)
    x = (torch.randn((A, F, T, P, 2), generator=g, device="cuda") * 8).round_().clamp_(-127, 127).to(torch.int8)
    xf = torch.empty((A, F, T, P), dtype=torch.complex64, device="cuda")
    yc = torch.empty((A, F * R, T // R, P), dtype=torch.complex64, device="cuda")
    ws_bytes = int(lib.blade_channelize_workspace_size(A, F, T, P, R))
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    out = torch.empty((A, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    n = A * F * T * P
    kernels = [
        ("cast", lambda: _lib.call("blade_cast", _lib.CI8, _lib.CF32, x.data_ptr(), xf.data_ptr(), n, sh), 2 * n + 8 * n),
        # four-step FFT: input read, workspace written and read back, output written
        ("channelize", lambda: _lib.call("blade_channelize", xf.data_ptr(), yc.data_ptr(),
                                         ws.data_ptr() if ws_bytes else None, A, F, T, P, R, sh),
         (32 if ws_bytes else 16) * n),
        ("polarize", lambda: _lib.call("blade_polarize", _lib.CF32, yc.data_ptr(), yc.data_ptr(), A * F * T, sh), 16 * n),
        ("detect", lambda: _lib.call("blade_detect", yc.data_ptr(), out.data_ptr(), A, F * R, T // R, P, I, 1, sh),
         8 * n + 4 * (n // P) // I),
    ]
    for _ in range(warmup):
        for _, fn, _ in kernels:
            fn()
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(kernels) + 1)] for _ in range(steps)]
    for k in range(steps):
        ev[k][0].record(s)
        for j, (_, fn, _) in enumerate(kernels):
            fn()
            ev[k][j + 1].record(s)
    torch.cuda.synchronize()
    per = [sum(ev[k][j].elapsed_time(ev[k][j + 1]) for k in range(steps)) / steps for j in range(len(kernels))]
    total = sum(per)
    fused_min = 2 * n + 4 * (n // P) // I
    _, _, peak_kind = load_peaks()
    hbm = load_peaks()[0]
    res = {"workload": "A=1 F=64 T=2^20 P=2, Cast->Channelizer(65536)->Polarizer->Detector(Stokes-I, I=8)",
           "ms_per_step": round(total, 4),
           "fused_min_bytes": fused_min,
           "gbs_vs_fused_min": round(fused_min / (total * 1e-3) / 1e9, 1),
           "fft_gflops": round(5 * n * np.log2(R) / (per[1] * 1e-3) / 1e9, 1),
           "kernels": {}}
    for (name, _, nbytes), ms in zip(kernels, per):
        gbs = nbytes / (ms * 1e-3) / 1e9
        res["kernels"][name] = {"ms": round(ms, 4), "bytes": nbytes, "gbs": round(gbs, 1),
                                "frac_of_hbm": round(gbs / hbm, 3)}
    res["hbm_peak_gbs"] = hbm
    # The same block through the fused ModeH path (blade_spectrometer): CI8 in,
    # Stokes-I out, one FP32 workspace round trip.
    del xf, yc
    fws = torch.empty(int(lib.blade_spectrometer_workspace_size(A, F, T, P, R)), dtype=torch.uint8, device="cuda")
    fout = torch.empty_like(out)

    def fused():
        _lib.call("blade_spectrometer", _lib.CI8, x.data_ptr(), _lib.F32, fout.data_ptr(), fws.data_ptr(), A, F, T, P,
                  R, I, 1, 1, sh)

    for _ in range(warmup):
        fused()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        fused()
    e1.record(s)
    torch.cuda.synchronize()
    fms = e0.elapsed_time(e1) / steps
    fbytes = 2 * n + 16 * n + 4 * (n // P) // I  # CI8 in, workspace out + in, Stokes-I out
    res["fused"] = {"api": "blade_spectrometer (ModeH)", "ms_per_step": round(fms, 4),
                    "gbs_vs_fused_min": round(fused_min / (fms * 1e-3) / 1e9, 1),
                    "bytes": fbytes, "gbs": round(fbytes / (fms * 1e-3) / 1e9, 1),
                    "frac_of_hbm": round(fbytes / (fms * 1e-3) / 1e9 / hbm, 3),
                    "speedup_over_module_chain": round(total / fms, 2),
                    "rel_l2_vs_module_chain": float((fout - out).norm() / out.norm())}
    del x, ws, out, fws, fout
    return res


def small_block_latency(calls):
    """Small ATA block (A=20 F=96 T=256 P=2 B=8, I=4): Cast -> Beamformer(FP32) -> Detector,
    three launches per call, eager against one CUDA graph replay; then the same chain
    as one fused FP32 launch and as the tensor-core pair (phasor split + fused kernel).
    Reports the host wall time of one call waited to completion (latency) and the
    device time per call when calls are issued back to back (throughput)."""
    from blade_b200 import _lib

    _lib.load()
    A, F, T, P, B, I = (SMALL[k] for k in ("A", "F", "T", "P", "B", "I"))
    g = torch.Generator(device="cuda").manual_seed(1001)
    x = (torch.randn((A, F, T, P, 2), generator=g, device="cuda") * 8).round_().clamp_(-127, 127).to(torch.int8)
    ph = torch.polar(torch.ones((B, A, F, 1, P), device="cuda"),
                     torch.rand((B, A, F, 1, P), generator=g, device="cuda") * 6.283185307)
    xf = torch.empty((A, F, T, P), dtype=torch.complex64, device="cuda")
    y = torch.empty((B, F, T, P), dtype=torch.complex64, device="cuda")
    out = torch.empty((B, F, T // I, 1), dtype=torch.float32, device="cuda")
    side = torch.cuda.Stream()

    lib = _lib.load()
    plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, P)), dtype=torch.uint8, device="cuda")
    out2 = torch.empty_like(out)

    def call(sh):
        _lib.call("blade_cast", _lib.CI8, _lib.CF32, x.data_ptr(), xf.data_ptr(), A * F * T * P, sh)
        _lib.call("blade_beamform_f32", xf.data_ptr(), ph.data_ptr(), y.data_ptr(), B, A, F, T, P, 0, 0, sh)
        _lib.call("blade_detect", y.data_ptr(), out.data_ptr(), B, F, T, P, I, 1, sh)

    def call_f32(sh):  # the same chain as one fused FP32 launch (CI8 in, Stokes-I out)
        _lib.call("blade_beamform_detect_f32", _lib.CI8, x.data_ptr(), ph.data_ptr(), out2.data_ptr(), B, A, F, T, P,
                  1, I, sh)

    def call_tc(sh):  # phasor split + the tensor-core chain: two launches, one call
        _lib.call("blade_beamform_prepare_detect_tc", ph.data_ptr(), plan.data_ptr(), x.data_ptr(), out2.data_ptr(),
                  B, A, F, T, P, 1, I, sh)

    res = {"workload": "A=20 F=96 T=256 P=2 B=8 I=4, Cast->Beamformer(FP32)->Detector, 3 launches"}
    with torch.cuda.stream(side):
        sh = side.cuda_stream
        for label, fn in (("", call), ("fused_f32_", call_f32), ("fused_tc_", call_tc)):
            for _ in range(10):
                fn(sh)
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=side):
                fn(torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            eager_lat, eager_dev = _measure_calls(lambda: fn(sh), side, calls)
            graph_lat, graph_dev = _measure_calls(graph.replay, side, calls)
            del graph
            res.update({f"{label}eager_us_per_call": round(eager_lat, 2), f"{label}graph_us_per_call": round(graph_lat, 2),
                        f"{label}eager_device_us_per_call": round(eager_dev, 2),
                        f"{label}graph_device_us_per_call": round(graph_dev, 2)})
            if not label:
                res["graph_tmacs"] = round(4 * B * A * F * T * P / (graph_dev * 1e-6) / 1e12, 4)
    res["fused_rel_l2_vs_chain"] = float((out2 - out).norm() / out.norm())
    return res


def _measure_calls(fn, side, calls):
    """Median host wall time of one call waited to completion, and device time per
    call back to back (CUDA events on the launching stream), in microseconds."""
    lat = []
    for _ in range(calls):
        t = time.perf_counter()
        fn()
        side.synchronize()
        lat.append(time.perf_counter() - t)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(side)
    for _ in range(calls):
        fn()
    e1.record(side)
    side.synchronize()
    return float(np.median(lat)) * 1e6, e0.elapsed_time(e1) * 1e3 / calls


def modeb_step(steps, warmup):
    """ATA ModeB in the reference's own order (include/blade/bundles/ata/mode_b.hh:99-199)
    on the production block: Cast -> Channelizer(rate 4) -> Beamformer with per-fine-
    channel phasors -> Detector (Stokes-I, I=4), CI8 in, through bl.module(bl.modeb):
    the tensor-core path (pre-beamformer stages into exact FP16, the tensor-core chain
    on the 768 fine channels, three launches; four with the incoherent beam), against
    the same chain module by module (Cast, Channelizer, Beamformer, Detector)."""
    import blade_b200 as bl
    from blade_b200.modules import BeamformerATA, Cast, Channelizer, Detector

    w = dict(WORK)
    A, F, T, P, B, R, I = (w[k] for k in ("A", "F", "T", "P", "B", "R", "I"))
    g = torch.Generator(device="cuda").manual_seed(1006)
    buf = bl.array_tensor((A, F, T, P), dtype=bl.ci8, device=bl.cuda)
    buf.as_torch().copy_((torch.randn((A, F, T, P, 2), generator=g, device="cuda") * 8).round_().clamp_(-127, 127))
    ph = bl.phasor_tensor((B, A, F * R, 1, P), dtype=bl.cf32, device=bl.cuda)
    ph.as_torch().copy_(torch.polar(torch.ones((B, A, F * R, 1, P), device="cuda"),
                                    torch.rand((B, A, F * R, 1, P), generator=g, device="cuda") * 6.283185307))
    s = torch.cuda.current_stream()

    def timed(process):
        for _ in range(warmup):
            process()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            process()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    res = {"workload": "A=28 F=192 T=8192 P=2 B=16, Cast->Channelizer(4)->Beamformer(fine phasors)"
                       "->Detector(Stokes-I, I=4)"}
    outs = {}
    for label, inc in (("", False), ("incoherent_", True)):
        cfg = {"input_shape": (A, F, T, P), "output_shape": (B + int(inc), F * R, T // (R * I), 1),
               "pre_beamformer_channelizer_rate": R, "beamformer_incoherent_beam": inc, "detector_enable": True,
               "detector_integration_size": I, "detector_number_of_output_polarizations": 1}
        mod = bl.module(bl.modeb, cfg, {"buffer": buf, "phasors": ph}, it=bl.ci8, ot=bl.f32, telescope=bl.ata)
        ms = timed(lambda: mod.process(0, s))
        res[f"{label}path"] = "tensor cores" if mod.tensor_cores else "module chain"
        res[f"{label}ms_per_step"] = round(ms, 4)
        res[f"{label}tmacs"] = round(tmac(w) / (ms * 1e-3) / 1e12, 3)
        outs[label] = mod.get_output().as_torch().clone()
        del mod
    # the same block module by module (with the incoherent beam, square-rooted before the detector)
    cast = Cast(Cast.config(), Cast.input(buf), it="ci8", ot="cf32")
    chan = Channelizer(Channelizer.config(R), Channelizer.input(cast.get_output()))
    bf = BeamformerATA(BeamformerATA.config(True, True), BeamformerATA.input(chan.get_output(), ph))
    det = Detector(Detector.config(I, 1), Detector.input(bf.get_output()))
    chain = [cast, chan, bf, det]
    ms = timed(lambda: [m.process(0, s) for m in chain])
    res["module_chain_ms_per_step"] = round(ms, 4)
    res["module_chain_tmacs"] = round(tmac(w) / (ms * 1e-3) / 1e12, 3)
    ref = det.get_output().as_torch()
    res["tc_vs_module_chain_rel_l2"] = float((outs["incoherent_"] - ref).norm() / ref.norm())
    del buf, ph, outs, chain, cast, chan, bf, det, ref
    return res


def adjoint_step(steps, warmup):
    """Forward + adjoint of the Stokes loss (A=28 B=1 F=192 T=2048 P=2, CF32 voltages):
    one blade_beamform_detect_adjoint call recomputes the beam tile by tile and returns
    the loss and dL/dconj(w); HBM-bound on the 176 MB voltage read."""
    from blade_b200 import _lib

    _lib.load()
    A, F, T, P, B = (ADJ[k] for k in ("A", "F", "T", "P", "B"))
    s = torch.cuda.current_stream()
    sh = s.cuda_stream
    g = torch.Generator(device="cuda").manual_seed(1005)
    x = torch.complex(torch.randn((A, F, T, P), generator=g, device="cuda"),
                      torch.randn((A, F, T, P), generator=g, device="cuda"))
    ph = torch.polar(torch.ones((B, A, F, 1, P), device="cuda"),
                     torch.rand((B, A, F, 1, P), generator=g, device="cuda") * 6.283185307)
    grad = torch.empty_like(ph)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(warmup):
        _lib.call("blade_beamform_detect_adjoint", x.data_ptr(), ph.data_ptr(), grad.data_ptr(), loss.data_ptr(),
                  B, A, F, T, P, sh)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        _lib.call("blade_beamform_detect_adjoint", x.data_ptr(), ph.data_ptr(), grad.data_ptr(), loss.data_ptr(),
                  B, A, F, T, P, sh)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    nbytes = A * F * T * P * 8 + 2 * B * A * F * P * 8
    hbm = load_peaks()[0]
    return {"workload": "A=28 B=1 F=192 T=2048 P=2 CF32, Stokes loss + dL/dconj(w)",
            "ms_per_step": round(ms, 4), "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1),
            "frac_of_hbm": round(nbytes / (ms * 1e-3) / 1e9 / hbm, 3),
            "macs_fwd_plus_adj": 2 * 4 * B * A * F * T * P}


def cpu_baseline(w, out_gpu, budget_s=10.0):
    """The reference's numpy formulas (FP64 oracle restatement) on a bounded
    channel sample of the same block, on every host core; also checks the GPU
    output of those channels against FP64."""
    from oracle import formulas as O

    x, tau = make_inputs(w, 1002, device=False)
    x = x.numpy()
    from blade_b200.synthetic import phasors_from_delays

    ph = phasors_from_delays(tau.numpy(), w["F"], w["P"])
    cores = len(os.sched_getaffinity(0))
    # one channel to size the sample
    t = time.perf_counter()
    O.beamform_channelize_detect(x[:, :1], ph[:, :, :1], w["R"], w["I"])
    one = max(time.perf_counter() - t, 1e-3)
    nch = int(max(1, min(w["F"], budget_s / one)))
    t = time.perf_counter()
    ref = O.beamform_channelize_detect(x[:, :nch], ph[:, :, :nch], w["R"], w["I"])
    dt = time.perf_counter() - t
    sample = dict(w, F=nch)
    err = None
    if out_gpu is not None:
        got = out_gpu[:, : nch * w["R"]].cpu().numpy()
        err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    return {"value": tmac(sample) / dt / 1e12, "unit": "TMAC/s", "cores": cores, "kind": "port",
            "sample": f"{nch} of {w['F']} channels of the block (FP64 numpy: matmul beamform, np.fft channelize, "
                      f"reshape-sum detect), {dt:.1f} s"}, err


# --------------------------------------------------------------------------- arms
def run_ours(args):
    world, rank, local = dist_setup(args)
    from blade_b200 import _lib

    _lib.load()
    hbm_peak, tc_peak, peak_kind = load_peaks()
    w = WORK
    stream = torch.cuda.current_stream().cuda_stream
    x, tau = make_inputs(w, 1002 + rank)
    ph = phasors_on_device(tau, w, stream)
    with ClockSampler(local) as clk:
        ms_tc, kern_tc, out_tc, launches = time_path(w, x, ph, "tc", args.steps, args.warmup, world)
        ms_tc_separate = time_path.separate_ms
        ms_f32, kern_f32, out_f32, _ = time_path(w, x, ph, "f32", args.steps, args.warmup, world)
        e2e_ms, h2d, d2h = e2e_runner(w, max(4, min(args.steps, 20)), args.warmup, world)
        # dense 64 x 64 workload, both paths
        xd, taud = make_inputs(DENSE, 1003 + rank)
        phd = phasors_on_device(taud, DENSE, stream)
        dms_tc, dk_tc, dout_tc, _ = time_path(DENSE, xd, phd, "tc", max(3, args.steps // 4), args.warmup, world)
        dms_f32, dk_f32, dout_f32, _ = time_path(DENSE, xd, phd, "f32", max(3, args.steps // 8), args.warmup, world)
        dense_agree = float((dout_tc - dout_f32).norm() / dout_f32.norm())
        del xd, phd, dout_tc, dout_f32
        torch.cuda.synchronize()
        extra = {}
        if not args.skip_extra and world == 1:
            extra["spectrometer"] = spectrometer(max(3, args.steps // 6), args.warmup)
            extra["small_block_latency"] = small_block_latency(100)
            extra["adjoint"] = adjoint_step(max(5, args.steps // 2), args.warmup)
            extra["modeb"] = modeb_step(max(3, args.steps // 6), args.warmup)
        torch.cuda.synchronize()
    clocks = clk.summary()
    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    value = world * tmac(w) / (ms_tc * 1e-3) / 1e12
    achieved = algorithmic_bytes(w) / (kern_tc * 1e-3) / 1e9
    traffic = load_traffic()
    base, err = cpu_baseline(w, out_tc) if world == 1 else (None, None)
    line = {
        "metric": METRIC,
        "value": round(value, 4),
        "unit": "TMAC/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_tc, 6),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f16 hi+lo split, f32 accumulate",
        "data": "synthetic (seeded CI8 sigma 8, delays U[-5us,5us]); no dataset",
        "config": {"workload": "ATA production chain: A=28 F=192 T=8192 P=2 B=16, Cast->Beamformer->"
                               "Channelizer(rate 4)->Detector(Stokes-I, I=4)",
                   "l2": "inputs larger than L2 (176 MB CI8 per block vs 126 MB L2)",
                   "parallelism": f"frequency-sharded x{world} (weak)"},
        "ingest_gbs": round(world * ingest_bytes(w) / (ms_tc * 1e-3) / 1e9, 2),
        "fp32_path": {"tmacs": round(world * tmac(w) / (ms_f32 * 1e-3) / 1e12, 4), "ms_per_step": round(ms_f32, 6),
                      "speedup_tc_over_fp32": round(ms_f32 / ms_tc, 3)},
        "dense_64x64": {"workload": "A=64 B=64 F=256 T=8192 P=2 rate 1 I=8",
                        "tc_tmacs": round(world * tmac(DENSE) / (dms_tc * 1e-3) / 1e12, 3),
                        "fp32_tmacs": round(world * tmac(DENSE) / (dms_f32 * 1e-3) / 1e12, 3),
                        "speedup_tc_over_fp32": round(dms_f32 / dms_tc, 3),
                        "tc_kernel_ms": round(dk_tc, 4),
                        "tensor_frac_of_measured_bf16": round(2 * tmac(DENSE) / (dk_tc * 1e-3) / 1e12 / tc_peak, 4),
                        "tc_vs_fp32_rel_l2": dense_agree},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                     "frac": round(achieved / hbm_peak, 4), "traffic": traffic,
                     "kernel": "bf_tc_kernel<4>", "peak_kind": f"{peak_kind} hbm_gbs (burst)",
                     "algorithmic_bytes_per_launch": algorithmic_bytes(w), "kernel_ms": round(kern_tc, 5),
                     "step_ms_separate_calls": round(ms_tc_separate, 5)},
        "cpu_baseline": base,
        "stokes_rel_err_vs_fp64": err,
        "e2e": {"value": round(world * tmac(w) / (e2e_ms * 1e-3) / 1e12, 4), "unit": "TMAC/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms, 4),
                "api": "bl.runner(graph=True) + bl.module(bl.beamform_detect) enqueue/dequeue"},
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
    }
    line.update(extra)
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORK
    from oracle import formulas as O
    from blade_b200.synthetic import phasors_from_delays

    x, tau = make_inputs(w, 1002, device=False)
    x = x.numpy()
    ph = phasors_from_delays(tau.numpy(), w["F"], w["P"])
    cores = len(os.sched_getaffinity(0))
    t = time.perf_counter()
    O.beamform_channelize_detect(x[:, :1], ph[:, :, :1], w["R"], w["I"])
    one = max(time.perf_counter() - t, 1e-3)
    nch = int(max(1, min(w["F"], 2.0 / one)))  # ~2 s per step
    sample = dict(w, F=nch)
    for _ in range(args.warmup):
        O.beamform_channelize_detect(x[:, :nch], ph[:, :, :nch], w["R"], w["I"])
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        O.beamform_channelize_detect(x[:, :nch], ph[:, :, :nch], w["R"], w["I"])
        times.append(time.perf_counter() - t)
    ms = 1e3 * sum(times) / len(times)
    value = tmac(sample) / (ms * 1e-3) / 1e12
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "TMAC/s",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded CI8 sigma 8, delays U[-5us,5us]); no dataset",
        "config": {"workload": "ATA production chain: A=28 F=192 T=8192 P=2 B=16, Cast->Beamformer->"
                               "Channelizer(rate 4)->Detector(Stokes-I, I=4)",
                   "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": "TMAC/s", "cores": cores, "kind": "port",
                         "sample": f"{nch} of {w['F']} channels per step: the reference's numpy test formulas "
                                   "(tests/modules/beamformer/ata.py, channelizer/advanced.py, "
                                   "detector/single_pol.py) in FP64"},
        "e2e": {"value": value, "unit": "TMAC/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-extra", action="store_true",
                    help="skip the spectrometer, small-block latency and adjoint legs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
