"""Benchmark of the beamform -> channelize -> detect hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload (the dense beamformer block, seeded synthetic data): A = 64
antennas, B = 64 beams, F = 256 channels, T = 8192 samples, P = 2
polarisations, CI8 voltages (sigma 8, clipped to +-127), phasors
exp(-i 2 pi f tau) with f = 6.0 GHz + 0.5 MHz k, tau ~ U[-5 us, 5 us];
Cast -> Beamformer -> Detector (Stokes-I, integration 8).

One step = one pass of the chain over one block: phasor hi/lo split + the fused
tcgen05 kernel.  value = 4 B A F T P / t in TMAC/s (whole job); the JSON line
also carries the ingest rate, the plain FP32 CUDA-core path on the same block,
the roofline of the dominant kernel (tensor-bound: the FP16-split contraction's
tensor FLOPs against the measured bf16 peak), the CPU baseline (the reference's
numpy formulas, FP64, on a bounded channel sample, which also checks the GPU
Stokes-I of those channels against FP64) and the end-to-end rate through the
public Runner API with host buffers (voltages and delays in, Stokes-I out).

Further legs: the ATA production chain (A = 28, F = 192, T = 8192, B = 16,
Channelizer rate 4, I = 4) on both paths with its HBM roofline; the
high-resolution spectrometer (A = 1, F = 64, T = 2^20, Cast ->
Channelizer(65536) -> Polarizer -> Detector I = 8); the small block's launch
latency eager against one CUDA graph (A = 20, F = 96, T = 256, B = 8); the
forward + adjoint step of the Stokes loss (A = 28, B = 1, F = 192, T = 2048,
CF32); the ATA ModeB bundle in the reference's order; the byte-movement modules
(Gather, Permutation, Duplicate) and the standalone Channelizer on the
reference's own benchmark shapes; --skip-extra leaves them out.

Multi-GPU (torchrun): weak scaling, every rank owns its own 256-channel band
(frequency sharding, no data-path collective); time = max over ranks.
"""

from __future__ import annotations

import os

# The CPU legs (numpy + BLAS) use every host core the process may run on; the
# thread counts are set before numpy loads its BLAS and reported with the numbers.
CORES = len(os.sched_getaffinity(0))
THREAD_VARS = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")
for _v in THREAD_VARS:
    os.environ.setdefault(_v, str(CORES))

import argparse  # noqa: E402
import json  # noqa: E402
import statistics  # noqa: E402
import subprocess  # noqa: E402
import sys  # noqa: E402
import threading  # noqa: E402
import time  # noqa: E402

import numpy as np  # noqa: E402
import torch  # noqa: E402

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DENSE = dict(A=64, F=256, T=8192, P=2, B=64, R=1, I=8)
ATA = dict(A=28, F=192, T=8192, P=2, B=16, R=4, I=4)
SEED = {"dense": 1003, "ata": 1002}
HEAD = DENSE
METRIC = "Beamform+detect TMAC/s & ingest GB/s: FP16-split TC vs FP32 at <=1e-5 rel err"
WORKLOAD_NAME = ("dense beamformer block: A=64 B=64 F=256 T=8192 P=2 CI8, Cast->Beamformer->Detector"
                 "(Stokes-I, I=8)")


def tmac(w):
    return 4.0 * w["B"] * w["A"] * w["F"] * w["T"] * w["P"]


def ingest_bytes(w):
    return w["A"] * w["F"] * w["T"] * w["P"] * 2


def algorithmic_bytes(w):
    # CI8 in + CF32 phasors + F32 Stokes-I out (the fused-chain minimum).
    out = w["B"] * w["F"] * w["R"] * (w["T"] // (w["R"] * w["I"])) * 4
    return ingest_bytes(w) + w["B"] * w["A"] * w["F"] * w["P"] * 8 + out


def split_tensor_flops(w):
    # FP16-split contraction: the hi and the lo phasor products, 2 flop per real MAC.
    return 2.0 * 2.0 * tmac(w)


def bench_config(world):
    """The config dict both arms print (identical for the same world size)."""
    return {"workload": WORKLOAD_NAME,
            "l2": "inputs larger than L2 (537 MB CI8 per block vs 126 MB L2)",
            "parallelism": f"frequency-sharded x{world} (weak)"}


def thread_settings():
    return {"cores": CORES, **{v: os.environ.get(v) for v in THREAD_VARS}}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def load_traffic(name):
    """Per-launch DRAM bytes of a kernel from its committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name)
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
def make_inputs(w, seed):
    """Host CI8 voltages [A, F, T, P, 2] and delays [B, A] (seconds, FP64)."""
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((w["A"], w["F"], w["T"], w["P"], 2), generator=g, dtype=torch.float32) * 8.0
    x = x.round_().clamp_(-127, 127).to(torch.int8)
    tau = (torch.rand((w["B"], w["A"]), generator=g, dtype=torch.float64) * 2 - 1) * 5e-6
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
            ev[0].record(s)
            _lib.call("blade_beamform_detect_tc", x.data_ptr(), plan.data_ptr(), out.data_ptr(), B, A, F, T, P, R, I,
                      sh)
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


def e2e_runner(w, x, tau, steps, warmup, world):
    """End to end through the public Runner API, as a streaming caller uses it:
    per step the H2D copy of the block's CI8 voltages and of the per-block delays
    [B, A] from pinned host memory, the Phasor module (delays -> phasors on the
    device, FP64) and the fused chain, then the D2H copy of the Stokes-I result;
    the two Runner slots overlap copies and compute.  Returns (ms per step, H2D
    bytes, D2H bytes, the last step's output on the host)."""
    import blade_b200 as bl
    from blade_b200.synthetic import DF_HZ, F0_HZ

    B, A, F, T, P, R, I = (w[k] for k in ("B", "A", "F", "T", "P", "R", "I"))

    @bl.runner(graph=True)
    class Chain:
        def __init__(self):
            self.input.buf = bl.array_tensor((A, F, T, P), dtype=bl.ci8)
            self.input.delays = bl.delay_tensor((B, A), dtype=bl.f64)
            self.output.buf = bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32)
            self.module.phasor = bl.module(bl.phasor, {"number_of_beams": B, "number_of_antennas": A,
                                                       "number_of_frequency_channels": F,
                                                       "number_of_polarizations": P,
                                                       "observation_frequency_hz": F0_HZ,
                                                       "channel_bandwidth_hz": DF_HZ, "total_bandwidth_hz": 0.0},
                                           (self.input.delays,), telescope=bl.ata)
            self.module.bd = bl.module(bl.beamform_detect, {"rate": R, "integration_size": I},
                                       (self.input.buf, self.module.phasor.get_phasors()), telescope=bl.ata)

    p = Chain()
    hx = [bl.array_tensor((A, F, T, P), dtype=bl.ci8, device=bl.cpu) for _ in range(2)]
    hd = [bl.delay_tensor((B, A), dtype=bl.f64, device=bl.cpu) for _ in range(2)]
    ho = [bl.array_tensor((B, F * R, T // (R * I), 1), dtype=bl.f32, device=bl.cpu) for _ in range(2)]
    for k in range(2):
        hx[k].as_torch().copy_(x)
        hd[k].as_torch().copy_(tau)
    h2d = hx[0].nbytes + hd[0].nbytes
    d2h = ho[0].nbytes

    def run(n):
        done, k = 0, 0
        while done < n:
            if k < n:
                j = k % 2

                def cin(j=j):
                    p.copy(p.input.buf, hx[j])
                    p.copy(p.input.delays, hd[j])

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
    last = ho[(steps - 1) % 2].as_torch().clone()
    p.runner.release_graphs()
    return max_over_ranks(ms, world), h2d, d2h, last


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

    w = dict(ATA)
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
    A, F, T, P = (ADJ[k] for k in ("A", "F", "T", "P"))
    s = torch.cuda.current_stream()
    sh = s.cuda_stream
    g = torch.Generator(device="cuda").manual_seed(1005)
    x = torch.complex(torch.randn((A, F, T, P), generator=g, device="cuda"),
                      torch.randn((A, F, T, P), generator=g, device="cuda"))
    hbm = load_peaks()[0]

    def timed(entry, B):
        ph = torch.polar(torch.ones((B, A, F, 1, P), device="cuda"),
                         torch.rand((B, A, F, 1, P), generator=g, device="cuda") * 6.283185307)
        grad = torch.empty_like(ph)
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")

        def call():
            _lib.call(entry, x.data_ptr(), ph.data_ptr(), grad.data_ptr(), loss.data_ptr(), B, A, F, T, P, sh)

        for _ in range(warmup):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            call()
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        nbytes = A * F * T * P * 8 + 2 * B * A * F * P * 8
        return {"ms_per_step": round(ms, 4), "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1),
                "frac_of_hbm": round(nbytes / (ms * 1e-3) / 1e9 / hbm, 3),
                "macs_fwd_plus_adj": 2 * 4 * B * A * F * T * P}

    res = {"workload": "A=28 F=192 T=2048 P=2 CF32, Stokes loss + dL/dconj(w); B=1 (the calibration block) and B=16"}
    res.update(timed("blade_beamform_detect_adjoint", 1))  # the default dispatch at B = 1: CUDA cores
    res["b1_tensor_cores"] = timed("blade_beamform_detect_adjoint_tc", 1)
    res["b16_tensor_cores"] = timed("blade_beamform_detect_adjoint_tc", 16)
    res["b16_cuda_cores"] = timed("blade_beamform_detect_adjoint_f32", 16)
    res["b16_speedup_tensor_cores"] = round(res["b16_cuda_cores"]["ms_per_step"] / res["b16_tensor_cores"]["ms_per_step"], 2)
    return res


GATHER_SHAPES = [("ata", (5, 192, 8192, 2)), ("vla", (5, 131072, 1, 2))]
PERMUTATIONS = [("AFTP", (0, 1, 2, 3)), ("ATFP", (0, 2, 1, 3)), ("ATPF", (0, 2, 3, 1))]


def copies(steps, warmup):
    """Byte-movement modules on the reference's own benchmark shapes, CF32:
    Gather axis 2, multiplier 64 of [5, 192, 8192, 2] (ATA) and [5, 131072, 1, 2]
    (VLA) inputs (benchmarks/modules/gather/generic.hh:13-32); Permutation of
    [2, 192, 8192, 2] as AFTP, ATFP, ATPF (benchmarks/modules/permutation/
    generic.hh:11-17); Duplicate of [20, 192, 8192, 2]
    (benchmarks/modules/duplicate/base.hh:19).  GB/s = bytes read + written per
    call / device time per call (CUDA events around back-to-back calls)."""
    from blade_b200 import _lib

    _lib.load()
    hbm = load_peaks()[0]
    s = torch.cuda.current_stream()
    sh = s.cuda_stream

    def timed(fn, nbytes):
        for _ in range(warmup):
            fn(0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for k in range(steps):
            fn(k)
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        gbs = nbytes / (ms * 1e-3) / 1e9
        return {"ms": round(ms, 4), "bytes": nbytes, "gbs": round(gbs, 1), "frac_of_hbm": round(gbs / hbm, 3)}

    res = {"hbm_peak_gbs": hbm}
    mult = 64
    for name, shape in GATHER_SHAPES:
        n = int(np.prod(shape))
        x = torch.randn(n * 2, device="cuda").view(torch.complex64)
        oshape = list(shape)
        oshape[2] *= mult
        y = torch.empty(n * mult, dtype=torch.complex64, device="cuda")
        shp = _lib.u64_array(shape)
        res[f"gather_{name}"] = timed(
            lambda k: _lib.call("blade_gather", 8, x.data_ptr(), y.data_ptr(), shp, 2, mult, k % mult, sh), 16 * n)
        del x, y
    shape = (2, 192, 8192, 2)
    n = int(np.prod(shape))
    x = torch.randn(n * 2, device="cuda").view(torch.complex64)
    y = torch.empty_like(x)
    shp = _lib.u64_array(shape)
    for name, idx in PERMUTATIONS:
        ix = _lib.u64_array(idx)
        res[f"permute_{name}"] = timed(lambda k: _lib.call("blade_permute", 8, x.data_ptr(), y.data_ptr(), shp, ix, sh),
                                       16 * n)
    del x, y
    n = 20 * 192 * 8192 * 2
    x = torch.randn(n * 2, device="cuda").view(torch.complex64)
    y = torch.empty_like(x)
    res["duplicate"] = timed(lambda k: _lib.call("blade_duplicate", x.data_ptr(), y.data_ptr(), 8 * n, sh), 16 * n)
    del x, y
    res["shapes"] = ("gather axis 2 x64 of CF32 [5,192,8192,2] and [5,131072,1,2]; permute CF32 [2,192,8192,2]; "
                     "duplicate CF32 [20,192,8192,2]")
    return res


def channelizer_module(steps, warmup):
    """The standalone Channelizer module, CF32 in and out, one launch per call:
    rate 4 on the ATA beams [16, 192, 8192, 2] (the ATA production chain's
    channelizer as a separate module) and rate 8192 on [16, 192, 8192, 2]
    (benchmarks/modules/channelizer/generic.hh:13-17).  GB/s counts the kernel's
    own reads and writes (input, output, and a workspace round trip where the
    four-step path uses one)."""
    from blade_b200 import _lib

    lib = _lib.load()
    hbm = load_peaks()[0]
    s = torch.cuda.current_stream()
    sh = s.cuda_stream
    A, F, T, P = 16, 192, 8192, 2
    n = A * F * T * P
    x = torch.randn(n * 2, device="cuda").view(torch.complex64)
    res = {"hbm_peak_gbs": hbm}
    for R in (4, 8192):
        y = torch.empty_like(x)
        wsb = int(lib.blade_channelize_workspace_size(A, F, T, P, R))
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")

        def fn():
            _lib.call("blade_channelize", x.data_ptr(), y.data_ptr(), ws.data_ptr() if wsb else None, A, F, T, P, R, sh)

        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        nbytes = (32 if wsb else 16) * n
        gbs = nbytes / (ms * 1e-3) / 1e9
        res[f"rate{R}"] = {"ms": round(ms, 4), "bytes": nbytes, "gbs": round(gbs, 1), "frac_of_hbm": round(gbs / hbm, 3),
                           "workspace": bool(wsb)}
        del y, ws
    res["shape"] = "CF32 [16, 192, 8192, 2]"
    del x
    return res


def cpu_reference_sample(w, x, tau, budget_s):
    """The reference's numpy formulas (FP64 restatement of its test oracles) on the
    first nch channels of the block, nch sized so the run takes about budget_s.
    Returns (Stokes-I of those channels, nch, seconds)."""
    from blade_b200.synthetic import phasors_from_delays
    from oracle import formulas as O

    xn = x.numpy()
    ph = phasors_from_delays(tau.numpy(), w["F"], w["P"])
    t = time.perf_counter()
    O.beamform_channelize_detect(xn[:, :1], ph[:, :, :1], w["R"], w["I"])
    one = max(time.perf_counter() - t, 1e-3)
    nch = int(max(1, min(w["F"], budget_s / one)))
    t = time.perf_counter()
    ref = O.beamform_channelize_detect(xn[:, :nch], ph[:, :, :nch], w["R"], w["I"])
    return ref, nch, time.perf_counter() - t


def cpu_baseline(w, x, tau, outs, budget_s=10.0):
    """CPU baseline on the host cores plus the FP64 check of the GPU Stokes-I
    (each output in `outs`) on the same channel sample."""
    ref, nch, dt = cpu_reference_sample(w, x, tau, budget_s)
    errs = {}
    for name, out in outs.items():
        got = out[:, : nch * w["R"]].cpu().numpy()
        errs[name] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    sample = dict(w, F=nch)
    base = {"value": tmac(sample) / dt / 1e12, "unit": "TMAC/s", "cores": CORES, "kind": "port",
            "threads": thread_settings(),
            "sample": f"{nch} of {w['F']} channels of the block, a per-channel rate (FP64 numpy: matmul beamform, "
                      f"np.fft channelize, reshape-sum detect), {dt:.1f} s"}
    return base, errs, nch


# --------------------------------------------------------------------------- arms
def run_ours(args):
    world, rank, local = dist_setup(args)
    from blade_b200 import _lib

    _lib.load()
    hbm_peak, tc_peak, peak_kind = load_peaks()
    w = HEAD
    stream = torch.cuda.current_stream().cuda_stream
    hx, htau = make_inputs(w, SEED["dense"] + rank)
    x, tau = hx.cuda(), htau.cuda()
    ph = phasors_on_device(tau, w, stream)
    # launch shapes tuned on this device for each timed workload (blade_*_autotune)
    import blade_b200 as bl

    tuning = {}
    for name, wk in (("dense", w), ("ata", ATA)):
        tc = bl.autotune.tensor_core(wk["B"], wk["A"], wk["F"], wk["T"], wk["R"], wk["I"])
        f32 = bl.autotune.fp32(wk["B"], wk["A"], wk["F"], wk["T"], wk["R"], wk["I"])
        tuning[name] = {"tc": {"mode": ["raw ring", "direct loads"][tc["params"][0]], "operand_stages": tc["params"][1],
                               "raw_stages": tc["params"][2], "tiles_per_raw_stage": tc["params"][3],
                               "candidates": tc["params"][4], "candidates_differing": tc["params"][5],
                               "us": round(tc["us"], 1)},
                        "fp32": {"TG": f32["params"][0], "candidates": f32["params"][4],
                                 "candidates_differing": f32["params"][5], "us": round(f32["us"], 1)}}
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms_tc, kern_tc, out_tc, launches = time_path(w, x, ph, "tc", args.steps, args.warmup, world)
        ms_tc_separate = time_path.separate_ms
        f32_steps = max(3, args.steps // 4)
        ms_f32, kern_f32, out_f32, _ = time_path(w, x, ph, "f32", f32_steps, args.warmup, world)
        tc_vs_f32 = float((out_tc - out_f32).norm() / out_f32.norm())
        out_tc_h, out_f32_h = out_tc.cpu(), out_f32.cpu()
        del x, ph, out_tc, out_f32
        torch.cuda.synchronize()
        e2e_ms, h2d, d2h, e2e_out = e2e_runner(w, hx, htau, max(4, min(args.steps, 16)), args.warmup, world)
        e2e_vs_device = float((e2e_out - out_tc_h).norm() / out_tc_h.norm())
        # the ATA production chain (A=28 F=192 T=8192 B=16, rate 4, I=4), both paths
        ax, atau = make_inputs(ATA, SEED["ata"] + rank)
        ax = ax.cuda()
        aph = phasors_on_device(atau.cuda(), ATA, stream)
        ams_tc, akern_tc, aout_tc, _ = time_path(ATA, ax, aph, "tc", args.steps, args.warmup, world)
        ams_tc_separate = time_path.separate_ms
        ams_f32, _, aout_f32, _ = time_path(ATA, ax, aph, "f32", max(3, args.steps // 2), args.warmup, world)
        ata_agree = float((aout_tc - aout_f32).norm() / aout_f32.norm())
        del ax, aph, aout_tc, aout_f32
        torch.cuda.synchronize()
        extra = {}
        if not args.skip_extra and world == 1:
            extra["spectrometer"] = spectrometer(max(3, args.steps // 6), args.warmup)
            extra["small_block_latency"] = small_block_latency(100)
            extra["adjoint"] = adjoint_step(max(5, args.steps // 2), args.warmup)
            extra["modeb"] = modeb_step(max(3, args.steps // 6), args.warmup)
            extra["copies"] = copies(max(5, args.steps // 2), args.warmup)
            extra["channelizer_module"] = channelizer_module(max(5, args.steps // 4), args.warmup)
        torch.cuda.synchronize()
    clocks = clk.summary()
    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    value = world * tmac(w) / (ms_tc * 1e-3) / 1e12
    tflops = split_tensor_flops(w) / (kern_tc * 1e-3) / 1e12
    base, errs, nch = (None, {}, 0)
    if world == 1:
        base, errs, nch = cpu_baseline(w, hx, htau, {"tc": out_tc_h, "f32": out_f32_h})
    a_achieved = algorithmic_bytes(ATA) / (akern_tc * 1e-3) / 1e9
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
        "config": bench_config(world),
        "ingest_gbs": round(world * ingest_bytes(w) / (ms_tc * 1e-3) / 1e9, 2),
        "stokes_rel_err_vs_fp64": errs.get("tc"),
        "fp32_path": {"tmacs": round(world * tmac(w) / (ms_f32 * 1e-3) / 1e12, 4), "ms_per_step": round(ms_f32, 6),
                      "speedup_tc_over_fp32": round(ms_f32 / ms_tc, 3),
                      "stokes_rel_err_vs_fp64": errs.get("f32"), "tc_vs_fp32_rel_l2": tc_vs_f32},
        "fp64_check": f"first {nch} of {w['F']} channels (all beams, all samples) against the FP64 numpy chain",
        "roofline": {"bound": "tensor", "achieved": round(tflops, 1), "peak": tc_peak, "unit": "TFLOP/s",
                     "frac": round(tflops / tc_peak, 4), "traffic": load_traffic("bf_tc_kernel_dense_64x64.md"),
                     "kernel": "bf_tc_kernel<1,3>", "peak_kind": f"{peak_kind} bf16_tflops (burst)",
                     "flops_per_launch": split_tensor_flops(w),
                     "flops_counted": "FP16-split contraction: hi and lo products, 2 flop per real MAC, "
                                      "4 B A F T P real MACs each",
                     "useful_frac": round(0.5 * tflops / tc_peak, 4),
                     "kernel_ms": round(kern_tc, 5), "step_ms_separate_calls": round(ms_tc_separate, 5),
                     "hbm_view": {"algorithmic_bytes_per_launch": algorithmic_bytes(w),
                                  "gbs": round(algorithmic_bytes(w) / (kern_tc * 1e-3) / 1e9, 1),
                                  "frac": round(algorithmic_bytes(w) / (kern_tc * 1e-3) / 1e9 / hbm_peak, 4)}},
        "cpu_baseline": base,
        "e2e": {"value": round(world * tmac(w) / (e2e_ms * 1e-3) / 1e12, 4), "unit": "TMAC/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms, 4),
                "rel_l2_vs_device_path": e2e_vs_device,
                "api": "bl.runner(graph=True): bl.module(bl.phasor) (delays in) + bl.module(bl.beamform_detect), "
                       "enqueue/dequeue with pinned host buffers"},
        "ata_production": {
            "workload": "ATA production chain: A=28 F=192 T=8192 P=2 B=16, Cast->Beamformer->Channelizer(rate 4)"
                        "->Detector(Stokes-I, I=4)",
            "tc_tmacs": round(world * tmac(ATA) / (ams_tc * 1e-3) / 1e12, 4), "tc_ms_per_step": round(ams_tc, 5),
            "fp32_tmacs": round(world * tmac(ATA) / (ams_f32 * 1e-3) / 1e12, 4),
            "speedup_tc_over_fp32": round(ams_f32 / ams_tc, 3), "tc_vs_fp32_rel_l2": ata_agree,
            "ingest_gbs": round(world * ingest_bytes(ATA) / (ams_tc * 1e-3) / 1e9, 2),
            "roofline": {"bound": "hbm", "achieved": round(a_achieved, 1), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(a_achieved / hbm_peak, 4),
                         "traffic": load_traffic("bf_tc_kernel_ata_production.md"), "kernel": "bf_tc_kernel<4,2>",
                         "peak_kind": f"{peak_kind} hbm_gbs (burst)",
                         "algorithmic_bytes_per_launch": algorithmic_bytes(ATA), "kernel_ms": round(akern_tc, 5),
                         "step_ms_separate_calls": round(ams_tc_separate, 5)}},
        "tuning": tuning,
        "gpu_launches": launches * args.steps * 2 + f32_steps * 2,
        "gpu_launches_counted": "headline tc loop (split + chain per step) run twice (fused call, then separate "
                                "calls with events), plus the fp32 loops; warm-up excluded",
        "clocks": clocks,
    }
    line.update(extra)
    print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_reference(args):
    """The reference's CPU formula for the path (its tests' numpy oracles, restated in
    FP64) on the host cores, on the headline block, a bounded channel sample per step."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    w = HEAD
    from blade_b200.synthetic import phasors_from_delays
    from oracle import formulas as O

    hx, htau = make_inputs(w, SEED["dense"])
    x = hx.numpy()
    ph = phasors_from_delays(htau.numpy(), w["F"], w["P"])
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
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded CI8 sigma 8, delays U[-5us,5us]); no dataset",
        "config": bench_config(world),
        "cpu_baseline": {"value": value, "unit": "TMAC/s", "cores": CORES, "kind": "port",
                         "threads": thread_settings(),
                         "sample": f"{nch} of {w['F']} channels per step, a per-channel rate: the reference's numpy "
                                   "test formulas (tests/modules/beamformer/ata.py, detector/single_pol.py) in FP64"},
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
                    help="skip the spectrometer, latency, adjoint, ModeB, copy and channelizer legs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
