"""Runs one hot-path kernel on one workload a few times, for profilers.

    python profile_case.py --workload ata-production --path tc --launches 4

Workloads: channelizer-rate4 and channelizer-rate8192 (the Channelizer module on
CF32 [16, 192, 8192, 2], path channelize), ata-small (A=20 F=96 T=256 B=8 rate 1 I=4), ata-production
(A=28 F=192 T=8192 B=16 rate 4 I=4), dense-64x64 (A=64 F=256 T=8192 B=64 rate 1
I=8), spectrometer (A=1 F=64 T=2^20, rate 65536, I=8, no beamformer) and
spectrometer-small (the same with F=16, for full profiler captures), calibration
(A=28 F=192 T=2048 B=1, CF32 voltages; path adjoint: the Stokes loss and its
gradient), modeb (the ATA production block through ModeB in the reference's
order: CF16 pre-channelizer, then the CF16 tensor-core chain on 768 fine
channels).  Paths: tc
(phasor split + tensor-core chain), f32 (fused FP32 chain), modules (Cast ->
Beamformer -> Channelizer -> Detector, one launch each; for the spectrometer
Cast -> Channelizer -> Polarizer -> Detector; path fused: blade_spectrometer).
Inputs are seeded synthetic CI8 voltages and phasors, created on the device.
"""

from __future__ import annotations

import argparse

import torch

from blade_b200 import _lib
from blade_b200.synthetic import DF_HZ, F0_HZ

WORKLOADS = {
    "ata-small": dict(A=20, F=96, T=256, B=8, R=1, I=4),
    "ata-production": dict(A=28, F=192, T=8192, B=16, R=4, I=4),
    "dense-64x64": dict(A=64, F=256, T=8192, B=64, R=1, I=8),
    "spectrometer": dict(A=1, F=64, T=1 << 20, B=0, R=65536, I=8),
    "spectrometer-small": dict(A=1, F=16, T=1 << 20, B=0, R=65536, I=8),
    "calibration": dict(A=28, F=192, T=2048, B=1, R=1, I=1),
    "modeb": dict(A=28, F=192, T=8192, B=16, R=4, I=4),
    # the standalone Channelizer module on CF32 [16, 192, 8192, 2] (path channelize)
    "channelizer-rate4": dict(A=16, F=192, T=8192, B=0, R=4, I=1),
    "channelizer-rate8192": dict(A=16, F=192, T=8192, B=0, R=8192, I=1),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="ata-production", choices=sorted(WORKLOADS))
    ap.add_argument("--path", default="tc", choices=["tc", "f32", "modules", "adjoint", "fused", "channelize"])
    ap.add_argument("--launches", type=int, default=4)
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    A, F, T, B, R, I, P = w["A"], w["F"], w["T"], w["B"], w["R"], w["I"], 2
    lib = _lib.load()
    s = torch.cuda.current_stream().cuda_stream
    g = torch.Generator(device="cuda").manual_seed(7)
    x = (torch.randn((A, F, T, P, 2), generator=g, device="cuda") * 8).round_().clamp_(-127, 127).to(torch.int8)
    if args.workload == "modeb":
        # ModeB in the reference's order on tensor cores: CF16 fine channels, then
        # the per-fine-channel phasor split and the CF16 tensor-core chain
        FR, TR = F * R, T // R
        pre = torch.empty((A, FR, TR, P, 2), dtype=torch.float16, device="cuda")
        ph = torch.polar(torch.ones((B, A, FR, 1, P), device="cuda"),
                         torch.rand((B, A, FR, 1, P), generator=g, device="cuda") * 6.283185307)
        plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, FR, P)), dtype=torch.uint8, device="cuda")
        out = torch.empty((B, FR, TR // I, 1), dtype=torch.float32, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_prechannelize_cf16", x.data_ptr(), pre.data_ptr(), A, F, T, P, R, 0, s)
            _lib.call("blade_beamform_tc_prepare", ph.data_ptr(), plan.data_ptr(), B, A, FR, P, s)
            _lib.call("blade_beamform_detect_tc_cf16", pre.data_ptr(), plan.data_ptr(), out.data_ptr(), B, A, FR, TR,
                      P, I, s)
        torch.cuda.synchronize()
        print(f"modeb tc: {args.launches} launches ok")
        return
    if args.path == "channelize":
        xc = torch.randn((A, F, T, P, 2), generator=g, device="cuda").view(torch.complex64).reshape(A, F, T, P)
        yc = torch.empty_like(xc)
        wsb = int(lib.blade_channelize_workspace_size(A, F, T, P, R))
        ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_channelize", xc.data_ptr(), yc.data_ptr(), ws.data_ptr() if wsb else None, A, F, T, P, R, s)
        torch.cuda.synchronize()
        print(f"{args.workload} channelize: {args.launches} launches ok")
        return
    if args.path == "adjoint":
        xc = torch.complex(torch.randn((A, F, T, P), generator=g, device="cuda"),
                           torch.randn((A, F, T, P), generator=g, device="cuda"))
        wc = torch.polar(torch.ones((B, A, F, 1, P), device="cuda"),
                         torch.rand((B, A, F, 1, P), generator=g, device="cuda") * 6.283185307)
        grad = torch.empty_like(wc)
        loss = torch.empty(1, dtype=torch.float64, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_beamform_detect_adjoint", xc.data_ptr(), wc.data_ptr(), grad.data_ptr(), loss.data_ptr(),
                      B, A, F, T, P, s)
        torch.cuda.synchronize()
        print(f"{args.workload} adjoint: {args.launches} launches ok")
        return
    if args.workload.startswith("spectrometer") and args.path == "fused":
        out = torch.empty((A, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
        ws = torch.empty(int(lib.blade_spectrometer_workspace_size(A, F, T, P, R)), dtype=torch.uint8, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_spectrometer", _lib.CI8, x.data_ptr(), _lib.F32, out.data_ptr(), ws.data_ptr(), A, F, T,
                      P, R, I, 1, 1, s)
        torch.cuda.synchronize()
        print(f"{args.workload} fused: {args.launches} launches ok")
        return
    if args.workload.startswith("spectrometer"):
        xf = torch.empty((A, F, T, P), dtype=torch.complex64, device="cuda")
        yc = torch.empty((A, F * R, T // R, P), dtype=torch.complex64, device="cuda")
        ws = torch.empty(int(lib.blade_channelize_workspace_size(A, F, T, P, R)), dtype=torch.uint8, device="cuda")
        out = torch.empty((A, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_cast", _lib.CI8, _lib.CF32, x.data_ptr(), xf.data_ptr(), A * F * T * P, s)
            _lib.call("blade_channelize", xf.data_ptr(), yc.data_ptr(), ws.data_ptr(), A, F, T, P, R, s)
            _lib.call("blade_polarize", _lib.CF32, yc.data_ptr(), yc.data_ptr(), A * F * T, s)
            _lib.call("blade_detect", yc.data_ptr(), out.data_ptr(), A, F * R, T // R, P, I, 1, s)
        torch.cuda.synchronize()
        print(f"{args.workload} modules: {args.launches} launches ok")
        return
    tau = (torch.rand((B, A), generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * 5e-6
    ph = torch.empty((B, A, F, 1, P), dtype=torch.complex64, device="cuda")
    _lib.call("blade_phasor_from_delays", tau.data_ptr(), None, ph.data_ptr(), B, A, F, P, F0_HZ, DF_HZ, 0.0, 0, s)
    out = torch.empty((B, F * R, T // (R * I), 1), dtype=torch.float32, device="cuda")
    if args.path == "tc":
        plan = torch.empty(int(lib.blade_beamform_tc_plan_size(B, A, F, P)), dtype=torch.uint8, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_beamform_tc_prepare", ph.data_ptr(), plan.data_ptr(), B, A, F, P, s)
            _lib.call("blade_beamform_detect_tc", x.data_ptr(), plan.data_ptr(), out.data_ptr(), B, A, F, T, P, R, I, s)
    elif args.path == "f32":
        for _ in range(args.launches):
            _lib.call("blade_beamform_detect_f32", _lib.CI8, x.data_ptr(), ph.data_ptr(), out.data_ptr(), B, A, F, T,
                      P, R, I, s)
    else:
        xf = torch.empty((A, F, T, P), dtype=torch.complex64, device="cuda")
        y = torch.empty((B, F, T, P), dtype=torch.complex64, device="cuda")
        yc = torch.empty((B, F * R, T // R, P), dtype=torch.complex64, device="cuda")
        for _ in range(args.launches):
            _lib.call("blade_cast", _lib.CI8, _lib.CF32, x.data_ptr(), xf.data_ptr(), A * F * T * P, s)
            _lib.call("blade_beamform_f32", xf.data_ptr(), ph.data_ptr(), y.data_ptr(), B, A, F, T, P, 0, 0, s)
            if R > 1:
                _lib.call("blade_channelize", y.data_ptr(), yc.data_ptr(), None, B, F, T, P, R, s)
            else:
                yc = y
            _lib.call("blade_detect", yc.data_ptr(), out.data_ptr(), B, F * R, T // R, P, I, 1, s)
    torch.cuda.synchronize()
    print(f"{args.workload} {args.path}: {args.launches} launches ok")


if __name__ == "__main__":
    main()
