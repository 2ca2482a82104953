"""Regenerates tests/golden/reference_kernels.npz: the outputs of the reference's own
CUDA kernels (oracle/_ref/libref_kernels.so and the device-only oracle/_ref/ref_*.cubin,
built from the reference sources by oracle/ref_kernels/build.sh) on the
deterministic inputs of golden_inputs.py.

Needs a GPU.  Usage:  python tests/golden/make_golden.py [output.npz]
"""

import ctypes
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import golden_inputs as G  # noqa: E402


def main(out_path):
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_kernels.so"))
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    res = {}

    x = G.cast_input()
    xd = dev(x)
    yd = torch.zeros(x.size, dtype=torch.float32, device="cuda")
    assert lib.ref_cast_ci8_cf32(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(yd.data_ptr())) == 0
    res["cast_ci8_cf32"] = yd.cpu().numpy()

    x, w = G.bf_inputs()
    xd, wd = dev(x), dev(w)
    B, F, T = G.BF["B"], G.BF["F"], G.BF["T"]
    od = torch.zeros((B + 1, F, T, 2), dtype=torch.complex64, device="cuda")
    assert lib.ref_beamformer(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(wd.data_ptr()),
                              ctypes.c_void_p(od.data_ptr())) == 0
    res["beamformer_inc_sqrt"] = od.cpu().numpy()
    od = torch.zeros((B, F, T, 2), dtype=torch.complex64, device="cuda")
    assert lib.ref_beamformer_plain(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(wd.data_ptr()),
                                    ctypes.c_void_p(od.data_ptr())) == 0
    res["beamformer"] = od.cpu().numpy()

    x = G.det_input()
    xd = dev(x)
    A, F, T, I = G.DET["A"], G.DET["F"], G.DET["T"], G.DET["I"]
    o1 = torch.zeros((A, F, T // I, 1), dtype=torch.float32, device="cuda")
    o4 = torch.zeros((A, F, T // I, 4), dtype=torch.float32, device="cuda")
    assert lib.ref_detector(ctypes.c_void_p(xd.data_ptr()), ctypes.c_void_p(o1.data_ptr()),
                            ctypes.c_void_p(o4.data_ptr())) == 0
    res["detector_1pol"] = o1.cpu().numpy()
    res["detector_4pol"] = o4.cpu().numpy()

    x = G.ch_input()
    xd = dev(x)
    assert lib.ref_channelizer(ctypes.c_void_p(xd.data_ptr())) == 0
    A, F, T = G.CH["A"], G.CH["F"], G.CH["T"]
    res["channelizer_rate_T"] = xd.cpu().numpy().reshape(A, F * T, 1, 2)

    # device-only kernels (polarizer, gather's accumulate, permutation), launched
    # with the reference modules' geometry: PadGridSize(input size, 512) x 512
    from oracle.ref_kernels import cubin as RK

    for key, x in (("polarizer_cf32", G.pol_input_cf32()), ("polarizer_cf16", G.pol_input_cf16())):
        k = RK.Kernel(key)
        xd = dev(x)
        v = RK.ref_vector(xd.data_ptr(), G.POL_SHAPE)  # in place: the module links its output to its input
        k.launch(RK.pad_grid(int(np.prod(G.POL_SHAPE)), 512), 512, v, v)
        res[key] = xd.cpu().numpy()

    k = RK.Kernel("gather_cf32")
    for c, (shape, axis, mult) in enumerate(G.GATHER_CASES):
        oshape = list(shape)
        oshape[axis] *= mult
        od = torch.zeros(oshape, dtype=torch.complex64, device="cuda")
        ov = RK.ref_vector(od.data_ptr(), oshape)
        for step, x in enumerate(G.gather_inputs(c)):
            xd = dev(x)
            k.launch(RK.pad_grid(x.size, 512), 512, RK.ref_vector(xd.data_ptr(), shape), ov,
                     ctypes.c_uint64(axis), ctypes.c_uint64(step * shape[axis]))
        res[f"gather_case{c}"] = od.cpu().numpy()

    k = RK.Kernel("permutation_cf32")
    x = G.perm_input()
    xd = dev(x)
    for idx in G.PERMS:
        oshape = [G.PERM_SHAPE[i] for i in idx]
        od = torch.zeros(oshape, dtype=torch.complex64, device="cuda")
        k.launch(RK.pad_grid(x.size, 512), 512, RK.ref_vector(xd.data_ptr(), G.PERM_SHAPE),
                 RK.ref_vector(od.data_ptr(), oshape), RK.ref_shape(idx))
        res["permute_" + "".join(map(str, idx))] = od.cpu().numpy()

    np.savez_compressed(out_path, **res)
    print("wrote", out_path, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_kernels.npz"))
