"""The C++ host layer (blade_b200/cpp/include/blade/*.hh): a BLADE-style program
(Runner + Modules, tests/cpp/test_pipeline.cc) compiles against the headers and
libblade_b200.so on the CPU; on the GPU it streams blocks through the
module-by-module chain and the fused tensor-core module and compares them."""

import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_pipeline.cc")
LIBDIR = os.path.join(ROOT, "blade_b200")


BUNDLES = os.path.join(ROOT, "tests", "cpp", "test_bundles.cc")


def _compile(out, src=SRC):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++20", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "blade_b200", "cpp", "include"), src, "-L", LIBDIR, "-lblade_b200",
           "-Xlinker", f"-rpath,{LIBDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_cpp_layer_compiles(tmp_path):
    _compile(str(tmp_path / "test_pipeline"))
    _compile(str(tmp_path / "test_bundles"), BUNDLES)


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_cpp_pipeline_runs(cuda, tmp_path, graphs):
    exe = _compile(str(tmp_path / "test_pipeline"))
    r = subprocess.run([exe] + ([] if graphs else ["--no-graphs"]), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["max_rel_l2_chain_vs_fused"] < 1e-5


def _read(path, dtype, shape):
    import numpy as np

    return np.fromfile(path, dtype=dtype).reshape(shape)


@pytest.mark.gpu
def test_cpp_bundles_match_oracle(cuda, tmp_path):
    """Bundles::ATA::ModeB and Bundles::Generic::ModeH (blade/bundles.hh) against the
    FP64 oracle of their chains, on the inputs the C++ program generated."""
    import numpy as np

    from oracle import formulas as O

    exe = _compile(str(tmp_path / "test_bundles"), BUNDLES)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    cases = [json.loads(line) for line in r.stdout.strip().splitlines()]
    fused = {d["case"]: d["fused"] for d in cases}
    assert fused == {"modeb_ci8_r4": False, "modeb_cf32_r1": True, "modeb_ci8_beams": False, "modeb_ci8_r4_tc": False,
                     "modeh_ci8_65536": True, "modeh_cf32_1024": False, "meerkat": False}
    assert [d["case"] for d in cases if d["tc"]] == ["modeb_ci8_r4", "modeb_ci8_r4_tc"]

    def rel(a, b):
        return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

    def ci8(name, A, F, T):
        return _read(tmp_path / f"{name}_in.bin", np.int8, (A, F, T, 2, 2))

    def cf32(name, A, F, T):
        return _read(tmp_path / f"{name}_in.bin", np.complex64, (A, F, T, 2))

    # ModeB, CI8, rate 4, circular, incoherent beam, detector I = 2
    x, w = ci8("modeb_ci8_r4", 12, 4, 512), _read(tmp_path / "modeb_ci8_r4_ph.bin", np.complex64, (3, 12, 16, 1, 2))
    got = _read(tmp_path / "modeb_ci8_r4_out.bin", np.float32, (4, 16, 64, 1))
    assert rel(got, O.mode_b(x, w, 4, True, True, True, 2, 1)) < 1e-5
    # ModeB, CI8, rate 4, circular, no incoherent beam: the tensor-core path on the fine channels
    x = ci8("modeb_ci8_r4_tc", 12, 4, 1024)
    w = _read(tmp_path / "modeb_ci8_r4_tc_ph.bin", np.complex64, (3, 12, 16, 1, 2))
    got = _read(tmp_path / "modeb_ci8_r4_tc_out.bin", np.float32, (3, 16, 128, 1))
    assert rel(got, O.mode_b(x, w, 4, True, False, True, 2, 1)) < 1e-5
    # ModeB, CF32, rate 1, Stokes-I: the fused launch
    x, w = cf32("modeb_cf32_r1", 20, 8, 512), _read(tmp_path / "modeb_cf32_r1_ph.bin", np.complex64, (2, 20, 8, 1, 2))
    got = _read(tmp_path / "modeb_cf32_r1_out.bin", np.float32, (2, 8, 128, 1))
    assert rel(got, O.mode_b(x, w, 1, integration=4)) < 1e-5
    # ModeB, CI8 in, CF32 beams (no detector), incoherent beam not square-rooted
    x, w = ci8("modeb_ci8_beams", 8, 4, 256), _read(tmp_path / "modeb_ci8_beams_ph.bin", np.complex64, (2, 8, 8, 1, 2))
    got = _read(tmp_path / "modeb_ci8_beams_out.bin", np.complex64, (3, 8, 128, 2))
    assert rel(got, O.mode_b(x, w, 2, incoherent=True, detector=False)) < 1e-5
    # ModeH at rate 65536: the fused spectrometer, circular, 4 products
    x = ci8("modeh_ci8_65536", 1, 2, 65536)
    got = _read(tmp_path / "modeh_ci8_65536_out.bin", np.float32, (1, 2 * 65536, 1, 4))
    assert rel(got, O.spectrometer(x, 65536, 1, polarizer=True, npols=4)) < 1e-5
    # ModeH at rate 1024 (T): the module chain, linear polarisation
    x = cf32("modeh_cf32_1024", 2, 3, 1024)
    got = _read(tmp_path / "modeh_cf32_1024_out.bin", np.float32, (2, 3 * 1024, 1, 1))
    ref = O.detect(O.channelize(x, 1024), 1, 1)
    assert rel(got, ref) < 1e-5
    # Beamformer::MeerKAT: one weight per (beam, antenna), incoherent beam zero
    x, w = cf32("meerkat", 6, 3, 128), _read(tmp_path / "meerkat_ph.bin", np.complex64, (4, 6, 3, 1, 2))
    got = _read(tmp_path / "meerkat_out.bin", np.complex64, (5, 3, 128, 2))
    ref = O.beamform_meerkat(x, w, 4, incoherent=True)
    assert rel(got[:4], ref[:4]) < 1e-5 and np.all(got[4] == 0)
