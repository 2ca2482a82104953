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


def _compile(out):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++20", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "blade_b200", "cpp", "include"), SRC, "-L", LIBDIR, "-lblade_b200",
           "-Xlinker", f"-rpath,{LIBDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_cpp_layer_compiles(tmp_path):
    _compile(str(tmp_path / "test_pipeline"))


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [True, False])
def test_cpp_pipeline_runs(cuda, tmp_path, graphs):
    exe = _compile(str(tmp_path / "test_pipeline"))
    r = subprocess.run([exe] + ([] if graphs else ["--no-graphs"]), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["max_rel_l2_chain_vs_fused"] < 1e-5
