"""CPU: the C-ABI library loads, exports every entry point include/blade_b200.h
declares, and its host-side validation returns the reference's error codes
without touching a GPU."""

import ctypes
import os
import re

import pytest

from blade_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "blade_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"BLADE_API\s+[\w\s\*]+?\b(blade_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert len(syms) >= 19
    for s in ["blade_cast", "blade_beamform_f32", "blade_channelize", "blade_detect", "blade_beamform_detect_tc",
              "blade_beamform_detect_adjoint", "blade_phasor_from_delays"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
        assert s in _lib.exported_symbols(), f"{s} has no ctypes signature"


def _header_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for ret, name, params in re.findall(r"BLADE_API\s+([\w\s\*]+?)\b(blade_\w+)\s*\(([^)]*)\)\s*;", text, flags=re.S):
        ps = [" ".join(p.split()) for p in params.split(",")]
        out[name] = (" ".join(ret.split()), [p for p in ps if p and p != "void"])
    return out


def _ctype_ok(decl, ct):
    """Whether ctypes type `ct` passes a C parameter (or return) declared as `decl`."""
    if "*" in decl or "[" in decl:
        if decl.startswith("const char"):
            return ct in (ctypes.c_char_p, ctypes.c_void_p)
        return ct is ctypes.c_void_p or (isinstance(ct, type) and issubclass(ct, ctypes._Pointer))
    base = re.sub(r"\s+\w+$", "", decl) if " " in decl else decl
    return {"uint64_t": ctypes.c_uint64, "int": ctypes.c_int, "double": ctypes.c_double,
            "blade_stream_t": ctypes.c_void_p, "uint32_t": ctypes.c_uint32}.get(base) is ct


def test_ctypes_signatures_match_the_header():
    # argument count, integer widths and pointer-versus-value for every entry point,
    # so a reordered or widened C parameter cannot drift silently from the binding
    protos = _header_prototypes()
    assert set(protos) == set(declared_symbols())
    for name, (ret, params) in protos.items():
        res, args = _lib._SIGNATURES[name]
        assert len(args) == len(params), (name, len(args), len(params))
        assert _ctype_ok(ret + (" r" if "*" not in ret else ""), res), (name, ret, res)
        for i, (decl, ct) in enumerate(zip(params, args)):
            assert _ctype_ok(decl, ct), (name, i, decl, ct)


def test_version():
    assert _lib.load().blade_version() == 10000


def _err(name, *args):
    st = getattr(_lib.load(), name)(*args)
    return st, _lib.last_error()


def test_detect_validation():
    st, msg = _err("blade_detect", None, None, 2, 4, 10, 2, 3, 1, None)
    assert st == _lib.ERROR and "divisible" in msg
    st, msg = _err("blade_detect", None, None, 2, 4, 10, 1, 2, 1, None)
    assert st == _lib.ERROR and "two (2)" in msg
    st, msg = _err("blade_detect", None, None, 2, 4, 10, 2, 2, 3, None)
    assert st == _lib.ERROR and "not supported" in msg


@pytest.mark.parametrize("T,P,rate", [(1024, 1, 1025), (1025, 1, 1025), (1025, 4, 1025), (100, 2, 7)])
def test_channelize_rejects_like_reference(T, P, rate):
    # The reference's should_fail cases (tests/modules/channelizer/meson.build:31-57)
    # that stay errors here: odd rate, rate not dividing T, P not in {1, 2}.
    st, msg = _err("blade_channelize", None, None, None, 8, 128, T, P, rate, None)
    assert st == _lib.ERROR


def test_cast_rejects_complex_to_real():
    st, msg = _err("blade_cast", _lib.CF32, _lib.F32, None, None, 10, None)
    assert st == _lib.ERROR and "complex" in msg


def test_gather_and_permute_validation():
    shape = _lib.u64_array([2, 3, 4, 5])
    st, msg = _err("blade_gather", 8, None, None, shape, 4, 2, 0, None)
    assert st == _lib.ERROR and "axis" in msg
    st, msg = _err("blade_gather", 8, None, None, shape, 1, 0, 0, None)
    assert st == _lib.ERROR and "multiplier" in msg
    st, msg = _err("blade_permute", 8, None, None, shape, _lib.u64_array([0, 1, 1, 3]), None)
    assert st == _lib.ERROR and "Repeated" in msg or "repeated" in msg


def test_tc_support_query():
    lib = _lib.load()
    assert lib.blade_beamform_detect_tc_supported(64, 64, 256, 8192, 2, 1, 8) == 1
    assert lib.blade_beamform_detect_tc_supported(16, 28, 192, 8192, 2, 4, 4) == 1
    assert lib.blade_beamform_detect_tc_supported(16, 65, 192, 8192, 2, 4, 4) == 0  # A > 64
    assert lib.blade_beamform_detect_tc_supported(16, 28, 192, 8000, 2, 4, 4) == 0  # T % 128
    assert lib.blade_beamform_detect_tc_supported(16, 28, 192, 8192, 2, 8, 4) == 0  # rate
    assert lib.blade_beamform_detect_tc_supported(16, 28, 192, 8192, 2, 4, 3) == 0  # integration
    # phasor image bytes per channel and 64-beam chunk: NB = beams rounded to 16,
    # KA = 32 or 64; hi/lo stacked along N when NB <= 32: (2 KA / 64) * 1024 * NB,
    # else 1536 * NB (KA = 64) or 1024 * NB (KA = 32).
    assert lib.blade_beamform_tc_plan_size(64, 64, 256, 2) == 256 * 1536 * 64
    assert lib.blade_beamform_tc_plan_size(100, 20, 3, 2) == 2 * 3 * 1024 * 64
    assert lib.blade_beamform_tc_plan_size(16, 28, 192, 2) == 192 * 1024 * 16
    assert lib.blade_beamform_tc_plan_size(32, 40, 5, 2) == 5 * 2 * 1024 * 32


def test_channelize_workspace_size():
    lib = _lib.load()
    assert lib.blade_channelize_workspace_size(1, 64, 1 << 20, 2, 4096) == 0
    assert lib.blade_channelize_workspace_size(1, 64, 1 << 20, 2, 65536) == 64 * (1 << 20) * 2 * 8


def test_spectrometer_validation():
    lib = _lib.load()
    R = 65536
    assert lib.blade_spectrometer_workspace_size(1, 64, 1 << 20, 2, R) == 64 * (1 << 20) * 2 * 8
    assert lib.blade_spectrometer_workspace_size(1, 64, 1 << 20, 2, 4096) == 0
    bad = [
        ((_lib.CF16, _lib.F32, 1, 1, 2 * R, 2, R, 1, 1), "input"),
        ((_lib.CI8, _lib.CF32, 1, 1, 2 * R, 2, R, 1, 1), "output"),
        ((_lib.CI8, _lib.F32, 1, 1, 2 * R, 1, R, 1, 1), "two"),
        ((_lib.CI8, _lib.F32, 1, 1, 2 * 4096, 2, 4096, 1, 1), "65536"),
        ((_lib.CI8, _lib.F32, 1, 1, 3 * R + 1, 2, R, 1, 1), "divisible"),
        ((_lib.CI8, _lib.F32, 1, 1, 32 * R, 2, R, 1, 1), "16 spectra"),
        ((_lib.CI8, _lib.F32, 1, 1, 2 * R, 2, R, 0, 1), "zero"),
        ((_lib.CI8, _lib.F32, 1, 1, 6 * R, 2, R, 4, 1), "integration"),
        ((_lib.CI8, _lib.F32, 1, 1, 2 * R, 2, R, 1, 2), "polarizations"),
    ]
    for (it, ot, A, F, T, P, rate, I, OP), word in bad:
        st, msg = _err("blade_spectrometer", it, None, ot, None, None, A, F, T, P, rate, I, OP, 0, None)
        assert st == _lib.ERROR and word in msg, (word, msg)


def test_modeb_tensor_core_entry_points_validate_on_the_host():
    # rate, T % rate, P and integration checks return before any device work
    for args, word in [((1, 1, 64, 2, 8, 0), "rate"), ((1, 1, 63, 2, 2, 0), "divisible"), ((1, 1, 64, 1, 2, 0), "P")]:
        st, msg = _err("blade_prechannelize_cf16", None, None, *args, None)
        assert st == _lib.ERROR and word in msg, (word, msg)
    st, msg = _err("blade_beamform_detect_tc_cf16", None, None, None, 16, 28, 4, 100, 2, 4, None)
    assert st == _lib.ERROR and "unsupported" in msg  # T % 128
    st, msg = _err("blade_beamform_detect_tc_cf16", None, None, None, 16, 28, 4, 128, 2, 3, None)
    assert st == _lib.ERROR and "unsupported" in msg  # I not a power of two
    for args, word in [((4, 2, 64, 1, 4), "P"), ((4, 2, 64, 2, 3), "integration"), ((4, 2, 64, 2, 64), "integration")]:
        st, msg = _err("blade_incoherent_detect_cf16", None, None, None, *args, None)
        assert st == _lib.ERROR and word in msg, (word, msg)


def test_prepare_detect_tc_validates_on_the_host():
    # shape and buffer checks return before the split or the chain is enqueued
    st, msg = _err("blade_beamform_prepare_detect_tc", None, None, None, None, 16, 28, 4, 100, 2, 4, 4, None)
    assert st == _lib.ERROR and "unsupported" in msg  # T % 128
    st, msg = _err("blade_beamform_prepare_detect_tc", None, None, None, None, 16, 65, 4, 128, 2, 4, 4, None)
    assert st == _lib.ERROR and "unsupported" in msg  # A > 64
    st, msg = _err("blade_beamform_prepare_detect_tc", None, None, None, None, 16, 28, 4, 128, 2, 4, 4, None)
    assert st == _lib.ERROR and "null" in msg
    st, msg = _err("blade_beamform_prepare_detect_tc_cf16", None, None, None, None, 16, 28, 4, 100, 2, 4, None)
    assert st == _lib.ERROR and "unsupported" in msg
    st, msg = _err("blade_beamform_prepare_detect_tc_cf16", None, None, None, None, 16, 28, 4, 128, 2, 4, None)
    assert st == _lib.ERROR and "null" in msg


def test_meerkat_validation():
    st, msg = _err("blade_beamform_meerkat_f32", None, None, None, 2, 4, 3, 16, 3, 0, None)
    assert st == _lib.ERROR and "P must be" in msg
    st, msg = _err("blade_beamform_meerkat_f32", None, None, None, 2, 4, 3, 16, 2, 0, None)
    assert st == _lib.ERROR and "null" in msg
