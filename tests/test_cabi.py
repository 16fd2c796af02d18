"""CPU checks of the C ABI library: it loads, exports every function include/*.h declares,
and reports failures as status codes without a GPU (no compute calls are made here)."""
import ctypes
import os
import re
import subprocess

import pytest

from seticore_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names.update(re.findall(r"\b(sc_dd_\w+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _capi.lib()
    decl = declared_functions()
    assert decl, "no declarations found"
    for name in decl:
        assert hasattr(lib, name), name
    assert set(decl) == set(_capi.EXPORTED)
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], capture_output=True, text=True).stdout
    for name in decl:
        assert re.search(rf"\bT {name}\b", out), name


def test_version_and_error_strings():
    lib = _capi.lib()
    assert b"seticore" in lib.sc_dd_version()
    assert isinstance(lib.sc_dd_last_error(), bytes)


def test_bad_arguments_are_rejected_without_gpu():
    lib = _capi.lib()
    h = ctypes.c_void_p()
    assert lib.sc_dd_create(1, 1000, 1.0, 1.0, 0, ctypes.byref(h)) == _capi.SC_DD_EINVAL
    assert b"num_timesteps" in lib.sc_dd_last_error()
    assert lib.sc_dd_create(16, 10, 1.0, 1.0, 0, ctypes.byref(h)) == _capi.SC_DD_EINVAL
    assert lib.sc_dd_create(16, 1000, 0.0, 1.0, 0, ctypes.byref(h)) == _capi.SC_DD_EINVAL
    assert lib.sc_dd_create(16, 1000, 1.0, 1.0, 0, None) == _capi.SC_DD_EINVAL
    n = ctypes.c_int()
    assert lib.sc_dd_search(None, None, 0, -1, 0, 1.0, 0.0, 10.0, None, 0, ctypes.byref(n), None) == _capi.SC_DD_EINVAL
    assert lib.sc_dd_memory_usage(None) == 0
    assert lib.sc_dd_destroy(None) == _capi.SC_DD_OK
    assert lib.sc_dd_set_paired_fp16(2) == _capi.SC_DD_EINVAL
    assert lib.sc_dd_set_paired_fp16(1) == _capi.SC_DD_OK


@pytest.mark.skipif(__import__("tests.conftest", fromlist=["has_gpu"]).has_gpu(), reason="checks the no-GPU path")
def test_create_without_gpu_reports_cuda_error():
    lib = _capi.lib()
    h = ctypes.c_void_p()
    rc = lib.sc_dd_create(16, 1000, 1.0, 1.0, 0, ctypes.byref(h))
    assert rc == _capi.SC_DD_ECUDA
    assert not h.value


def test_cpp_header_compiles():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"),
                        "-I/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "dedoppler_api_test.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_c_header_is_plain_c():
    src = '#include "seticore_b200.h"\nint main(void) { sc_dd_hit h; (void)h; return SC_DD_OK; }\n'
    r = subprocess.run(["gcc", "-std=c99", "-x", "c", "-fsyntax-only", "-I" + os.path.join(ROOT, "include"), "-"],
                       input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
