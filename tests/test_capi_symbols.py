"""CPU-side checks of the drop-in boundary: the library builds, loads, and exports exactly the
entry points that include/bastr_gpu.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "bastr_gpu.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"BASTR_API\s+int\s+(bastr_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("bastr_create", "bastr_destroy", "bastr_set_state", "bastr_get_state", "bastr_step",
              "bastr_spectra", "bastr_fft", "bastr_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(gpu_lib):
    lib = ctypes.CDLL(gpu_lib._name)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from bastr_b200 import EXPORTED
    assert sorted(EXPORTED) == declared_symbols()


def test_create_rejects_bad_parameters_without_gpu(gpu_lib):
    """Parameter validation happens before any CUDA call, so it runs on a CPU-only host."""
    from bastr_b200 import CParams
    lib = ctypes.CDLL(gpu_lib._name)
    lib.bastr_create.argtypes = [ctypes.POINTER(CParams), ctypes.POINTER(ctypes.c_void_p)]
    lib.bastr_last_error.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32]
    lib.bastr_destroy.argtypes = [ctypes.c_void_p]
    cases = [
        (dict(ia=64, ja=64, ka=0, timemethod=3), -1, "time method"),
        (dict(ia=64, ja=64, ka=0, forcemethod=6), -1, "forcemethod 6"),
        (dict(ia=96, ja=96, ka=0), -2, "power of two"),
        (dict(ia=64, ja=16, ka=0), -2, "2*floor"),
        (dict(ia=1024, ja=1024, ka=1024), -2, "3D extents"),
    ]
    for kw, code, text in cases:
        p = CParams(kw.get("ia"), kw.get("ja"), kw.get("ka"), 273.15, 5000.0, 1e-4, 100,
                    kw.get("timemethod", 1), kw.get("forcemethod", 0), 5, 0.075, 0, 0, 0, 1)
        h = ctypes.c_void_p()
        rc = lib.bastr_create(ctypes.byref(p), ctypes.byref(h))
        buf = ctypes.create_string_buffer(512)
        lib.bastr_last_error(h, buf, 512)
        lib.bastr_destroy(h)
        assert rc == code, (kw, rc, buf.value)
        assert text in buf.value.decode()
