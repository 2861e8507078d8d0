"""The C ABI library loads, exports every function include/*.h declares, and
fails with a status code (not a crash, not a CPU fallback) without a GPU."""
import ctypes
import glob
import os
import re

import pytest

import infraga_b200 as ig
from infraga_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(iga_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_functions():
    assert "iga_fan_run" in declared_functions()


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    L = ig.lib()
    assert hasattr(L, name), f"{name} declared in include/ but not exported by libinfraga_gpu.so"


def test_binding_covers_header():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_status_strings():
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert _lib.strerror(code)


def test_invalid_arguments_rejected_without_device():
    L = ig.lib()
    n = ctypes.c_int()
    assert L.iga_fan_run(None, None, None, None, 0, None, 0, ctypes.byref(n), None, None, None, None, None) == _lib.IGA_E_INVALID
    assert L.iga_atmo_load(None, b"zTuvdp", 0, None) == _lib.IGA_E_INVALID
    h = ctypes.c_void_p()
    met = os.path.join(ROOT, "tests", "golden", "profiles", "gen0.met").encode()
    assert L.iga_atmo_load_topo(None, b"t.dat", b"zTuvdp", 0, 0, ctypes.byref(h)) == _lib.IGA_E_INVALID
    assert L.iga_atmo_load_topo(met, b"t.dat", b"zTuvdp", 0, 7, ctypes.byref(h)) == _lib.IGA_E_INVALID
    # a missing terrain file fails in the host loader, before any device call
    assert L.iga_atmo_load_topo(met, b"/nonexistent/t.dat", b"zTuvdp", 0, 0, ctypes.byref(h)) == _lib.IGA_E_IO
    assert not h.value
    z = (ctypes.c_double * 1)(0.0)
    out = (ctypes.c_double * 4)()
    assert L.iga_atmo_sample(None, None, 0.0, 0.0, z, 1, out) == _lib.IGA_E_INVALID
    assert L.iga_fan_paths(None, None, None, None, 0, 2, None, None, 0, None, None, None, 0, None, None) == \
        _lib.IGA_E_INVALID


def test_no_silent_cpu_fallback_when_no_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(ig.IgaError):
        ig.Atmosphere.load(os.path.join(ROOT, "tests", "golden", "profiles", "gen0.met"))


def test_static_scratch_covers_fan_workspace():
    """iga_fan_run_device_noalloc refuses fans whose scratch need exceeds its
    static array; the fan's need is a constant that must fit."""
    text = open(os.path.join(ROOT, "include", "infraga_gpu.h")).read()
    m = re.search(r"#define\s+IGA_FAN_STATIC_SCRATCH_BYTES\s+(\d+)", text)
    assert m, "IGA_FAN_STATIC_SCRATCH_BYTES not defined in the header"
    assert 0 < ig.fan_workspace_bytes() <= int(m.group(1))
    # without a device the entry point fails on its arguments, before any CUDA call
    L = ig.lib()
    assert L.iga_fan_run_device_noalloc(None, None, None, None, 0, None, None, None, None, None, None) == \
        _lib.IGA_E_INVALID
