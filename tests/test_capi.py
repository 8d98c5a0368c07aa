"""The C-ABI library: it loads, and exports every function its headers declare.

No compute call runs here (there is no GPU in the CPU suite); engine creation
must fail cleanly with RODV_ERR_NO_DEVICE instead.
"""
import ctypes
import os
import re
import subprocess

import pytest

from rodv_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rodv_pairhmm.h")


def declared_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(rodv_[a-z0-9_]+)\s*\(",
                       text, flags=re.M)
    return sorted(set(names))


def exported_symbols(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True,
                         text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_library_exports_every_declared_function():
    names = declared_functions(HEADER)
    assert len(names) >= 14
    syms = exported_symbols(_lib.LIB_PATH)
    missing = [n for n in names if n not in syms]
    assert not missing, f"declared but not exported: {missing}"
    # every declared function also has a ctypes signature in the binding
    bound = {name for name, _, _ in _lib.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_schedule_pairhmm_cpp_symbol_exported():
    """The drop-in C++ symbol with roDV's exact signature (pairhmm_schedule.h:14-25)."""
    syms = exported_symbols(_lib.LIB_PATH)
    mangled = ("_ZN7pairhmm8schedule16schedule_pairhmmERKSt6vectorIS1_IhSaIhEESaIS3_EES7_"
               "RS1_IS1_IdSaIdEESaIS9_EES7_S7_S7_S7_bddb")
    assert mangled in syms


def test_library_loads_and_reports_status_strings():
    lib = _lib.load()
    assert lib.rodv_status_string(0) == b"ok"
    assert lib.rodv_status_string(3) == b"base outside A, C, G, T, N"
    assert lib.rodv_status_string(999) == b"unknown status"


def test_default_options():
    lib = _lib.load()
    o = _lib.Options()
    o.device = 7
    lib.rodv_default_options(ctypes.byref(o))
    assert o.device == 0 and o.force_fp64 == 0


def test_device_code_is_sm100a_only():
    """The library holds device code for sm_100a (cuobjdump lists ELF arches only)."""
    r = subprocess.run(["cuobjdump", "--list-elf", _lib.LIB_PATH], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    arches = set(re.findall(r"sm_\d+a?", r.stdout))
    assert arches == {"sm_100a"}, arches


def test_engine_create_without_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.rodv_engine_create(None, ctypes.byref(h))
    assert st == 4  # RODV_ERR_NO_DEVICE
    assert not h.value


def test_python_engine_raises_without_device():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from rodv_b200 import Engine, RodvError
    with pytest.raises(RodvError) as ei:
        Engine(0)
    assert ei.value.status == 4


def test_service_create_without_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.rodv_service_create(None, ctypes.byref(h)) == 4  # RODV_ERR_NO_DEVICE
    assert not h.value
    # calls on a null service are argument errors, never crashes
    t = ctypes.c_uint64()
    assert lib.rodv_submit_region(None, None, ctypes.byref(t)) == 1
    assert lib.rodv_poll(None, 1, None, None) == 1
    assert lib.rodv_service_last_error(None) == b""
