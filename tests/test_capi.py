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


C_CALLER = r"""
#include <stdio.h>
#include <string.h>
#include "rodv_pairhmm.h"

int main(void) {
  /* one region: two haplotypes x two reads */
  const char* haps = "ACGTACGTACGTAAAACCCCGGGG";
  const char* reads = "ACGTAACCCC";
  const uint64_t hap_off[2] = {0, 12};
  const uint32_t hap_len[2] = {12, 12};
  const uint64_t read_off[2] = {0, 5};
  const uint32_t read_len[2] = {5, 5};
  uint8_t q[10], gi[10], gc[10];
  rodv_region reg = {0, 2, 0, 2};
  rodv_batch b;
  rodv_options o;
  rodv_engine* e = NULL;
  char msg[128];
  rodv_status s;
  memset(q, 30, sizeof q); memset(gi, 45, sizeof gi); memset(gc, 10, sizeof gc);
  b.num_regions = 1; b.regions = &reg;
  b.num_haps = 2; b.hap_bases = (const uint8_t*)haps; b.hap_offsets = hap_off;
  b.hap_lengths = hap_len; b.num_reads = 2; b.read_bases = (const uint8_t*)reads;
  b.base_quals = q; b.ins_quals = gi; b.del_quals = gi; b.gcp_quals = gc;
  b.read_offsets = read_off; b.read_lengths = read_len;
  if (rodv_batch_num_pairs(&b) != 4) return 10;
  if (rodv_batch_validate(&b, msg, sizeof msg) != RODV_OK) return 11;
  reg.num_reads = 3;                       /* indexes past the read arrays */
  if (rodv_batch_validate(&b, msg, sizeof msg) != RODV_ERR_INVALID_ARG) return 12;
  reg.num_reads = 2;
  rodv_default_options(&o);
  s = rodv_engine_create(&o, &e);
  if (s == RODV_OK) rodv_engine_destroy(e);
  else if (s != RODV_ERR_NO_DEVICE) return 13;
  printf("%s\n", rodv_status_string(s));
  return 0;
}
"""


def test_header_is_c99_and_a_c_caller_links(tmp_path):
    """A plain C99 caller (gcc -std=c99 -pedantic -Werror) includes the header,
    builds a batch, validates it and creates an engine (no device here: the
    clean RODV_ERR_NO_DEVICE status)."""
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", libdir, "-l:librodv_pairhmm.so", f"-Wl,-rpath,{libdir}"],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert r.stdout.strip() in ("ok", "no usable CUDA device"), r.stdout
