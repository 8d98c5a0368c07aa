"""The reference's own scheduler tests run against the B200 engine.

oracle/_ref/ref_schedule_tests_on_rodv is built (oracle/Makefile, target
`conformance`) from the reference's unchanged test sources
src/core/test/pairhmm_schedule_unittest.cpp and
src/core/test/pairhmm_unitest_from_assemble.cpp, with a minimal gtest
(oracle/conformance/gtest/gtest.h), linked with the reference's CPU kernels
(the tests compare schedule_pairhmm against computeLikelihoodsAVX512/AVX2)
but not with its pairhmm_schedule.cpp: schedule_pairhmm resolves to
librodv_pairhmm.so, i.e. the GPU engine.  The assemble test reads
resouces/pairhmm_debug.txt relative to its working directory; the test below
writes the 8 real chrY regions there from the committed fixture.
"""
import os
import subprocess

import pytest

import oracle
from conftest import load_assemble
from rodv_b200 import _lib

BIN = oracle.CONFORMANCE_BIN
built = pytest.mark.skipif(not os.path.exists(BIN),
                           reason="conformance binary not built (needs the reference tree)")


@built
def test_conformance_binary_takes_schedule_pairhmm_from_the_engine():
    syms = subprocess.run(["nm", "-C", BIN], capture_output=True, text=True, check=True).stdout
    lines = [ln for ln in syms.splitlines() if "pairhmm::schedule::schedule_pairhmm(" in ln]
    assert lines and all(" U " in ln for ln in lines), lines  # undefined: from the library
    deps = subprocess.run(["ldd", BIN], capture_output=True, text=True).stdout
    assert os.path.realpath(_lib.LIB_PATH) in {os.path.realpath(p.split()[2])
                                               for p in deps.splitlines() if "librodv" in p}


@built
@pytest.mark.gpu
def test_reference_scheduler_tests_pass_on_the_engine(tmp_path):
    os.makedirs(tmp_path / "resouces")
    oracle.write_assemble_log(load_assemble(), str(tmp_path / "resouces" / "pairhmm_debug.txt"))
    r = subprocess.run([BIN], cwd=tmp_path, capture_output=True, text=True, timeout=900)
    out = r.stdout
    assert r.returncode == 0, out[-3000:] + r.stderr[-3000:]
    assert "[  FAILED  ]" not in out and "[  SKIPPED ]" not in out, out
    # 3 tests of pairhmm_schedule_unittest.cpp + 1 of pairhmm_unitest_from_assemble.cpp
    assert out.count("[       OK ]") == 4, out
