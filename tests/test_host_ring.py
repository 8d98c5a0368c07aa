"""The streaming service's host ring (rodv_b200/csrc/host_ring.h), which holds
submitted requests' bases until their batch is packed: a randomised C++ check
of its allocation (no overlapping or out-of-range ranges, releases in any
order, blocking acquire, stop), compiled and run on the CPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_host_ring_allocation(tmp_path):
    exe = tmp_path / "host_ring_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I",
                    os.path.join(ROOT, "rodv_b200", "csrc"),
                    os.path.join(HERE, "host_ring_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "OK", r.stdout + r.stderr
