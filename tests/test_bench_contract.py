"""bench.py's reference arm (the reference's CPU schedule_pairhmm, built under
oracle/_ref) keeps the one-JSON-line contract on CPU: rank 0 prints the line
with the metric, the bounded per-step sample, a cpu_baseline describing the
run and an e2e entry without transfers; other ranks exit 0 and print nothing.
Also the roofline's traffic figure, read from the committed ncu summary."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="oracle/_ref not built (needs the reference tree)")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "2", "--warmup", "1", "--ref-seconds", "0.3"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


@needs_ref
def test_reference_arm_prints_one_contract_line():
    lines = _run({"WORLD_SIZE": "1", "RANK": "0", "LOCAL_RANK": "0"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GCUPS" and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["higher_is_better"] is True and d["ms_per_step"] > 0
    assert d["metric"].startswith("PairHMM GCUPS")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert "regions" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "GCUPS", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@needs_ref
def test_reference_arm_other_ranks_exit_quietly():
    assert _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"}) == []


def test_roofline_traffic_comes_from_a_capture_of_these_kernels():
    """The committed traffic capture was taken on the kernel sources of this
    build (bench.py reports no traffic from a capture of other kernels, and
    this test fails until the capture is taken again)."""
    sys.path.insert(0, ROOT)
    import bench
    f = bench.profile_fields()
    assert f.get("kernel_source_sha16") == bench.kernel_source_sha(), (
        "profiles/forward_kernels_dram_traffic_uneven.md was captured on other kernel "
        "sources; capture it again")
    t, note = bench.step_traffic_bytes("uneven", 1.0)
    assert t is not None and 2e8 < t < 5e9, note
    assert bench.step_traffic_bytes("uneven", 0.5)[0] is None
    assert bench.step_traffic_bytes("stream", 1.0)[0] is None


def test_kernel_source_hash_ignores_comments_only():
    """The capture's source hash follows the compiled code: comments, blank
    lines and trailing spaces do not change it, any code change does, and
    comment markers inside string literals are code."""
    sys.path.insert(0, ROOT)
    import bench
    a = 'int f() {\n  return 1;  // one\n}\n/* block\n comment */\nconst char* s = "a//b";\n'
    b = '// new header\nint f() {\n  return 1;\n}\n\nconst char* s = "a//b";   \n'
    c = 'int f() {\n  return 2;\n}\nconst char* s = "a//b";\n'
    d = 'int f() {\n  return 1;\n}\nconst char* s = "a";\n'
    assert bench._code_only(a) == bench._code_only(b)
    assert bench._code_only(a) != bench._code_only(c)
    assert bench._code_only(a) != bench._code_only(d)
