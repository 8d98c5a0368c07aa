"""The CPU oracle pinned against the reference's golden vectors and its own outputs.

The oracle (oracle/pairhmm_oracle.c) is the checker for every GPU parity test,
so it is checked first against everything the reference holds for this path:
the 104 golden lines of resouces/pairhmm-testdata.txt (tolerance as
src/core/test/pairhmm_unittest.cpp:378-390, relative 1e-5), the two
hand-computed values of pairhmm_unittest.cpp:103-137 (abs 1e-5), and the
reference's own intra/schedule outputs recorded in tests/golden/.
"""
import numpy as np
import pytest

import oracle
from conftest import assemble_batch, synthetic_batch


def test_golden_file_reference_mode(gkl_cases):
    assert len(gkl_cases) == 104
    for hap, read, q, i, d, c, expected, _, _ in gkl_cases:
        got = oracle.pair_log10(hap, read, q, i, d, c, oracle.REFERENCE)
        assert abs(got - expected) / abs(expected) < 1e-5
        assert abs(got - expected) < 1e-5


@pytest.mark.parametrize("mode", [oracle.FP64, oracle.SCALED])
def test_golden_file_fp64_modes(gkl_cases, mode):
    for hap, read, q, i, d, c, expected, _, _ in gkl_cases:
        got = oracle.pair_log10(hap, read, q, i, d, c, mode)
        assert abs(got - expected) / abs(expected) < 1e-5


def test_golden_file_matches_reference_run(gkl_cases):
    """Against the reference's own computeLikelihoodsAVX512 outputs, FP32 and FP64."""
    for hap, read, q, i, d, c, _, ref_f, ref_d in gkl_cases:
        assert abs(oracle.pair_log10(hap, read, q, i, d, c, oracle.REFERENCE) - ref_f) < 5e-6
        assert abs(oracle.pair_log10(hap, read, q, i, d, c, oracle.FP64) - ref_d) < 1e-9


def test_simple_known_answers():
    q4 = [43] * 4
    assert abs(oracle.pair_log10("ACGT", "ACGT", q4, q4, q4, q4) - (-6.022797e-01)) < 1e-5
    q5 = [43] * 5
    assert abs(oracle.pair_log10("ACGTA", "ACGTA", q5, q5, q5, q5) -
               (-0.69925308227539062)) < 1e-5


def test_assemble_regions_match_reference_schedule():
    b, ref = assemble_batch()
    assert b.num_pairs == len(ref)
    got = oracle.batch_log10(b, oracle.REFERENCE)
    assert np.abs(got - ref).max() < 1e-5


def test_synthetic_with_n_matches_reference():
    b, sched, intra = synthetic_batch()
    got = oracle.batch_log10(b, oracle.REFERENCE)
    # N pairs go through the reference's intra path inside schedule_pairhmm
    assert np.abs(got - intra).max() < 1e-5
    assert np.abs(got - sched).max() < 1e-5


def test_scaled_mode_agrees_where_fp64_is_in_range(gkl_cases):
    for hap, read, q, i, d, c, *_ in gkl_cases[:20]:
        a = oracle.pair_log10(hap, read, q, i, d, c, oracle.FP64)
        s = oracle.pair_log10(hap, read, q, i, d, c, oracle.SCALED)
        assert abs(a - s) < 1e-9


def test_scaled_mode_reaches_below_fp64_range():
    """A pair whose likelihood is below the 2^1020-scaled FP64 range."""
    rng = np.random.default_rng(3)
    hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 3000)]
    read = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 1500)]
    q = np.full(1500, 40, np.uint8)
    gi = np.full(1500, 45, np.uint8)
    gc = np.full(1500, 10, np.uint8)
    ref_style = oracle.pair_log10(hap, read, q, gi, gi, gc, oracle.FP64)
    true = oracle.pair_log10(hap, read, q, gi, gi, gc, oracle.SCALED)
    assert np.isfinite(true) and true < -700
    assert not np.isfinite(ref_style) or ref_style < -600


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_oracle_matches_reference_library_on_uneven_sample():
    from rodv_b200 import workloads
    b = workloads.make_workload("uneven", scale=0.002)
    ref = oracle.ref_schedule(b)
    got = oracle.batch_log10(b, oracle.REFERENCE)
    assert np.abs(got - ref).max() < 1e-5


def test_assemble_log_reader_round_trips_the_logged_regions(tmp_path):
    """rodv_b200.assemble_log reads roDV's assemble-log format: the 8 chrY
    regions written in that format come back as the same batch."""
    from conftest import assemble_batch, load_assemble
    from rodv_b200 import assemble_log
    regs = load_assemble()
    path = tmp_path / "pairhmm_debug.txt"
    oracle.write_assemble_log(regs, str(path))
    parsed = assemble_log.parse_file(str(path))
    assert [p.name for p in parsed] == [r["region"] for r in regs]
    assert all(p.skipped_reads == 0 for p in parsed)
    b = assemble_log.to_batch(parsed)
    ref_b, _ = assemble_batch()
    for f in ("regions", "hap_bases", "hap_lengths", "read_bases", "base_quals", "ins_quals",
              "del_quals", "gcp_quals", "read_lengths"):
        assert np.array_equal(getattr(b, f), getattr(ref_b, f)), f
    # a read whose quality line is short is dropped and counted
    text = path.read_text().replace("  gcp: 10 10 10 10 10 10 10 10 10 10 10 10 10 10 10\n",
                                    "  gcp: 10 10\n", 1)
    bad = assemble_log.parse_lines(text.splitlines(keepends=True))
    assert bad[0].skipped_reads == 1 and len(bad[0].reads) == len(parsed[0].reads) - 1
