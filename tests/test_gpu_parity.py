"""GPU parity: the engine (through the C ABI) against the oracle and the reference.

Tolerance: |delta log10| <= 1e-3 is the engine's contract; these tests use the
reference's own test tolerance (1e-5 absolute, pairhmm_unittest.cpp and
pairhmm_schedule_unittest.cpp) wherever the oracle runs the same precision
path, and 1e-3 only where noted.
"""
import numpy as np
import pytest

import oracle
from conftest import assemble_batch, synthetic_batch
from rodv_b200 import RodvError, TestCase, compute_likelihoods, schedule_pairhmm, workloads
from rodv_b200.batch import Batch

pytestmark = pytest.mark.gpu
TOL = 1e-5          # same-path tolerance (reference tests' abs 1e-5)
CONTRACT = 1e-3     # engine contract in log10 units


def max_err(got, ref):
    """Max |got - ref| over finite references; non-finite ones must match exactly.

    A pair whose likelihood is below the FP64 range of the 2^1020 scaling
    gives -inf in the reference (log10 of 0), and must give -inf here too.
    """
    fin = np.isfinite(ref)
    assert np.array_equal(got[~fin], ref[~fin]), (got[~fin], ref[~fin])
    return float(np.abs(got[fin] - ref[fin]).max()) if fin.any() else 0.0


def test_simple_known_answers(engine):
    q4 = [43] * 4
    assert abs(engine.pair("ACGT", "ACGT", q4, q4, q4, q4) - (-6.022797e-01)) < TOL
    q5 = [43] * 5
    assert abs(engine.pair("ACGTA", "ACGTA", q5, q5, q5, q5) - (-0.69925308227539062)) < TOL
    assert abs(engine.pair("ACGTA", "ACGTA", q5, q5, q5, q5, use_double=True) -
               (-0.69925308227539062)) < TOL


def test_golden_file_one_pair_at_a_time(engine, gkl_cases):
    for hap, read, q, i, d, c, expected, ref_f, ref_d in gkl_cases[:40]:
        got = engine.pair(hap, read, q, i, d, c)
        assert abs(got - expected) / abs(expected) < 1e-5
        assert abs(got - ref_f) < TOL
        got_d = engine.pair(hap, read, q, i, d, c, use_double=True)
        assert abs(got_d - ref_d) < 1e-9


def test_golden_file_as_one_batch(engine, gkl_cases):
    """All 104 golden cases as single-pair regions of one batch (the inter tests' shape)."""
    regions = [([hap], [read], [q], [i], [d], [c]) for hap, read, q, i, d, c, *_ in gkl_cases]
    b = Batch.from_regions(regions)
    got = engine.batch(b)
    exp = np.array([x[6] for x in gkl_cases])
    ref = np.array([x[7] for x in gkl_cases])
    assert np.all(np.abs(got - exp) / np.abs(exp) < 1e-5)
    assert np.abs(got - ref).max() < TOL
    got_d = engine.batch(b, use_double=True)
    ref_d = np.array([x[8] for x in gkl_cases])
    assert np.abs(got_d - ref_d).max() < 1e-9


def test_assemble_regions_match_reference(engine):
    b, ref = assemble_batch()
    got, st = engine.batch(b, stats=True)
    assert st["pairs"] == len(ref)
    assert np.abs(got - ref).max() < TOL
    assert np.abs(got - oracle.batch_log10(b)).max() < TOL


def test_fp64_rescue_only_where_fp32_falls_below_its_bound(engine):
    """The FP64 pass must only see pairs whose FP32 likelihood is below the
    acceptance bound: a wrong (NaN, zero) FP32 result would be rescued
    silently and every value check would still pass.  The real chrY regions
    all stay in FP32; on a synthetic batch the rescue count matches the
    oracle's FP32 values below the bound (1e-28, or 1e-28/(mi*gapm) for the
    scaled uniform-gap form) up to pairs within 1e-5 of it."""
    b, _ = assemble_batch()
    _, st = engine.batch(b, stats=True)
    assert st["fp64_pairs"] == 0
    b = workloads.make_workload("plain")
    _, st = engine.batch(b, stats=True)
    raw = oracle.batch_log10(b, oracle.FP32_RAW)
    c = oracle.oracle_lib().oracle_ph2pr_f(45) * (1 - oracle.oracle_lib().oracle_ph2pr_f(10))
    bound = 1e-28 / c          # every read of this workload has ins=del=45, gcp=10
    below = int(np.sum(raw < bound))
    near = int(np.sum(np.abs(raw / bound - 1) < 1e-5))
    assert abs(st["fp64_pairs"] - below) <= near, (st["fp64_pairs"], below, near)


def test_multi_pass_sweeps_stop_only_for_pairs_fp32_rejects(engine):
    """Long reads (several 256-row passes) that stay in FP32 mixed with long
    reads whose likelihood falls below the FP32 bound after a few passes, with
    uniform and per-row gap qualities.  A sweep may stop after a pass once
    the boundary row's sum bounds the likelihood below the acceptance bound;
    the pairs that reach FP64 must be exactly those whose full FP32 sweep is
    below its bound, and every result must match the oracle."""
    rng = np.random.default_rng(77)
    regions, bounds = [], []
    lib = oracle.oracle_lib()
    for k in range(24):
        hl = int(rng.integers(800, 1300))
        hap = workloads._random_seq(rng, hl)
        rl = int(rng.integers(600, 780))
        start = int(rng.integers(0, hl - rl + 1))
        fail = k % 2 == 0
        rd = workloads._mutate(rng, hap[start:start + rl], 0.08 if fail else 0.001,
                               0.01 if fail else 0.0)
        n = len(rd)
        q = workloads._quals(rng, n, 25, 40)
        if k % 3 == 0:  # per-row gap qualities: the unscaled kernels
            ins, dele, gcp = (workloads._quals(rng, n, 30, 45) for _ in range(3))
            bounds.append(1e-28)
        else:
            ins = dele = np.full(n, 45, np.uint8)
            gcp = np.full(n, 10, np.uint8)
            bounds.append(1e-28 / (lib.oracle_ph2pr_f(45) * (1 - lib.oracle_ph2pr_f(10))))
        reads = [rd]
        if k % 4 == 1:  # a second read of the same haplotype: a same-haplotype item
            rd2 = workloads._mutate(rng, hap[start:start + rl], 0.001, 0.0)
            reads.append(rd2)
            n2 = len(rd2)
            ins2 = dele2 = np.full(n2, 45, np.uint8)
            regions.append(([hap], reads, [q, workloads._quals(rng, n2, 25, 40)],
                            [ins, ins2], [dele, dele2], [gcp, np.full(n2, 10, np.uint8)]))
            bounds.append(bounds[-1] if k % 3 else 1e-28 / (
                lib.oracle_ph2pr_f(45) * (1 - lib.oracle_ph2pr_f(10))))
            continue
        regions.append(([hap], reads, [q], [ins], [dele], [gcp]))
    b = Batch.from_regions(regions)
    got, st = engine.batch(b, stats=True)
    ref = oracle.batch_log10(b)
    assert np.abs(got - ref).max() < TOL
    raw = oracle.batch_log10(b, oracle.FP32_RAW)
    bounds = np.array(bounds)
    below = int(np.sum(raw < bounds))
    assert 0 < below < b.num_pairs
    assert st["fp64_pairs"] == below, (st["fp64_pairs"], below)


def test_odd_reads_pair_across_regions_without_changing_results(engine):
    """The odd single-pass read of a region (every read of a one-read region)
    is computed in two-haplotype items with other regions' odd reads.  Its
    results must match the oracle and be bitwise the same whether its region
    runs alone (no partner) or in a batch (a partner from another region)."""
    rng = np.random.default_rng(31)
    regions = []
    for k in range(40):
        nh = int(rng.integers(1, 6))
        nr = 1 if k % 2 == 0 else 3
        regions.append(workloads.random_region(rng, nh, nr, hap_len=(40, 400),
                                               read_len=(10, 250), vary_gap_quals=k % 4 == 1))
    b = Batch.from_regions(regions)
    got = engine.batch(b)
    assert np.abs(got - oracle.batch_log10(b)).max() < TOL
    off = b.out_offsets()
    for g in range(0, len(regions), 3):
        alone = engine.batch(b.subset([g]))
        assert np.array_equal(alone, got[int(off[g]):int(off[g + 1])]), g


def test_synthetic_n_bases_and_per_row_quals(engine):
    b, sched, intra = synthetic_batch()
    got = engine.batch(b)
    assert np.abs(got - intra).max() < TOL
    assert np.abs(got - sched).max() < TOL


@pytest.mark.parametrize("name,scale", [("tiny", 4.0), ("plain", 1.0), ("uneven", 0.01),
                                        ("stream", 0.02)])
def test_workloads_match_oracle(engine, name, scale):
    b = workloads.make_workload(name, scale=scale)
    got, st = engine.batch(b, stats=True)
    ref = oracle.batch_log10(b)
    assert np.isfinite(got).all()
    assert np.abs(got - ref).max() < TOL, (name, np.abs(got - ref).max())
    true = oracle.batch_log10(b, oracle.SCALED)
    assert np.abs(got - true).max() < CONTRACT


def test_underflow_sample_rescued_in_fp64(engine):
    b = workloads.make_workload("underflow", scale=0.002)
    got, st = engine.batch(b, stats=True)
    assert st["fp64_pairs"] == b.num_pairs  # every FP32 result falls below 1e-28
    ref = oracle.batch_log10(b, oracle.FP64)
    assert np.abs(got - ref).max() < 1e-9
    true = oracle.batch_log10(b, oracle.SCALED)
    assert np.abs(got - true).max() < CONTRACT


def test_long_pairs_multi_pass(engine):
    b = workloads.make_workload("long", scale=0.004)  # 8 pairs of 1-2 kb reads x 2-5 kb haps
    got = engine.batch(b)
    ref = oracle.batch_log10(b, oracle.REFERENCE)
    finite = np.isfinite(ref)
    assert np.abs(got[finite] - ref[finite]).max() < TOL


def test_long_pairs_c3_sample_against_reference(engine):
    """64 pairs of the long-pair configuration (1-2 kb reads x 2-5 kb
    haplotypes, 5% substitutions, 1% indels: every pair goes to FP64) against
    the reference's own schedule_pairhmm output and the FP64 oracle."""
    b = workloads.make_workload("long", scale=0.032)
    assert b.num_pairs == 64
    got, st = engine.batch(b, stats=True)
    assert np.abs(got - oracle.batch_log10(b, oracle.REFERENCE)).max() < TOL
    if oracle.ref_available():
        ref = oracle.ref_schedule(b)
        fin = np.isfinite(ref)
        assert np.array_equal(fin, np.isfinite(got))
        assert np.abs(got[fin] - ref[fin]).max() < TOL
    assert st["fp64_pairs"] == b.num_pairs


def _long_mixed_batch(seed=21):
    """Long reads of both multi-pass classes (uniform and per-row gap
    qualities), one to three reads per region (same-haplotype items and
    two-haplotype leftovers), lengths around the pass boundaries of both
    strip heights (128 and 256 rows), some pairs below the FP32 bound."""
    rng = np.random.default_rng(seed)
    regs = []
    lengths = [257, 300, 383, 384, 385, 511, 512, 513, 640, 767, 768, 1100]
    for k, L in enumerate(lengths):
        hl = L + int(rng.integers(40, 400))
        hap = workloads._random_seq(rng, hl)
        reads, qs, ins, dele, gcp = [], [], [], [], []
        for j in range(1 + k % 3):
            st = int(rng.integers(0, hl - L + 1))
            rd = workloads._mutate(rng, hap[st:st + L], 0.06 if (k + j) % 4 == 0 else 0.005, 0.0)
            n = len(rd)
            reads.append(rd)
            qs.append(workloads._quals(rng, n, 20, 40))
            if k % 2:
                ins.append(workloads._quals(rng, n, 30, 45))
                dele.append(workloads._quals(rng, n, 30, 45))
                gcp.append(workloads._quals(rng, n, 5, 15))
            else:
                ins.append(np.full(n, 45, np.uint8))
                dele.append(np.full(n, 45, np.uint8))
                gcp.append(np.full(n, 10, np.uint8))
        hap2 = workloads._mutate(rng, hap, 0.01, 0.001)
        regs.append(([hap, hap2], reads, qs, ins, dele, gcp))
    return Batch.from_regions(regs)


def _engine_with_multi_variants(tmp_path, v32, v64, force_fp64=False):
    """An engine whose two multi-pass classes use FP32 variant v32 and FP64
    variant v64 (from a tuning cache written for it); single-pass classes
    keep the tuned choice."""
    from rodv_b200 import Engine
    base = tmp_path / "tuned.txt"
    if not base.exists():
        e = Engine(0)
        e.autotune(str(base))
        e.close()
    lines = []
    for ln in base.read_text().splitlines():
        key, c, v, w = ln.split()
        if int(c) >= 16:
            v, w = str(v32), str(v64)
        lines.append(" ".join((key, c, v, w)))
    path = tmp_path / f"multi_{v32}_{v64}.txt"
    path.write_text("\n".join(lines) + "\n")
    e = Engine(0, autotune=1, tune_cache=str(path), force_fp64=force_fp64)
    tv = e.tuned_variants()
    assert tv["fp32"][16:] == [v32, v32] and tv["fp64"][16:] == [v64, v64]
    return e


def test_multi_pass_variants_give_identical_results(tmp_path):
    """Every strip height (4 or 8 rows per lane) and every number of warps
    sweeping one item's passes (2 or 4) gives bitwise the same results, FP32
    with rescue and forced FP64 alike, and they match the oracle."""
    b = _long_mixed_batch()
    ref = oracle.batch_log10(b)
    ref64 = oracle.batch_log10(b, oracle.FP64)
    first32 = first64 = None
    for v in range(4):
        e = _engine_with_multi_variants(tmp_path, v, v)
        got, st = e.batch(b, stats=True)
        e.close()
        assert 0 < st["fp64_pairs"] < b.num_pairs
        assert np.abs(got - ref).max() < TOL, v
        if first32 is None:
            first32 = got
        assert np.array_equal(got, first32), v
        e = _engine_with_multi_variants(tmp_path, v, v, force_fp64=True)
        got64 = e.batch(b)
        e.close()
        assert np.abs(got64 - ref64).max() < 1e-9, v
        if first64 is None:
            first64 = got64
        assert np.array_equal(got64, first64), v


def test_multi_pass_fp32_path():
    """Reads longer than one pass that stay in FP32 range (high identity)."""
    from rodv_b200 import Engine
    e = Engine(0)
    rng = np.random.default_rng(11)
    regs = []
    for L in (257, 300, 511, 512, 513, 800):
        hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L + 40)]
        read = hap[20:20 + L].copy()
        q = rng.integers(30, 41, L).astype(np.uint8)
        regs.append(([hap], [read], [q], [np.full(L, 45, np.uint8)],
                     [np.full(L, 45, np.uint8)], [np.full(L, 10, np.uint8)]))
        # per-row gap quals too
        regs.append(([hap], [read], [q], [rng.integers(30, 50, L).astype(np.uint8)],
                     [rng.integers(30, 50, L).astype(np.uint8)],
                     [rng.integers(5, 20, L).astype(np.uint8)]))
    b = Batch.from_regions(regs)
    got, st = e.batch(b, stats=True)
    ref = oracle.batch_log10(b)
    assert st["fp64_pairs"] < b.num_pairs
    assert np.abs(got - ref).max() < TOL
    e.close()


def test_edge_lengths(engine):
    """Reads of 1 base, reads longer than the haplotype, one-base haplotypes,
    every rows-per-lane class boundary (32*R and 32*R+1), odd pair counts."""
    rng = np.random.default_rng(7)
    regs = []
    for L in (1, 2, 31, 32, 33, 63, 64, 65, 96, 97, 128, 129, 160, 192, 224, 255, 256):
        for H in (1, 5, L + 3, 2 * L + 1):
            hap = np.frombuffer(b"ACGTN", np.uint8)[rng.integers(0, 4, H)]
            read = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L)]
            regs.append(([hap], [read], [rng.integers(6, 44, L).astype(np.uint8)],
                         [rng.integers(6, 44, L).astype(np.uint8)],
                         [rng.integers(6, 44, L).astype(np.uint8)],
                         [rng.integers(6, 44, L).astype(np.uint8)]))
    b = Batch.from_regions(regs)
    got = engine.batch(b)
    ref = oracle.batch_log10(b)
    assert max_err(got, ref) < TOL


def test_chain_items_many_haps_mixed_reads(engine):
    """Regions swept as chains: more haplotypes than one chain holds (32),
    one-base and long haplotypes side by side, an odd read count, reads of
    neighbouring row classes paired together, uniform and per-row gap quals in
    one region, N bases on both sides."""
    rng = np.random.default_rng(21)
    regs = []
    for nh, nr in ((70, 9), (33, 4), (32, 1), (5, 7), (1, 3)):
        base = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 700)]
        haps = []
        for k in range(nh):
            H = int(rng.choice([1, 2, 31, 32, 33, 100, 257, 600]))
            h = base[:H].copy()
            mut = rng.random(H) < 0.02
            h[mut] = np.frombuffer(b"ACGTN", np.uint8)[rng.integers(0, 5, mut.sum())]
            haps.append(h)
        reads, q, ins, dl, gc = [], [], [], [], []
        for k in range(nr):
            L = int(rng.choice([1, 31, 32, 33, 64, 65, 150, 255, 256]))
            st = int(rng.integers(0, 700 - L))
            r = base[st:st + L].copy()
            if k % 3 == 0:
                r[rng.integers(0, L)] = ord("N")
            reads.append(r)
            q.append(rng.integers(10, 41, L).astype(np.uint8))
            if k % 2:
                ins.append(rng.integers(20, 46, L).astype(np.uint8))
                dl.append(rng.integers(20, 46, L).astype(np.uint8))
                gc.append(rng.integers(5, 16, L).astype(np.uint8))
            else:
                ins.append(np.full(L, 45, np.uint8))
                dl.append(np.full(L, 45, np.uint8))
                gc.append(np.full(L, 10, np.uint8))
        regs.append((haps, reads, q, ins, dl, gc))
    b = Batch.from_regions(regs)
    got, st = engine.batch(b, stats=True)
    ref = oracle.batch_log10(b)
    assert max_err(got, ref) < TOL
    true = oracle.batch_log10(b, oracle.SCALED)
    fin = np.isfinite(true)
    assert np.abs(got[fin] - true[fin]).max() < CONTRACT


def test_gap_qual_extremes(engine):
    """gcp quality 0 (gap continuation probability 1) and ins/del quality 0."""
    rng = np.random.default_rng(9)
    regs = []
    for gq, iq in ((0, 45), (1, 45), (10, 0), (127, 127), (255, 200)):
        L, H = 40, 60
        hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, H)]
        read = hap[5:5 + L].copy()
        regs.append(([hap], [read], [rng.integers(10, 40, L).astype(np.uint8)],
                     [np.full(L, iq, np.uint8)], [np.full(L, iq, np.uint8)],
                     [np.full(L, gq, np.uint8)]))
    b = Batch.from_regions(regs)
    got = engine.batch(b)
    ref = oracle.batch_log10(b)
    ok = np.isfinite(ref)
    assert np.array_equal(np.isfinite(got), ok)
    assert np.abs(got[ok] - ref[ok]).max() < TOL


def test_force_fp64_matches_fp64_oracle(engine):
    b = workloads.make_workload("tiny", scale=2.0)
    got, st = engine.batch(b, use_double=True, stats=True)
    assert st["fp64_pairs"] == b.num_pairs
    assert np.abs(got - oracle.batch_log10(b, oracle.FP64)).max() < 1e-9


def test_device_batch_reruns_are_identical(engine):
    b = workloads.make_workload("uneven", scale=0.002)
    db = engine.upload(b)
    db.run()
    first = db.download()
    db.run()
    second = db.download()
    assert np.array_equal(first, second)
    assert np.abs(first - engine.batch(b)).max() == 0.0
    db.free()


def test_chain_length_does_not_change_results(engine):
    """A region computed alone (one haplotype per chain item: a small batch)
    and inside thousands of copies (whole-region chains) gives bitwise the
    same results, for reads that fill every row of their lanes (length a
    multiple of 32) and for reads that do not."""
    rng = np.random.default_rng(12)
    base = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 200)]
    haps = []
    for k in range(8):
        h = base[:100 + 60 * (k % 2)].copy()
        h[rng.random(len(h)) < 0.02] = ord("G")
        haps.append(h)
    reads, q, ins, gcp = [], [], [], []
    for L in (64, 95, 96, 128, 127, 160):
        st = int(rng.integers(0, 200 - L))
        reads.append(base[st:st + L].copy())
        q.append(rng.integers(10, 41, L).astype(np.uint8))
        ins.append(np.full(L, 45, np.uint8))
        gcp.append(np.full(L, 10, np.uint8))
    region = (haps, reads, q, ins, ins, gcp)
    alone = engine.batch(Batch.from_regions([region]))
    many = engine.batch(Batch.from_regions([region] * 2000))
    n = len(alone)
    assert np.array_equal(many[:n], alone)
    assert np.array_equal(many[-n:], alone)


def test_stacked_read_pairs_match_one_pair_items(engine):
    """Read pairs stacked down the lanes of one chain item (a region with many
    uniform-gap reads, packed into multi-pair items of whatever class is
    cheapest) give bitwise the results the same two reads give as the only
    pair of a region (one pair per item, the class of the longer read): a
    read's arithmetic does not depend on its partner, lanes, item or class.
    Lengths include each class's last (32R - 2 bases) and a multiple of 32."""
    rng = np.random.default_rng(77)
    base = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 320)]
    haps = []
    for k in range(6):
        h = base[:180 + 16 * k].copy()
        h[rng.random(len(h)) < 0.02] = ord("T")
        haps.append(h)
    lens = [20, 30, 31, 33, 50, 62, 64, 70, 94, 95, 100, 120, 126, 127, 150, 158, 160, 190,
            222, 224, 230, 254, 40, 45, 55, 60, 75, 80, 85, 90, 105, 110, 115, 135, 140, 170,
            200, 210, 240, 250]
    reads, q, ins, gcp = [], [], [], []
    for L in lens:
        st = int(rng.integers(0, 320 - L))
        reads.append(base[st:st + L].copy())
        q.append(rng.integers(10, 41, L).astype(np.uint8))
        ins.append(np.full(L, 45, np.uint8))
        gcp.append(np.full(L, 10, np.uint8))
    n = len(reads)
    big_batch = Batch.from_regions([(haps, reads, q, ins, ins, gcp)])
    big = engine.batch(big_batch)
    assert np.abs(big - oracle.batch_log10(big_batch)).max() < TOL
    for i, j in ((0, 1), (4, 21), (13, 14), (18, 19), (21, 39), (2, 3)):
        pair = [i, j]
        small = engine.batch(Batch.from_regions([(haps, [reads[k] for k in pair],
                                                  [q[k] for k in pair], [ins[k] for k in pair],
                                                  [ins[k] for k in pair],
                                                  [gcp[k] for k in pair])]))
        for h in range(len(haps)):
            assert small[h * 2] == big[h * n + i], (i, j, h)
            assert small[h * 2 + 1] == big[h * n + j], (i, j, h)


def test_chunked_host_path_matches_resident(engine):
    """A batch large enough for the pipelined host-buffer path (region ranges
    packed and uploaded while the previous range computes) gives bitwise the
    results of the same batch computed resident in one piece."""
    b = workloads.make_workload("uneven", scale=0.26)  # ~1.3e11 cells: 2 ranges
    assert b.cells() >= 1.2e11
    got, st = engine.batch(b, stats=True)
    assert st["pairs"] == b.num_pairs and st["cells"] == b.cells()
    db = engine.upload(b)
    db.run()
    resident = db.download()
    db.free()
    assert np.array_equal(got, resident)
    # a second call reuses the lanes' buffers
    assert np.array_equal(engine.batch(b), resident)


def test_plain_form_matches_batched(engine):
    b = workloads.make_workload("tiny", scale=1.0)
    db = engine.upload(b)
    got, st = engine.plain(db)
    assert st["kernel_launches"] >= b.num_pairs
    assert np.abs(got - oracle.batch_log10(b)).max() < TOL
    db.free()


def test_schedule_pairhmm_mirror():
    b = workloads.make_workload("tiny", scale=1.0)
    haps, reads, q, i, d, c = b.region(0)
    result = []
    assert schedule_pairhmm(haps, reads, result, q, i, d, c)
    assert len(result) == len(haps) and all(len(r) == len(reads) for r in result)
    flat = np.array(result).ravel()
    assert np.abs(flat - oracle.batch_log10(b.subset([0]))).max() < TOL
    assert schedule_pairhmm([], reads, result, q, i, d, c) is False
    assert schedule_pairhmm(haps, [], result, [], [], [], []) is False


def test_compute_likelihoods_mirror(gkl_cases):
    hap, read, q, i, d, c, expected, *_ = gkl_cases[0]
    tc = TestCase(hap, read, q, i, d, c)
    assert abs(compute_likelihoods(tc) - expected) / abs(expected) < 1e-5
    assert abs(compute_likelihoods(tc, use_double=True) - expected) / abs(expected) < 1e-5


def test_invalid_inputs_fail_loudly(engine):
    good = ([b"ACGT"], [b"ACG"], [[30] * 3], [[45] * 3], [[45] * 3], [[10] * 3])
    with pytest.raises(RodvError) as ei:
        engine.batch(Batch.from_regions([([b"ACGU"],) + good[1:]]))
    assert ei.value.status == 3
    with pytest.raises(RodvError) as ei:
        engine.batch(Batch.from_regions([(good[0], [b"acg"]) + good[2:]]))
    assert ei.value.status == 3
    with pytest.raises(RodvError) as ei:
        engine.batch(Batch.from_regions([([], ) + good[1:]]))
    assert ei.value.status == 2
    with pytest.raises(RodvError) as ei:
        engine.batch(Batch.from_regions([([b""],) + good[1:]]))
    assert ei.value.status == 1
    # the engine stays usable after rejected calls
    assert np.isfinite(engine.batch(Batch.from_regions([good]))).all()


def test_peaks_are_measured(engine):
    p = engine.measure_peaks()
    assert p["fp32_gflops"] > 1e4 and p["fp64_gflops"] > 1e3 and p["sm_mhz"] > 300


def test_autotune_picks_variants_and_keeps_results(tmp_path):
    """The autotuner picks one kernel variant per work class (occupancy target;
    for reads up to 128 bases also one or two chain items per warp), caches
    it, and the results do not depend on the variant (bitwise)."""
    from rodv_b200 import Engine
    b = workloads.make_workload("uneven", scale=0.003)
    e = Engine(0)
    before = e.batch(b)
    cache = str(tmp_path / "tune.txt")
    variants = e.autotune(cache)
    assert len(variants) == 18
    # classes 0-7: single-pass reads up to 128 bases (8 variants); others 4
    assert all(0 <= v < (8 if c < 8 else 4) for c, v in enumerate(variants)), variants
    assert open(cache).read().count("\n") == 18
    after = e.batch(b)
    assert np.array_equal(after, before)
    assert np.abs(after - oracle.batch_log10(b)).max() < TOL
    e2 = Engine(0, autotune=1, tune_cache=cache)   # loads the cache, no re-tuning
    assert np.abs(e2.batch(b) - before).max() < TOL
    e.close()
    e2.close()


def test_forced_fp64_device_batch_graph_replays():
    """A device batch of an FP64-forced engine: the captured launch graph
    replays with the list lengths restored from device memory every run."""
    from rodv_b200 import Engine
    e = Engine(0, force_fp64=True)
    b = workloads.make_workload("tiny", scale=1.0)
    db = e.upload(b)
    s1 = db.run()
    r1 = db.download()
    s2 = db.run()
    r2 = db.download()
    assert s1["fp64_pairs"] == s2["fp64_pairs"] == b.num_pairs
    assert np.array_equal(r1, r2)
    assert np.abs(r1 - oracle.batch_log10(b, oracle.FP64)).max() < 1e-9
    db.free()
    e.close()


def test_raw_output_matches_log10_output(engine):
    """rodv_pairhmm_batch_raw (the inter API's islog10 = false) returns the
    scaled likelihood and its precision; log10 of it with that precision's
    offset is the log10 result, FP32 raws agree with the oracle's FP32 sum,
    and a likelihood below the FP64 normal range comes back as 0 (-inf).
    The uneven sample is large enough for the pipelined host path (region
    ranges over three lanes)."""
    for b in (workloads.make_workload("tiny", scale=4.0),
              workloads.make_workload("underflow", scale=0.002),
              workloads.make_workload("uneven", scale=0.05)):
        want = engine.batch(b)
        raw, prec = engine.batch_raw(b)
        assert set(np.unique(prec)) <= {0, 1}
        off = np.where(prec == 0, float(np.float32(36.1236000061)), 307.050595577260822)
        with np.errstate(divide="ignore"):
            got = np.log10(raw) - off
        fin = np.isfinite(want)
        assert np.array_equal(fin, np.isfinite(got))
        assert np.abs(got[fin] - want[fin]).max() < 1e-12
        assert np.all(raw[prec == 0] >= 1e-28)
        sel = prec == 0
        if b.num_pairs < 5000 and sel.any():
            f32 = oracle.batch_log10(b, oracle.FP32_RAW)
            assert np.abs(raw[sel] / f32[sel] - 1).max() < 1e-4
    # forced FP64: every precision byte is 1
    b = workloads.make_workload("tiny", scale=2.0)
    raw, prec = engine.batch_raw(b, use_double=True)
    assert np.all(prec == 1)
    with np.errstate(divide="ignore"):
        got = np.log10(raw) - 307.050595577260822
    want = engine.batch(b, use_double=True)
    fin = np.isfinite(want)
    assert np.abs(got[fin] - want[fin]).max() < 1e-12
