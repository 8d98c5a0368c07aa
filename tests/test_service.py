"""The streaming service (rodv_service_*): continuous batching must not change
any result.  A region's log10 likelihoods are bitwise identical whether it is
computed alone, in whatever batch the service forms while other requests
arrive, or in one rodv_pairhmm_batch call with everything else."""
import threading

import numpy as np
import pytest

import oracle
from rodv_b200 import Engine, RodvError, Service, workloads
from rodv_b200.batch import Batch

pytestmark = pytest.mark.gpu
TOL = 1e-5


def mixed_regions():
    """Regions of every kind the batcher can mix: the streaming workload's
    shapes (1-32 haplotypes of 100-800 bases, 1-300 reads), per-row gap quals
    and N bases, multi-pass reads of different pass counts (whose pairing as
    leftovers depends on the batch), one-base haplotypes."""
    rng = np.random.default_rng(31)
    regs = []
    stream = workloads.make_workload("stream", scale=0.012)
    for g in range(len(stream.regions)):
        regs.append(stream.region(g))
    for g in range(6):
        regs.append(workloads.random_region(rng, int(rng.integers(1, 40)),
                                            int(rng.integers(1, 12)), n_rate=0.01))
    for L in (300, 520, 700, 1100):
        hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L + 60)]
        read = hap[30:30 + L].copy()
        regs.append(([hap], [read], [rng.integers(25, 41, L).astype(np.uint8)],
                     [np.full(L, 45, np.uint8)], [np.full(L, 45, np.uint8)],
                     [np.full(L, 10, np.uint8)]))
    regs.append(([b"A", b"C"], [b"ACG", b"T"], [[30] * 3, [30]], [[45] * 3, [45]],
                 [[45] * 3, [45]], [[10] * 3, [10]]))
    return regs


def test_results_do_not_depend_on_batching():
    regs = mixed_regions()
    whole = Batch.from_regions(regs)
    singles = [Batch.from_regions([r]) for r in regs]
    eng = Engine(0)
    ref_engine = eng.batch(whole)
    eng.close()

    sv = Service(0)
    # 1. one request with everything
    t = sv.submit(whole)
    got_whole = sv.wait(t)
    # 2. each region alone: submit, wait, next
    got_alone = np.concatenate([sv.wait(sv.submit(b)) for b in singles])
    # 3. all regions as separate requests from two threads at once: the
    #    worker batches whatever is queued when a slot frees up
    tickets = [None] * len(singles)

    def submit(k0):
        for k in range(k0, len(singles), 2):
            tickets[k] = sv.submit(singles[k])

    th = [threading.Thread(target=submit, args=(k,)) for k in (0, 1)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    outs = [sv.wait(t, stats=True) for t in tickets]
    got_mixed = np.concatenate([o for o, _ in outs])
    batch_sizes = {s["batch_id"]: s["batch_regions"] for _, s in outs}
    st = sv.stats()
    sv.close()

    assert np.array_equal(got_whole, ref_engine)
    assert np.array_equal(got_alone, ref_engine)
    assert np.array_equal(got_mixed, ref_engine)
    # results are also right, not just stable
    ref = oracle.batch_log10(whole)
    fin = np.isfinite(ref)
    assert np.array_equal(np.isfinite(ref_engine), fin)
    assert np.abs(ref_engine[fin] - ref[fin]).max() < TOL
    n_req = 1 + 2 * len(singles)
    assert st["submitted"] == st["completed"] == n_req and st["failed"] == 0
    assert st["pairs"] == 3 * whole.num_pairs
    assert 0 < st["latency_p50_ms"] <= st["latency_p99_ms"] <= st["latency_max_ms"]
    assert st["batches"] >= 2 and len(batch_sizes) >= 1


def test_admission_bad_input_and_tickets():
    sv = Service(0, device_memory_budget=1 << 16)  # 32 KB per batch slot
    rng = np.random.default_rng(5)
    big = Batch.from_regions([workloads.random_region(rng, 4, 60, read_len=(150, 150))])
    with pytest.raises(RodvError) as ei:
        sv.submit(big)
    assert ei.value.status == 9  # RODV_ERR_ADMISSION
    small = Batch.from_regions([workloads.random_region(rng, 2, 3, hap_len=(20, 40),
                                                        read_len=(10, 30))])
    bad = Batch.from_regions([([b"ACGU"], [b"ACG"], [[30] * 3], [[45] * 3], [[45] * 3],
                               [[10] * 3])])
    with pytest.raises(RodvError) as ei:
        sv.submit(bad)
    assert ei.value.status == 3  # RODV_ERR_INVALID_BASE
    t = sv.submit(small)
    out, rs = sv.wait(t, stats=True)
    assert np.abs(out - oracle.batch_log10(small)).max() < TOL
    assert rs["pairs"] == small.num_pairs and rs["latency_ms"] >= rs["queue_ms"] >= 0
    with pytest.raises(RodvError) as ei:
        sv.poll(t)  # results are handed out once
    assert ei.value.status == 10  # RODV_ERR_NOT_FOUND
    with pytest.raises(RodvError) as ei:
        sv.poll(123456789)
    assert ei.value.status == 10
    sv.reset_stats()
    assert sv.stats()["submitted"] == 0
    sv.close()


def test_close_finishes_submitted_work():
    b = workloads.make_workload("tiny", scale=2.0)
    sv = Service(0)
    tickets = [sv.submit(b.subset([g])) for g in range(len(b.regions))]
    # wait for the last one only; the service must still hand out the others
    last = sv.wait(tickets[-1])
    assert last is not None
    outs = [sv.wait(t) for t in tickets[:-1]] + [last]
    sv.close()
    assert np.array_equal(np.concatenate(outs), Engine(0).batch(b))
