"""rodv_pairhmm_batch_noalloc: the batch call that allocates no device memory.

It serves callers that cannot call cudaMalloc -- code that owns all device
memory through its own allocator or a start-up pool, or that runs where an
allocation would synchronise the device.  Here the test plays that caller: it
allocates the device inputs and output itself (with torch), then calls the
entry point through the C ABI twice in a row, on two different batches, and
checks each result against the allocating entry point rodv_pairhmm_batch
within the parity tolerance of the other GPU tests (1e-5 log10).  The file
is named to be collected last, so that a failure here comes after every other
test has run; it passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from rodv_b200 import _lib, workloads
from rodv_b200.batch import Batch

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _device_struct(b: Batch, torch):
    """A rodv_batch whose arrays live in device memory (allocated by the caller)."""
    keep = {}

    def dev(name, arr):
        t = torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8).copy()).cuda()
        keep[name] = t
        return t.data_ptr()

    c = _lib.CBatch()
    c.num_regions = len(b.regions)
    c.regions = dev("regions", b.regions)
    c.num_haps = len(b.hap_lengths)
    c.hap_bases = ctypes.cast(dev("hb", b.hap_bases), _lib._u8p)
    c.hap_offsets = ctypes.cast(dev("ho", b.hap_offsets), _lib._u64p)
    c.hap_lengths = ctypes.cast(dev("hl", b.hap_lengths), _lib._u32p)
    c.num_reads = len(b.read_lengths)
    c.read_bases = ctypes.cast(dev("rb", b.read_bases), _lib._u8p)
    c.base_quals = ctypes.cast(dev("q", b.base_quals), _lib._u8p)
    c.ins_quals = ctypes.cast(dev("i", b.ins_quals), _lib._u8p)
    c.del_quals = ctypes.cast(dev("d", b.del_quals), _lib._u8p)
    c.gcp_quals = ctypes.cast(dev("c", b.gcp_quals), _lib._u8p)
    c.read_offsets = ctypes.cast(dev("ro", b.read_offsets), _lib._u64p)
    c.read_lengths = ctypes.cast(dev("rl", b.read_lengths), _lib._u32p)
    return c, keep


def _batches():
    first = workloads.make_workload("tiny", scale=3.0)
    rng = np.random.default_rng(5)
    regs = []
    for L, H in ((300, 400), (40, 2000), (700, 900)):   # multi-pass reads, long haps
        hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, H)]
        read = hap[30:30 + L].copy()
        regs.append(([hap, hap[::-1].copy()], [read], [rng.integers(20, 41, L).astype(np.uint8)],
                     [rng.integers(30, 50, L).astype(np.uint8)],
                     [rng.integers(30, 50, L).astype(np.uint8)],
                     [rng.integers(5, 15, L).astype(np.uint8)]))
    second = Batch.from_regions(regs + [workloads.random_region(rng, 3, 5, n_rate=0.02)])
    return first, second


def test_noalloc_matches_allocating_call_twice(engine):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    for use_double, batch in zip((0, 0), _batches()):
        expected = engine.batch(batch, use_double=bool(use_double))
        cb, keep = _device_struct(batch, torch)
        out = torch.full((batch.num_pairs,), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.rodv_pairhmm_batch_noalloc(ctypes.byref(cb), use_double, out.data_ptr(), None)
        assert st == 0, _lib.STATUS_NAMES.get(st, st)
        got = out.cpu().numpy()
        fin = np.isfinite(expected)
        assert np.array_equal(got[~fin], expected[~fin])
        assert np.abs(got[fin] - expected[fin]).max() < TOL
        del keep


def test_noalloc_fp64_and_limits(engine):
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    batch = workloads.make_workload("tiny", scale=1.0)
    expected = engine.batch(batch, use_double=True)
    cb, keep = _device_struct(batch, torch)
    out = torch.empty((batch.num_pairs,), dtype=torch.float64, device="cuda")
    assert lib.rodv_pairhmm_batch_noalloc(ctypes.byref(cb), 1, out.data_ptr(), None) == 0
    assert np.abs(out.cpu().numpy() - expected).max() < 1e-9
    cb.num_reads = 16385   # above RODV_NOALLOC_MAX_READS: rejected before any launch
    assert lib.rodv_pairhmm_batch_noalloc(ctypes.byref(cb), 0, out.data_ptr(), None) == 7
    del keep


def _one_region(L=120, H=300, seed=9):
    rng = np.random.default_rng(seed)
    hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, H)]
    read = hap[10:10 + L].copy()
    q = [rng.integers(10, 41, L).astype(np.uint8), np.full(L, 45, np.uint8),
         np.full(L, 45, np.uint8), np.full(L, 10, np.uint8)]
    return Batch.from_regions([([hap, hap[::-1].copy()], [read, read[::-1].copy()], *[[x, x]
                                                                                    for x in q])])


def _faulty(kind):
    """A small batch with one fault the device-side checks must catch (every
    array stays in bounds: the checks refuse the batch before any kernel
    reads past what the caller passed)."""
    b = _one_region()
    if kind == "base":          # a base outside A, C, G, T, N
        b.read_bases[3] = ord("X")
    elif kind == "empty":       # a region without reads
        b.regions[0]["num_reads"] = 0
    elif kind == "index":       # a region indexing past the haplotype array
        b.regions[0]["num_haps"] = 3
    elif kind == "zero":        # an empty read
        b.read_lengths[1] = 0
    elif kind == "hap_len":     # a haplotype above RODV_NOALLOC_MAX_HAP_LEN
        rng = np.random.default_rng(3)
        long_hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 2100)]
        b = Batch.from_regions([([long_hap], [long_hap[:100].copy()], [np.full(100, 30, np.uint8)],
                                 [np.full(100, 45, np.uint8)], [np.full(100, 45, np.uint8)],
                                 [np.full(100, 10, np.uint8)])])
    elif kind == "read_len":    # one read above RODV_MAX_READ_LEN (65,536 bases)
        rng = np.random.default_rng(4)
        L = 70000
        hap = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 400)]
        read = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L)]
        b = Batch.from_regions([([hap], [read], [np.full(L, 30, np.uint8)],
                                 [np.full(L, 45, np.uint8)], [np.full(L, 45, np.uint8)],
                                 [np.full(L, 10, np.uint8)])])
    return b


# status codes of include/rodv_pairhmm.h
_EXPECTED = {"base": 3, "empty": 2, "index": 1, "zero": 1, "hap_len": 7, "read_len": 7}


def test_noalloc_device_checks_then_valid_call(engine):
    """Each device-side check maps its fault to the documented status; a host
    array is refused before any launch; a valid call afterwards still matches
    rodv_pairhmm_batch."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    for kind, status in _EXPECTED.items():
        b = _faulty(kind)
        cb, keep = _device_struct(b, torch)
        n = max(1, int(np.sum(b.regions["num_haps"].astype(np.int64) *
                              b.regions["num_reads"].astype(np.int64))))
        out = torch.empty((n,), dtype=torch.float64, device="cuda")
        st = lib.rodv_pairhmm_batch_noalloc(ctypes.byref(cb), 0, out.data_ptr(), None)
        assert st == status, (kind, _lib.STATUS_NAMES.get(st, st))
        del keep
    # host arrays (what the other entry points take) are refused, nothing launched
    from rodv_b200 import _CBatchHolder
    good = _one_region()
    holder = _CBatchHolder(good)
    out = torch.empty((good.num_pairs,), dtype=torch.float64, device="cuda")
    assert lib.rodv_pairhmm_batch_noalloc(ctypes.byref(holder.c), 0, out.data_ptr(), None) == 1
    # and a valid call still gives the allocating call's results
    expected = engine.batch(good)
    cb, keep = _device_struct(good, torch)
    assert lib.rodv_pairhmm_batch_noalloc(ctypes.byref(cb), 0, out.data_ptr(), None) == 0
    assert np.abs(out.cpu().numpy() - expected).max() < TOL
    del keep
