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
