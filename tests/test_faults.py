"""Allocation failures on the host: every entry point that allocates returns
RODV_ERR_OUT_OF_MEMORY, releases what it had allocated, and leaves the
engine usable.

The failure is made on the host by the library's testing hook
(rodv_fault_inject_alloc): the n-th next device (cudaMalloc) or pinned-host
(cudaMallocHost) allocation fails exactly as an exhausted one would.  No GPU
memory is actually exhausted and nothing faults on the device.
rodv_debug_live_allocations counts the library's live allocations, so each
test checks that a failed call left none behind."""
import ctypes

import numpy as np
import pytest

from rodv_b200 import Engine, RodvError, Service, _CBatchHolder, _lib, workloads

pytestmark = pytest.mark.gpu
OOM = 6
DEVICE, PINNED = 0, 1


def _live():
    d, p = ctypes.c_uint64(), ctypes.c_uint64()
    _lib.load().rodv_debug_live_allocations(ctypes.byref(d), ctypes.byref(p))
    return d.value, p.value


class _Fault:
    """Arms the n-th next allocation of `kind` to fail; disarms on exit."""

    def __init__(self, kind, nth=1):
        self.kind, self.nth = kind, nth

    def __enter__(self):
        assert _lib.load().rodv_fault_inject_alloc(self.kind, self.nth) == 0
        return self

    def __exit__(self, *exc):
        _lib.load().rodv_fault_inject_alloc(self.kind, 0)


@pytest.fixture(scope="module")
def batch():
    return workloads.make_workload("tiny", scale=2.0)


@pytest.mark.parametrize("kind", [DEVICE, PINNED])
def test_batch_call_out_of_memory_then_recovers(engine, batch, kind):
    want = engine.batch(batch)
    before = _live()
    eng = Engine(0)
    with _Fault(kind):
        with pytest.raises(RodvError) as ei:
            eng.batch(batch)
    assert ei.value.status == OOM
    assert "out of memory" in str(ei.value).lower() or "allocation" in str(ei.value).lower()
    # the same engine computes the batch afterwards, with the same results
    assert np.array_equal(eng.batch(batch), want)
    eng.close()
    assert _live() == before


def test_every_nth_allocation_of_a_call_fails_cleanly(engine, batch):
    """Failing the 1st, 2nd, ... allocation of a fresh engine's first call:
    each failure is reported as out of memory and, once the engine is closed,
    no allocation of the library is left alive."""
    want = engine.batch(batch)
    base = _live()
    for kind in (DEVICE, PINNED):
        for nth in range(1, 6):
            eng = Engine(0)
            with _Fault(kind, nth):
                try:
                    got = eng.batch(batch)
                    failed = False
                except RodvError as e:
                    assert e.status == OOM, (kind, nth, e)
                    failed = True
            if not failed:  # fewer than nth allocations in the call
                assert np.array_equal(got, want)
            assert np.array_equal(eng.batch(batch), want)
            eng.close()
            assert _live() == base, (kind, nth, _live(), base)


def test_device_batch_upload_out_of_memory(engine, batch):
    lib = _lib.load()
    base = _live()
    holder = _CBatchHolder(batch)
    h = ctypes.c_void_p()
    with _Fault(DEVICE):
        st = lib.rodv_device_batch_upload(engine.h, ctypes.byref(holder.c), ctypes.byref(h))
    assert st == OOM and not h.value
    assert _live() == base
    db = engine.upload(batch)  # works again
    db.run()
    assert np.array_equal(db.download(), engine.batch(batch))
    db.free()
    assert _live() == base


@pytest.mark.parametrize("kind", [DEVICE, PINNED])
def test_service_create_out_of_memory(kind):
    base = _live()
    with _Fault(kind, 2):  # past the engine's own table allocation
        with pytest.raises(RodvError) as ei:
            Service(0)
    assert ei.value.status == OOM
    assert _live() == base
    sv = Service(0)  # creation works again
    sv.close()
    assert _live() == base


@pytest.mark.parametrize("use_double", [False, True])
def test_pipelined_wait_expiry_is_reported_and_device_stays_usable(engine, use_double):
    """Long reads' multi-pass sweeps run one item's passes on several warps
    that wait for one another's published progress, each wait bounded.  With
    the testing hook on, nothing is published: every wait runs out, the kernel
    records kErrWaitTimeout and returns, the call fails with
    RODV_ERR_DEVICE_CHECK, and the same engine then computes the batch
    correctly (no hang, no fault, the context stays usable)."""
    b = workloads.make_workload("long", scale=0.002)   # 4 long pairs, several passes each
    want = engine.batch(b, use_double=use_double)
    lib = _lib.load()
    assert lib.rodv_fault_inject_wait(1) == 0
    try:
        with pytest.raises(RodvError) as ei:
            engine.batch(b, use_double=use_double)
    finally:
        lib.rodv_fault_inject_wait(0)
    assert ei.value.status == 8, ei.value       # RODV_ERR_DEVICE_CHECK
    assert "error flags 16" in str(ei.value)     # kErrWaitTimeout
    assert np.array_equal(engine.batch(b, use_double=use_double), want)
