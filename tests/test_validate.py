"""Host-side input faults, checked without a device through
rodv_batch_validate, which applies the rules the compute calls apply.  The
reference checks only M == 0 or N == 0 (src/core/pairhmm_schedule.cpp:130-132)
and reads other invalid input out of bounds (a lowercase base indexes past
ConvertChar's table, src/core/common.h:42-56); the engine rejects it with a
status and a description instead."""
import ctypes

import numpy as np
import pytest

from rodv_b200 import RodvError, _lib, validate_batch, workloads
from rodv_b200.batch import Batch


def region(hap="ACGTACGTAC", read="ACGTA"):
    q = np.full(len(read), 30, np.uint8)
    return ([hap], [read], [q], [q], [q], [q])


def status_of(b):
    try:
        validate_batch(b)
    except RodvError as e:
        return e.status, str(e)
    return _lib.RODV_OK, ""


def test_valid_batches_pass():
    validate_batch(workloads.make_workload("tiny", scale=2.0))
    validate_batch(Batch.from_regions([region("ACGTNNACGT", "NNACG")]))  # N on either side


@pytest.mark.parametrize("hap,read", [("ACGTacgt", "ACGT"), ("ACGT", "ACxT"), ("ACG-T", "ACG")])
def test_bases_outside_acgtn_are_rejected(hap, read):
    st, msg = status_of(Batch.from_regions([region(hap, read)]))
    assert st == 3 and "A, C, G, T, N" in msg  # RODV_ERR_INVALID_BASE


def test_region_without_haplotypes_or_reads_is_rejected():
    st, msg = status_of(Batch.from_regions([region(), ([], ["ACG"], [np.full(3, 30, np.uint8)],
                                                        [np.full(3, 45, np.uint8)],
                                                        [np.full(3, 45, np.uint8)],
                                                        [np.full(3, 10, np.uint8)])]))
    assert st == 2 and "region 1" in msg  # RODV_ERR_EMPTY
    st, _ = status_of(Batch.from_regions([(["ACGT"], [], [], [], [], [])]))
    assert st == 2


def test_empty_sequences_are_rejected():
    st, msg = status_of(Batch.from_regions([region(hap="")]))
    assert st == 1 and "haplotype 0 is empty" in msg  # RODV_ERR_INVALID_ARG
    st, msg = status_of(Batch.from_regions([region(read="")]))
    assert st == 1 and "read 0 is empty" in msg


def test_region_indexing_past_the_arrays_is_rejected():
    b = Batch.from_regions([region(), region()])
    b.regions["num_reads"][1] = 5
    st, msg = status_of(b)
    assert st == 1 and "out of range" in msg


def test_lengths_above_the_limits_are_rejected():
    limit = 65536  # RODV_MAX_READ_LEN and RODV_MAX_HAP_LEN
    st, _ = status_of(Batch.from_regions([region(hap="ACGT", read="A" * (limit + 1))]))
    assert st == 7  # RODV_ERR_TOO_LONG
    st, _ = status_of(Batch.from_regions([region(hap="A" * (limit + 1), read="ACGT")]))
    assert st == 7
    st, _ = status_of(Batch.from_regions([region(hap="A" * limit, read="A" * limit)]))
    assert st == _lib.RODV_OK


def test_null_batch_and_message_buffer_bounds():
    lib = _lib.load()
    msg = ctypes.create_string_buffer(64)
    assert lib.rodv_batch_validate(None, msg, len(msg)) == 1
    assert msg.value == b"null batch"
    # a one-byte buffer gets only the terminating zero; a null one is allowed
    from rodv_b200 import _CBatchHolder
    h = _CBatchHolder(Batch.from_regions([region(hap="ACGTx")]))
    tiny = ctypes.create_string_buffer(b"\x7f", 1)
    assert lib.rodv_batch_validate(ctypes.byref(h.c), tiny, 1) == 3
    assert tiny.raw == b"\x00"
    assert lib.rodv_batch_validate(ctypes.byref(h.c), None, 0) == 3
