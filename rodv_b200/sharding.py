"""Sharding a batch's regions over several GPUs (one engine per device).

Regions are independent (no exchange step), so a batch splits into one
sub-batch per device with no collective on the data path.  The plan and the
merge are the library's own host-only C entry points (``rodv_shard_plan``,
``rodv_shard_merge``, rodv_b200/csrc/multi.cpp): regions are assigned
longest-processing-time first by their cell count (sum of read_len x hap_len
over their pairs), which balances the devices' work to within one region's
cells, and every process of a multi-process job computes the same plan.  Each
device computes its shard; :func:`merge_results` puts the results back in
the batch's own order (hap-major per region, regions in order).
``rodv_multi_batch`` (:class:`rodv_b200.MultiEngine`) does all three steps in
one call with one host thread per device.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import numpy as np

from . import _lib
from .batch import Batch


def region_cells(batch: Batch) -> np.ndarray:
    """Cells of every region: (sum of its haplotype lengths) x (sum of its read lengths)."""
    hl = batch.hap_lengths.astype(np.int64)
    rl = batch.read_lengths.astype(np.int64)
    hcum = np.concatenate([[0], np.cumsum(hl)])
    rcum = np.concatenate([[0], np.cumsum(rl)])
    r = batch.regions
    hs = hcum[r["hap_start"] + r["num_haps"]] - hcum[r["hap_start"]]
    rs = rcum[r["read_start"] + r["num_reads"]] - rcum[r["read_start"]]
    return hs * rs


def _check(st: int, what: str) -> None:
    if st != _lib.RODV_OK:
        raise _lib.RodvError(st, what)


def shard_plan(batch: Batch, world: int):
    """(shard index of every region, cells per shard) from rodv_shard_plan."""
    from . import _CBatchHolder
    if world < 1:
        raise ValueError("world must be >= 1")
    lib = _lib.load()
    holder = _CBatchHolder(batch)
    assign = np.empty(batch.num_regions, dtype=np.uint32)
    cells = np.empty(world, dtype=np.uint64)
    _check(lib.rodv_shard_plan(ctypes.byref(holder.c), world,
                               assign.ctypes.data_as(_lib._u32p),
                               cells.ctypes.data_as(_lib._u64p)), "rodv_shard_plan")
    return assign, cells


def shard_regions(batch: Batch, world: int) -> List[List[int]]:
    """Region indices per shard (each list ascending), balanced by cells (LPT)."""
    assign, _ = shard_plan(batch, world)
    return [np.nonzero(assign == k)[0].astype(int).tolist() for k in range(world)]


def merge_results(batch: Batch, shards: Sequence[Sequence[int]],
                  results: Sequence[np.ndarray]) -> np.ndarray:
    """The batch's flat results from per-shard results (each in its shard's
    region order, as computing ``batch.subset(shard)`` gives them), through
    rodv_shard_merge."""
    from . import _CBatchHolder
    lib = _lib.load()
    world = len(shards)
    assign = np.full(batch.num_regions, world, dtype=np.uint32)
    off = batch.out_offsets()
    for k, regs in enumerate(shards):
        regs = list(regs)
        if regs != sorted(regs):
            raise ValueError("shard region lists must be ascending")
        assign[regs] = k
        n = int(sum(int(off[g + 1] - off[g]) for g in regs))
        if len(results[k]) != n:
            raise ValueError("shard result length does not match its regions")
    if np.any(assign == world):
        raise ValueError("every region must belong to one shard")
    res = [np.ascontiguousarray(r, dtype=np.float64) for r in results]
    ptrs = (_lib._f64p * world)(*[r.ctypes.data_as(_lib._f64p) for r in res])
    out = np.empty(int(off[-1]), dtype=np.float64)
    holder = _CBatchHolder(batch)
    _check(lib.rodv_shard_merge(ctypes.byref(holder.c), world, assign.ctypes.data_as(_lib._u32p),
                                ptrs, out.ctypes.data_as(_lib._f64p)), "rodv_shard_merge")
    return out
