"""Sharding a batch's regions over several GPUs (one engine per device).

Regions are independent (no exchange step), so a batch splits into one
sub-batch per device with no collective on the data path.  Regions are
assigned longest-processing-time first by their cell count (sum of
read_len x hap_len over their pairs), which balances the devices' work to
within one region's cells.  Each device computes its shard; the results are
put back in the batch's own order (hap-major per region, regions in order)
with :func:`merge_results`.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np

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


def shard_regions(batch: Batch, world: int) -> List[List[int]]:
    """Region indices per shard (each list ascending), balanced by cells (LPT)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cells = region_cells(batch)
    order = np.argsort(-cells, kind="stable")
    heap = [(0, k) for k in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for g in order:
        load, k = heapq.heappop(heap)
        shards[k].append(int(g))
        heapq.heappush(heap, (load + int(cells[g]), k))
    return [sorted(s) for s in shards]


def merge_results(batch: Batch, shards: Sequence[Sequence[int]],
                  results: Sequence[np.ndarray]) -> np.ndarray:
    """The batch's flat results from per-shard results (each in its shard's
    region order, as computing ``batch.subset(shard)`` gives them)."""
    off = batch.out_offsets()
    out = np.empty(int(off[-1]), dtype=np.float64)
    for regs, res in zip(shards, results):
        pos = 0
        for g in regs:
            n = int(off[g + 1] - off[g])
            out[int(off[g]):int(off[g]) + n] = res[pos:pos + n]
            pos += n
        if pos != len(res):
            raise ValueError("shard result length does not match its regions")
    return out
