"""Flat host-side batch of PairHMM regions, laid out like ``rodv_batch``.

A region is the unit of roDV's ``schedule_pairhmm`` call
(src/core/pairhmm_schedule.h:14-25): M haplotypes x N reads, each read with
four per-base quality arrays (base, insertion, deletion, gap continuation;
raw Phred integers).  Its result is an M x N matrix of log10 likelihoods,
hap-major (``result[h][r]``, pairhmm_schedule.cpp:134-138).

A :class:`Batch` concatenates many regions into the flat arrays that the
C ABI in ``include/rodv_pairhmm.h`` takes: one byte buffer for all
haplotype bases, one per read field, offset and length arrays, and a region
table.  Results of region g start at ``out_offsets()[g]``.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

REGION_DTYPE = np.dtype([("hap_start", "<u4"), ("num_haps", "<u4"), ("read_start", "<u4"),
                         ("num_reads", "<u4")])


def _as_u8(x) -> np.ndarray:
    if isinstance(x, np.ndarray):
        return np.ascontiguousarray(x, dtype=np.uint8)
    if isinstance(x, str):
        x = x.encode()
    return np.frombuffer(bytes(bytearray(x)), dtype=np.uint8)


@dataclass
class Batch:
    regions: np.ndarray          # REGION_DTYPE[num_regions]
    hap_bases: np.ndarray        # u8, ASCII A/C/G/T/N
    hap_offsets: np.ndarray      # u64[num_haps]
    hap_lengths: np.ndarray      # u32[num_haps]
    read_bases: np.ndarray       # u8, ASCII A/C/G/T/N
    base_quals: np.ndarray       # u8, raw Phred, same offsets as read_bases
    ins_quals: np.ndarray
    del_quals: np.ndarray
    gcp_quals: np.ndarray
    read_offsets: np.ndarray     # u64[num_reads]
    read_lengths: np.ndarray     # u32[num_reads]

    @property
    def num_regions(self) -> int:
        return len(self.regions)

    @property
    def num_pairs(self) -> int:
        return int((self.regions["num_haps"].astype(np.uint64) *
                    self.regions["num_reads"].astype(np.uint64)).sum())

    def out_offsets(self) -> np.ndarray:
        n = (self.regions["num_haps"].astype(np.uint64) *
             self.regions["num_reads"].astype(np.uint64))
        off = np.zeros(len(n) + 1, dtype=np.uint64)
        np.cumsum(n, out=off[1:])
        return off

    def cells(self) -> int:
        """Sum over all pairs of read_len * hap_len (real cells, no padding)."""
        total = 0
        hl = self.hap_lengths.astype(np.int64)
        rl = self.read_lengths.astype(np.int64)
        hs = np.zeros(len(hl) + 1, dtype=np.int64)
        np.cumsum(hl, out=hs[1:])
        rs = np.zeros(len(rl) + 1, dtype=np.int64)
        np.cumsum(rl, out=rs[1:])
        r = self.regions
        h0 = r["hap_start"].astype(np.int64)
        h1 = h0 + r["num_haps"]
        r0 = r["read_start"].astype(np.int64)
        r1 = r0 + r["num_reads"]
        total = int(((hs[h1] - hs[h0]) * (rs[r1] - rs[r0])).sum())
        return total

    def input_bytes(self) -> int:
        return int(self.hap_bases.nbytes + 5 * self.read_bases.nbytes)

    def region(self, g: int):
        """Region g as the reference's vector-of-vectors arguments."""
        rg = self.regions[g]
        haps = [bytes(self.hap_bases[self.hap_offsets[h]:self.hap_offsets[h] +
                                     self.hap_lengths[h]])
                for h in range(rg["hap_start"], rg["hap_start"] + rg["num_haps"])]
        fields = []
        for arr in (self.read_bases, self.base_quals, self.ins_quals, self.del_quals,
                    self.gcp_quals):
            fields.append([arr[self.read_offsets[r]:self.read_offsets[r] +
                               self.read_lengths[r]].copy()
                           for r in range(rg["read_start"], rg["read_start"] + rg["num_reads"])])
        return haps, fields[0], fields[1], fields[2], fields[3], fields[4]

    @staticmethod
    def from_regions(regions: Sequence[tuple]) -> "Batch":
        """Builds a batch from ``(haps, reads, quals, ins, dels, gcps)`` tuples.

        Every element may be ``str``/``bytes``/list of ints/``np.ndarray``.
        """
        hap_list: List[np.ndarray] = []
        read_fields: List[List[np.ndarray]] = [[], [], [], [], []]
        reg = np.zeros(len(regions), dtype=REGION_DTYPE)
        for g, (haps, reads, quals, ins, dels, gcps) in enumerate(regions):
            reg[g] = (len(hap_list), len(haps), len(read_fields[0]), len(reads))
            hap_list.extend(_as_u8(h) for h in haps)
            for k, col in enumerate((reads, quals, ins, dels, gcps)):
                read_fields[k].extend(_as_u8(x) for x in col)
        return Batch._pack(reg, hap_list, read_fields)

    @staticmethod
    def _pack(reg, hap_list, read_fields) -> "Batch":
        hl = np.array([len(h) for h in hap_list], dtype=np.uint32)
        ho = np.zeros(len(hap_list), dtype=np.uint64)
        if len(hl):
            ho[1:] = np.cumsum(hl[:-1], dtype=np.uint64)
        rl = np.array([len(r) for r in read_fields[0]], dtype=np.uint32)
        for k in range(1, 5):
            for r, x in enumerate(read_fields[k]):
                if len(x) != rl[r]:
                    raise ValueError(f"read {r}: quality array {k} has length {len(x)}, "
                                     f"read has {rl[r]}")
        ro = np.zeros(len(rl), dtype=np.uint64)
        if len(rl):
            ro[1:] = np.cumsum(rl[:-1], dtype=np.uint64)

        def cat(lst):
            return (np.concatenate(lst).astype(np.uint8) if lst else np.zeros(0, np.uint8))

        return Batch(reg, cat(hap_list), ho, hl, cat(read_fields[0]), cat(read_fields[1]),
                     cat(read_fields[2]), cat(read_fields[3]), cat(read_fields[4]), ro, rl)

    def subset(self, region_ids: Sequence[int]) -> "Batch":
        """A new batch holding only the given regions (in that order)."""
        regs = []
        for g in region_ids:
            haps, reads, q, i, d, c = self.region(int(g))
            regs.append((haps, reads, q, i, d, c))
        return Batch.from_regions(regs)
