"""Seeded synthetic PairHMM workloads with the shapes of the benchmark configs.

The reference publishes no benchmark dataset; these generators produce
seeded stand-ins with the stated shapes, sizes and value distributions:

* ``plain``      1 region, 8 haps of 250-400 bp, 64 reads of 150 bp
* ``uneven``     10,000 regions, 20-200 reads (50-250 bp) x 2-16 haps (100-600 bp);
                 a region's haplotypes are mutated copies of one locus whose
                 length is drawn per region (assembled haplotypes of one
                 active region, as in the reference's resouces/pairhmm_debug.txt)
* ``uneven_windows``  the same shape with each haplotype a random window of
                 its own length (the reference unit-test generator's model):
                 reads from one haplotype's flank do not align to another, so
                 ~27% of pairs fall below the FP32 threshold (FP64 stress)
* ``long``       2,000 pairs, reads 1,000-2,000 bp vs haps 2,000-5,000 bp
* ``underflow``  200,000 pairs, 250 bp reads vs unrelated random 400 bp haps,
                 base quals Phred 2-8
* ``stream``     regions with 1-300 reads (50-250 bp) x 1-32 haps (100-800 bp)

Within a region the haplotypes are mutated copies of one uniform-ACGT base
sequence and reads are mutated substrings of a uniformly chosen haplotype,
the model of the reference's own generator
(src/core/test/pairhmm_schedule_unittest.cpp:244-334); ``uneven`` and
``stream`` copy the whole locus, the others take random windows.  Mutation model:
1% substitutions and 0.1% indels of 1-3 bp per base (5% / 1% for ``long``).
Base quals are uniform Phred 10-40 unless stated; ins = del = 45, gcp = 10.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

from .batch import Batch, REGION_DTYPE

ACGT = np.frombuffer(b"ACGT", dtype=np.uint8)

SEEDS: Dict[str, int] = {"plain": 1001, "uneven": 1002, "long": 1003, "underflow": 1004,
                         "stream": 1005, "tiny": 1006, "uneven_windows": 1007}


def _random_seq(rng: np.random.Generator, n: int) -> np.ndarray:
    return ACGT[rng.integers(0, 4, size=n)]


def _mutate(rng: np.random.Generator, seq: np.ndarray, p_sub: float,
            p_indel: float) -> np.ndarray:
    """Substitutions (always to a different base) and 1-3 bp indels."""
    out = seq.copy()
    n = len(out)
    if n == 0:
        return out
    sub = np.nonzero(rng.random(n) < p_sub)[0]
    if len(sub):
        codes = np.searchsorted(ACGT, out[sub])  # A0 C1 G2 T3 order of ACGT
        out[sub] = ACGT[(codes + rng.integers(1, 4, size=len(sub))) % 4]
    nind = rng.binomial(n, p_indel) if p_indel > 0 else 0
    if nind == 0:
        return out
    pos = np.sort(rng.integers(0, n, size=nind))[::-1]
    lst = out.tolist()
    for p in pos:
        ln = int(rng.integers(1, 4))
        if rng.random() < 0.5:  # insertion after p
            lst[p + 1:p + 1] = _random_seq(rng, ln).tolist()
        else:                   # deletion starting at p
            del lst[p:p + ln]
    return np.array(lst, dtype=np.uint8)


def _quals(rng, n, lo, hi):
    return rng.integers(lo, hi + 1, size=n).astype(np.uint8)


class _Builder:
    def __init__(self):
        self.regions: List[Tuple[int, int, int, int]] = []
        self.haps: List[np.ndarray] = []
        self.reads: List[List[np.ndarray]] = [[], [], [], [], []]

    def add_region(self, haps, reads, quals):
        self.regions.append((len(self.haps), len(haps), len(self.reads[0]), len(reads)))
        self.haps.extend(haps)
        self.reads[0].extend(reads)
        for k in range(4):
            self.reads[k + 1].extend(q[k] for q in quals)

    def build(self) -> Batch:
        reg = np.array(self.regions, dtype=np.uint32).reshape(-1, 4)
        r = np.zeros(len(reg), dtype=REGION_DTYPE)
        for k, name in enumerate(REGION_DTYPE.names):
            r[name] = reg[:, k]
        return Batch._pack(r, self.haps, self.reads)


def _region(rng, n_haps, hap_len_rng, n_reads, read_len_rng, p_sub, p_indel, bq=(10, 40),
            ins=45, dele=45, gcp=10, independent_haps=False, locus=False):
    """One region.  Haplotypes are mutated copies of one base sequence: random
    windows of it with their own lengths (the reference generator's model), or,
    with ``locus``, full copies of one locus whose length is drawn per region."""
    if locus:
        loc_len = int(rng.integers(hap_len_rng[0], hap_len_rng[1] + 1))
        base = _random_seq(rng, loc_len)
        haps = [_mutate(rng, base, p_sub, p_indel) for _ in range(n_haps)]
        haps = [h if len(h) else base.copy() for h in haps]
        hap_lens = None
    else:
        hap_lens = rng.integers(hap_len_rng[0], hap_len_rng[1] + 1, size=n_haps)
        base = _random_seq(rng, int(hap_lens.max()) + 16)
        haps = []
    for hl in (hap_lens if hap_lens is not None else []):
        if independent_haps:
            haps.append(_random_seq(rng, int(hl)))
            continue
        h = _mutate(rng, base, p_sub, p_indel)
        if len(h) < hl:
            h = np.concatenate([h, _random_seq(rng, int(hl) - len(h))])
        start = int(rng.integers(0, len(h) - hl + 1))
        haps.append(h[start:start + int(hl)].copy())
    reads, quals = [], []
    for _ in range(n_reads):
        src = haps[int(rng.integers(0, n_haps))]
        rl = int(rng.integers(read_len_rng[0], read_len_rng[1] + 1))
        rl = min(rl, len(src))
        start = int(rng.integers(0, len(src) - rl + 1))
        rd = _mutate(rng, src[start:start + rl], p_sub, p_indel)
        if len(rd) == 0:
            rd = src[start:start + 1].copy()
        n = len(rd)
        reads.append(rd)
        quals.append((_quals(rng, n, *bq), np.full(n, ins, np.uint8),
                      np.full(n, dele, np.uint8), np.full(n, gcp, np.uint8)))
    return haps, reads, quals


def make_workload(name: str, seed: int | None = None, scale: float = 1.0) -> Batch:
    """Builds the named workload; ``scale`` < 1 shrinks the region/pair count."""
    rng = np.random.default_rng(SEEDS[name] if seed is None else seed)
    b = _Builder()
    if name == "plain":
        haps, reads, quals = _region(rng, 8, (250, 400), 64, (150, 150), 0.01, 0.001)
        b.add_region(haps, reads, quals)
    elif name in ("uneven", "uneven_windows"):
        for _ in range(max(1, int(round(10_000 * scale)))):
            nh = int(rng.integers(2, 17))
            nr = int(rng.integers(20, 201))
            b.add_region(*_region(rng, nh, (100, 600), nr, (50, 250), 0.01, 0.001,
                                  locus=(name == "uneven")))
    elif name == "stream":
        for _ in range(max(1, int(round(1_000 * scale)))):
            nh = int(rng.integers(1, 33))
            nr = int(rng.integers(1, 301))
            b.add_region(*_region(rng, nh, (100, 800), nr, (50, 250), 0.01, 0.001, locus=True))
    elif name == "long":
        for _ in range(max(1, int(round(2_000 * scale)))):
            b.add_region(*_region(rng, 1, (2000, 5000), 1, (1000, 2000), 0.05, 0.01))
    elif name == "underflow":
        for _ in range(max(1, int(round(200_000 * scale)))):
            hap = _random_seq(rng, 400)
            rd = _random_seq(rng, 250)
            b.add_region([hap], [rd], [(_quals(rng, 250, 2, 8), np.full(250, 45, np.uint8),
                                        np.full(250, 45, np.uint8),
                                        np.full(250, 10, np.uint8))])
    elif name == "tiny":
        for _ in range(max(1, int(round(8 * scale)))):
            nh = int(rng.integers(1, 5))
            nr = int(rng.integers(1, 9))
            b.add_region(*_region(rng, nh, (10, 120), nr, (5, 90), 0.02, 0.01, bq=(6, 43)))
    else:
        raise KeyError(f"unknown workload {name!r}")
    return b.build()


def random_region(rng: np.random.Generator, n_haps: int, n_reads: int, hap_len=(30, 300),
                  read_len=(10, 150), vary_gap_quals: bool = True, n_rate: float = 0.0):
    """A region with per-row ins/del/gcp quals (the golden-file style) for tests.

    Returns ``(haps, reads, quals, ins, dels, gcps)`` as Batch.from_regions takes.
    """
    haps, reads, quals = _region(rng, n_haps, hap_len, n_reads, read_len, 0.02, 0.005,
                                 bq=(6, 43))
    if vary_gap_quals:
        quals = [(q[0], _quals(rng, len(q[0]), 6, 43), _quals(rng, len(q[0]), 6, 43),
                  _quals(rng, len(q[0]), 6, 43)) for q in quals]
    if n_rate > 0:
        for s in list(haps) + list(reads):
            s[rng.random(len(s)) < n_rate] = ord("N")
    return (haps, reads, [q[0] for q in quals], [q[1] for q in quals], [q[2] for q in quals],
            [q[3] for q in quals])
