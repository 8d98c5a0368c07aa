"""Reader of roDV's assemble-log PairHMM dumps (the format its assembler
writes and src/core/test/assemble_log_parser.cpp:13-149 reads) into a
:class:`Batch`, so that logged real regions can be replayed on the engine.

Format, per region::

    === Region: <name> ===
    Haplotypes: <M>
    Reads: <N>

    H0: <bases>
    ...
    R0: <bases>
      read-qual: <ints>
      read-ins-qual: <ints>
      read-del-qual: <ints>
      gcp: <ints>
    ...

Blank lines between blocks are ignored.  A read whose four quality lines do
not all match its length is dropped (as the reference's test drops it), and
counted in the region's ``skipped_reads``.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field
from typing import Iterable, List, Tuple

import numpy as np

from .batch import Batch

_REGION = re.compile(r"^=== Region: (.*) ===\s*$")
_COUNT = re.compile(r"^(Haplotypes|Reads): (\d+)\s*$")
_QUAL_KEYS = {"read-qual": 0, "read-ins-qual": 1, "read-del-qual": 2, "gcp": 3}


@dataclass
class LoggedRegion:
    name: str
    haps: List[bytes] = field(default_factory=list)
    reads: List[bytes] = field(default_factory=list)
    quals: List[Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]] = field(
        default_factory=list)
    skipped_reads: int = 0

    def as_batch_region(self):
        """The (haps, reads, quals, ins, dels, gcps) tuple Batch.from_regions takes."""
        return (self.haps, self.reads, [q[0] for q in self.quals], [q[1] for q in self.quals],
                [q[2] for q in self.quals], [q[3] for q in self.quals])


def parse_lines(lines: Iterable[str]) -> List[LoggedRegion]:
    regions: List[LoggedRegion] = []
    cur = None
    read = None  # [bases, [q, ins, del, gcp]]

    def close_read():
        nonlocal read
        if read is None:
            return
        seq, qs = read
        if all(q is not None and len(q) == len(seq) for q in qs):
            cur.reads.append(seq)
            cur.quals.append(tuple(qs))
        else:
            cur.skipped_reads += 1
        read = None

    for raw in lines:
        line = raw.rstrip("\n")
        m = _REGION.match(line)
        if m:
            if cur is not None:
                close_read()
            cur = LoggedRegion(m.group(1))
            regions.append(cur)
            continue
        if cur is None or not line.strip():
            continue
        if _COUNT.match(line):
            continue
        s = line.strip()
        key, _, val = s.partition(":")
        if key.startswith("H") and key[1:].isdigit() and not line.startswith(" "):
            cur.haps.append(val.strip().encode())
        elif key.startswith("R") and key[1:].isdigit() and not line.startswith(" "):
            close_read()
            read = [val.strip().encode(), [None, None, None, None]]
        elif key in _QUAL_KEYS and read is not None:
            read[1][_QUAL_KEYS[key]] = np.array([int(v) for v in val.split()], dtype=np.uint8)
    if cur is not None:
        close_read()
    return regions


def parse_file(path: str) -> List[LoggedRegion]:
    with open(path) as fh:
        return parse_lines(fh)


def to_batch(regions: List[LoggedRegion]) -> Batch:
    """All regions with at least one haplotype and one read, as one batch."""
    return Batch.from_regions([r.as_batch_region() for r in regions if r.haps and r.reads])
