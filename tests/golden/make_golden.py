"""Generates the committed golden fixtures in tests/golden/ from the reference.

Run in a container where the reference tree exists and oracle/_ref is built
(``make -C oracle REF=<roDV>``):

    python tests/golden/make_golden.py [--ref PATH_TO_ROOT_OF_roDV]

Fixtures written (all small, all derived from the reference):

* ``gkl_testdata.tsv``   the 104 lines of roDV's resouces/pairhmm-testdata.txt
  (hap, read, 4 quality strings ASCII+33, expected log10), plus two columns
  with the reference's own intra output run here: FP32 with FP64 rescue, and
  forced FP64 (computeLikelihoodsAVX512, src/core/pairhmm/intra/pairhmm_api.cpp).
* ``assemble_regions.json.gz``  the 8 chrY regions of resouces/pairhmm_debug.txt,
  parsed as the reference's AssembleLogParser does
  (src/core/test/assemble_log_parser.cpp:13-149; reads whose quality arrays do
  not match the read length are skipped, like
  src/core/test/pairhmm_unitest_from_assemble.cpp:88-97), with the outputs of
  the reference's schedule_pairhmm at idle ratios 0.5/0.7 (as that test uses).
* ``synthetic_ref.npz``  seeded synthetic regions with per-row ins/del/gcp quals
  and 'N' bases, with the reference's schedule_pairhmm output and its intra
  output per pair (N semantics are pinned only by these: the golden file has
  no 'N').
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from rodv_b200.batch import Batch  # noqa: E402
from rodv_b200 import workloads  # noqa: E402


def gkl(ref_root: str) -> None:
    src = os.path.join(ref_root, "resouces", "pairhmm-testdata.txt")
    lines = open(src).read().splitlines()
    out = [lines[0] + " ref_intra ref_intra_fp64"]
    for ln in lines[1:]:
        f = ln.split()
        if len(f) < 7:
            continue
        q = [np.frombuffer(s.encode(), np.uint8) - 33 for s in f[2:6]]
        a = oracle.ref_intra(f[0], f[1], *q, use_double=False)
        d = oracle.ref_intra(f[0], f[1], *q, use_double=True)
        out.append(" ".join(f[:7] + [repr(a), repr(d)]))
    with open(os.path.join(HERE, "gkl_testdata.tsv"), "w") as fh:
        fh.write("\n".join(out) + "\n")
    print(f"gkl_testdata.tsv: {len(out) - 1} cases")


def parse_assemble(path: str):
    """Regions of an assemble log, field for field like AssembleLogParser."""
    regions = []
    lines = open(path).read().splitlines()
    i = 0
    while i < len(lines):
        if "=== Region:" not in lines[i]:
            i += 1
            continue
        name = lines[i].split("=== Region:")[1].strip(" =")
        nh = int(lines[i + 1].split(":")[1])
        nr = int(lines[i + 2].split(":")[1])
        i += 4
        haps = []
        for _ in range(nh):
            haps.append(lines[i].split(":", 1)[1].strip())
            i += 1
        i += 1
        reads = []
        for _ in range(nr):
            seq = lines[i].split(":", 1)[1].strip()
            i += 1
            quals = {}
            while len(quals) < 4 and i < len(lines) and "=== Region:" not in lines[i]:
                ln = lines[i].strip()
                i += 1
                if not ln:
                    continue
                key, vals = ln.split(":", 1)
                quals[key.strip()] = [int(v) for v in vals.split()]
            reads.append((seq, quals))
        regions.append((name, haps, reads))
    return regions


def assemble(ref_root: str) -> None:
    regs = parse_assemble(os.path.join(ref_root, "resouces", "pairhmm_debug.txt"))
    out = []
    tuples = []
    for name, haps, reads in regs:
        keep = [(s, q) for s, q in reads
                if all(len(q.get(k, [])) == len(s)
                       for k in ("read-qual", "read-ins-qual", "read-del-qual", "gcp"))]
        rec = {"region": name, "haps": haps, "reads": [s for s, _ in keep],
               "q": [q["read-qual"] for _, q in keep], "ins": [q["read-ins-qual"] for _, q in keep],
               "del": [q["read-del-qual"] for _, q in keep], "gcp": [q["gcp"] for _, q in keep],
               "skipped_reads": len(reads) - len(keep)}
        out.append(rec)
        tuples.append((haps, rec["reads"], rec["q"], rec["ins"], rec["del"], rec["gcp"]))
    b = Batch.from_regions(tuples)
    res = oracle.ref_schedule(b, ratio_f=0.5, ratio_d=0.7, threads=4)
    off = b.out_offsets()
    for g, rec in enumerate(out):
        rec["ref_schedule"] = [float(x) for x in res[off[g]:off[g + 1]]]
    with gzip.open(os.path.join(HERE, "assemble_regions.json.gz"), "wt") as fh:
        json.dump(out, fh)
    print(f"assemble_regions.json.gz: {len(out)} regions, {int(off[-1])} pairs")


def synthetic() -> None:
    rng = np.random.default_rng(20241203)
    regs = []
    for k in range(12):
        nh, nr = int(rng.integers(1, 6)), int(rng.integers(1, 9))
        regs.append(workloads.random_region(rng, nh, nr, hap_len=(8, 400), read_len=(1, 300),
                                            vary_gap_quals=(k % 2 == 0),
                                            n_rate=0.03 if k % 3 == 0 else 0.0))
    b = Batch.from_regions(regs)
    sched = oracle.ref_schedule(b, threads=4)
    intra = np.empty_like(sched)
    off = b.out_offsets()
    for g in range(b.num_regions):
        haps, reads, q, i, d, c = b.region(g)
        for h in range(len(haps)):
            for r in range(len(reads)):
                intra[off[g] + h * len(reads) + r] = oracle.ref_intra(haps[h], reads[r], q[r], i[r],
                                                                      d[r], c[r])
    np.savez_compressed(os.path.join(HERE, "synthetic_ref.npz"), regions=b.regions,
                        hap_bases=b.hap_bases, hap_offsets=b.hap_offsets,
                        hap_lengths=b.hap_lengths, read_bases=b.read_bases,
                        base_quals=b.base_quals, ins_quals=b.ins_quals, del_quals=b.del_quals,
                        gcp_quals=b.gcp_quals, read_offsets=b.read_offsets,
                        read_lengths=b.read_lengths, ref_schedule=sched, ref_intra=intra)
    print(f"synthetic_ref.npz: {b.num_regions} regions, {b.num_pairs} pairs, "
          f"{int((b.read_bases == ord('N')).sum() + (b.hap_bases == ord('N')).sum())} N bases")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None,
                    help="roDV source tree (default: oracle.default_reference_dir())")
    a = ap.parse_args()
    a.ref = a.ref or oracle.default_reference_dir()
    if not oracle.ref_available():
        oracle.build(a.ref)
    gkl(a.ref)
    assemble(a.ref)
    synthetic()


if __name__ == "__main__":
    main()
