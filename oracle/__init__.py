"""CPU oracle and reference loader for the PairHMM engine's tests.

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg and ``--impl reference`` arm of ``bench.py`` import this
package.  The engine in ``rodv_b200`` never calls it and has no CPU fallback.

* :func:`oracle_lib` loads ``oracle/liboracle.so``, the plain-C restatement in
  ``pairhmm_oracle.c`` (its header cites the reference lines it follows).
* :func:`ref_lib` loads ``oracle/_ref/libref_pairhmm.so``: the reference's own
  ``src/core`` compiled in place by ``oracle/Makefile``, wrapped by
  ``ref_capi.cpp``.  It exists only where the reference tree was present at
  build time; it is then shipped next to the engine as a prebuilt file.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_pairhmm.so")

# Modes of oracle_pair_log10 (pairhmm_oracle.c)
REFERENCE = 0  # FP32, FP64 rescue below 1e-28: the reference's answer
FP64 = 1       # FP64 with 2^1020 scaling for every pair
SCALED = 2     # FP64 with per-row renormalisation: the true value
FP32_RAW = 3   # raw scaled FP32 sum

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)

_oracle: Optional[ctypes.CDLL] = None
_ref: Optional[ctypes.CDLL] = None


def default_reference_dir() -> str:
    """The roDV source tree: $RODV_REFERENCE, else a checkout named
    ``reference`` beside this repository's checkout."""
    return os.environ.get("RODV_REFERENCE") or os.path.normpath(
        os.path.join(HERE, "..", "..", "reference"))


def build(ref_dir: Optional[str] = None, quiet: bool = True) -> None:
    """Compiles liboracle.so, and the reference library when its tree exists."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=out)
    ref_dir = ref_dir or default_reference_dir()
    if os.path.isdir(os.path.join(ref_dir, "src", "core")):
        subprocess.run(["make", "-C", HERE, "ref", f"REF={ref_dir}", "-j8"], check=True,
                       stdout=out)
        # the reference's scheduler tests linked against the engine's
        # schedule_pairhmm (needs rodv_b200/librodv_pairhmm.so)
        if os.path.exists(os.path.join(HERE, "..", "rodv_b200", "librodv_pairhmm.so")):
            subprocess.run(["make", "-C", HERE, "conformance", f"REF={ref_dir}", "-j8"],
                           check=True, stdout=out)


CONFORMANCE_BIN = os.path.join(HERE, "_ref", "ref_schedule_tests_on_rodv")


def write_assemble_log(regions, path: str) -> None:
    """Writes regions (the assemble fixture's dicts: region, haps, reads, q,
    ins, del, gcp) in the format AssembleLogParser reads
    (src/core/test/assemble_log_parser.cpp:13-149)."""
    with open(path, "w") as fh:
        for r in regions:
            fh.write(f"=== Region: {r['region']} ===\n")
            fh.write(f"Haplotypes: {len(r['haps'])}\nReads: {len(r['reads'])}\n\n")
            for k, h in enumerate(r["haps"]):
                fh.write(f"H{k}: {h}\n")
            fh.write("\n")
            for k, seq in enumerate(r["reads"]):
                fh.write(f"R{k}: {seq}\n")
                for label, key in (("read-qual", "q"), ("read-ins-qual", "ins"),
                                   ("read-del-qual", "del"), ("gcp", "gcp")):
                    fh.write(f"  {label}: " + " ".join(str(int(v)) for v in r[key][k]) + "\n")
            fh.write("\n")


def oracle_lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_pair_log10.restype = ctypes.c_double
        lib.oracle_pair_log10.argtypes = [_u8p, ctypes.c_uint32, _u8p, _u8p, _u8p, _u8p, _u8p,
                                          ctypes.c_uint32, ctypes.c_int]
        lib.oracle_batch.restype = ctypes.c_int
        lib.oracle_batch.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _u8p, _u64p, _u32p,
                                     _u8p, _u8p, _u8p, _u8p, _u8p, _u64p, _u32p, _u64p, _f64p,
                                     ctypes.c_int, ctypes.c_int]
        for name in ("oracle_ph2pr", "oracle_mm_prob"):
            getattr(lib, name).restype = ctypes.c_double
        for name in ("oracle_ph2pr_f", "oracle_mm_prob_f"):
            getattr(lib, name).restype = ctypes.c_float
        lib.oracle_mm_prob.argtypes = [ctypes.c_int, ctypes.c_int]
        lib.oracle_mm_prob_f.argtypes = [ctypes.c_int, ctypes.c_int]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_SO)
        lib.ref_isa.restype = ctypes.c_int
        lib.ref_intra_pair.restype = ctypes.c_double
        lib.ref_intra_pair.argtypes = [_u8p, ctypes.c_uint32, _u8p, _u8p, _u8p, _u8p, _u8p,
                                       ctypes.c_uint32, ctypes.c_int]
        lib.ref_schedule_batch.restype = ctypes.c_int
        lib.ref_schedule_batch.argtypes = [ctypes.c_void_p, ctypes.c_uint32, _u8p, _u64p, _u32p,
                                           _u8p, _u8p, _u8p, _u8p, _u8p, _u64p, _u32p, _u64p,
                                           _f64p, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_int]
        _ref = lib
    return _ref


def _ptr(a: np.ndarray, typ):
    return a.ctypes.data_as(typ)


def _bytes(x) -> np.ndarray:
    if isinstance(x, str):
        x = x.encode()
    return np.ascontiguousarray(np.frombuffer(bytes(x), dtype=np.uint8)) if not isinstance(
        x, np.ndarray) else np.ascontiguousarray(x, dtype=np.uint8)


def pair_log10(hap, read, q, ins, dele, gcp, mode: int = REFERENCE) -> float:
    """One (hap, read) pair; quals are raw Phred integers (not +33)."""
    h, r = _bytes(hap), _bytes(read)
    qs = [_bytes(a) for a in (q, ins, dele, gcp)]
    return oracle_lib().oracle_pair_log10(_ptr(h, _u8p), len(h), _ptr(r, _u8p),
                                          *[_ptr(a, _u8p) for a in qs], len(r), mode)


def ref_intra(hap, read, q, ins, dele, gcp, use_double: bool = False) -> float:
    h, r = _bytes(hap), _bytes(read)
    qs = [_bytes(a) for a in (q, ins, dele, gcp)]
    return ref_lib().ref_intra_pair(_ptr(h, _u8p), len(h), _ptr(r, _u8p),
                                    *[_ptr(a, _u8p) for a in qs], len(r), int(use_double))


def _batch_args(b):
    return (b.regions.ctypes.data, len(b.regions), _ptr(b.hap_bases, _u8p),
            _ptr(b.hap_offsets, _u64p), _ptr(b.hap_lengths, _u32p), _ptr(b.read_bases, _u8p),
            _ptr(b.base_quals, _u8p), _ptr(b.ins_quals, _u8p), _ptr(b.del_quals, _u8p),
            _ptr(b.gcp_quals, _u8p), _ptr(b.read_offsets, _u64p), _ptr(b.read_lengths, _u32p))


def batch_log10(batch, mode: int = REFERENCE, threads: int = 0) -> np.ndarray:
    """Every pair of every region of a ``rodv_b200.Batch``; flat hap-major output."""
    off = batch.out_offsets()
    out = np.empty(int(off[-1]), dtype=np.float64)
    threads = threads or os.cpu_count() or 1
    oracle_lib().oracle_batch(*_batch_args(batch), _ptr(off, _u64p), _ptr(out, _f64p), mode,
                              threads)
    return out


def ref_schedule(batch, use_double: bool = False, ratio_f: float = 0.1, ratio_d: float = 0.1,
                 threads: int = 0, quiet: bool = True) -> np.ndarray:
    """The reference's schedule_pairhmm over every region, one region per task."""
    off = batch.out_offsets()
    out = np.empty(int(off[-1]), dtype=np.float64)
    threads = threads or os.cpu_count() or 1
    fails = ref_lib().ref_schedule_batch(*_batch_args(batch), _ptr(off, _u64p),
                                         _ptr(out, _f64p), int(use_double), ratio_f, ratio_d,
                                         threads, int(quiet))
    if fails:
        raise RuntimeError(f"reference schedule_pairhmm returned false for {fails} regions")
    return out
