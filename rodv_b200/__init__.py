"""roDV-B200: the PairHMM forward likelihood on NVIDIA B200.

The compute path is hand-written sm_100a CUDA behind the C ABI of
``include/rodv_pairhmm.h`` (``librodv_pairhmm.so`` in this directory).  This
module is a thin ctypes layer over it that mirrors roDV's own interface:

* :func:`schedule_pairhmm` -- ``pairhmm::schedule::schedule_pairhmm``
  (src/core/pairhmm_schedule.h:14-25): M haplotypes x N reads of one region
  in, ``result[h][r]`` log10 likelihoods out, ``False`` for an empty region.
* :func:`compute_likelihoods` -- ``pairhmm::intra::computeLikelihoods*``
  (src/core/pairhmm/intra/pairhmm_api.h:17-20): one pair.
* :class:`Engine` -- batches of many regions (:class:`Batch`), device-resident
  batches, the plain one-pair-per-launch form, and the peak measurement.
* :class:`Service` -- the streaming service: regions submitted as they come,
  continuously batched on the device, results by ticket, latency statistics.
"""
from __future__ import annotations

import ctypes
import threading
from typing import List, NamedTuple, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import RodvError
from .batch import Batch

__all__ = ["Engine", "DeviceBatch", "MultiEngine", "Service", "Batch", "RodvError", "schedule_pairhmm",
           "compute_likelihoods", "TestCase", "default_engine", "validate_batch"]


def _ptr(a: np.ndarray, typ):
    return a.ctypes.data_as(typ)


class _CBatchHolder:
    """Keeps the numpy arrays alive while the C struct points into them."""

    def __init__(self, b: Batch):
        self.b = b
        self.regions = np.ascontiguousarray(b.regions)
        self.c = _lib.CBatch(
            len(self.regions), self.regions.ctypes.data, len(b.hap_lengths),
            _ptr(b.hap_bases, _lib._u8p), _ptr(b.hap_offsets, _lib._u64p),
            _ptr(b.hap_lengths, _lib._u32p), len(b.read_lengths), _ptr(b.read_bases, _lib._u8p),
            _ptr(b.base_quals, _lib._u8p), _ptr(b.ins_quals, _lib._u8p),
            _ptr(b.del_quals, _lib._u8p), _ptr(b.gcp_quals, _lib._u8p),
            _ptr(b.read_offsets, _lib._u64p), _ptr(b.read_lengths, _lib._u32p))


def validate_batch(b: Batch) -> None:
    """Checks a batch on the host (no device needed) by the rules the compute
    calls apply (rodv_batch_validate); raises RodvError with the status a
    compute call would return and its description."""
    holder = _CBatchHolder(b)
    msg = ctypes.create_string_buffer(256)
    st = _lib.load().rodv_batch_validate(ctypes.byref(holder.c), msg, len(msg))
    if st != _lib.RODV_OK:
        raise RodvError(st, msg.value.decode(errors="replace"))


class DeviceBatch:
    """A batch packed and resident in device memory (rodv_device_batch)."""

    def __init__(self, engine: "Engine", handle: ctypes.c_void_p, batch: Batch):
        self.engine = engine
        self.handle = handle
        self.num_pairs = batch.num_pairs
        self.cells = batch.cells()

    def run(self) -> dict:
        st = _lib.Stats()
        self.engine._check(self.engine.lib.rodv_device_batch_run(self.engine.h, self.handle,
                                                                 ctypes.byref(st)))
        return st.as_dict()

    def download(self) -> np.ndarray:
        out = np.empty(self.num_pairs, dtype=np.float64)
        self.engine._check(self.engine.lib.rodv_device_batch_download(
            self.engine.h, self.handle, _ptr(out, _lib._f64p)))
        return out

    def free(self) -> None:
        if self.handle:
            self.engine.lib.rodv_device_batch_free(self.engine.h, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine:
    """A PairHMM engine on one CUDA device (rodv_engine)."""

    def __init__(self, device: int = 0, force_fp64: bool = False, verbose: bool = False,
                 device_memory_budget: int = 0, max_inflight: int = 0, autotune: int = 0,
                 tune_cache: Optional[str] = None):
        self.lib = _lib.load()
        opts = _lib.Options()
        self.lib.rodv_default_options(ctypes.byref(opts))
        opts.device = device
        opts.force_fp64 = int(force_fp64)
        opts.verbose = int(verbose)
        opts.device_memory_budget = device_memory_budget
        opts.max_inflight = max_inflight
        opts.autotune = autotune
        self._tune_cache = tune_cache.encode() if tune_cache else None
        opts.tune_cache = self._tune_cache
        h = ctypes.c_void_p()
        st = self.lib.rodv_engine_create(ctypes.byref(opts), ctypes.byref(h))
        if st != _lib.RODV_OK:
            detail = self.lib.rodv_last_error(None) or b""
            raise RodvError(st, "engine creation failed: " + detail.decode(errors="replace"))
        self.h = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.rodv_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _lib.RODV_OK:
            detail = self.lib.rodv_last_error(self.h) if self.h else b""
            raise RodvError(st, detail.decode(errors="replace") if detail else "")

    def batch(self, b: Batch, use_double: bool = False, stats: bool = False):
        """All pairs of all regions; flat hap-major log10 results per region."""
        holder = _CBatchHolder(b)
        out = np.empty(b.num_pairs, dtype=np.float64)
        st = _lib.Stats()
        self._check(self.lib.rodv_pairhmm_batch(self.h, ctypes.byref(holder.c), int(use_double),
                                                _ptr(out, _lib._f64p), ctypes.byref(st)))
        return (out, st.as_dict()) if stats else out

    def batch_raw(self, b: Batch, use_double: bool = False):
        """Raw scaled likelihoods and the precision of each (0: FP32 at 2^120,
        1: FP64 at 2^1020) -- roDV's inter API with islog10 = false."""
        holder = _CBatchHolder(b)
        out = np.empty(b.num_pairs, dtype=np.float64)
        prec = np.empty(b.num_pairs, dtype=np.uint8)
        st = _lib.Stats()
        self._check(self.lib.rodv_pairhmm_batch_raw(self.h, ctypes.byref(holder.c),
                                                    int(use_double), _ptr(out, _lib._f64p),
                                                    _ptr(prec, _lib._u8p), ctypes.byref(st)))
        return out, prec

    def batch_into(self, holder: _CBatchHolder, out: np.ndarray, use_double: bool = False) -> dict:
        """Like :meth:`batch` with a prepared struct and output (no allocation)."""
        st = _lib.Stats()
        self._check(self.lib.rodv_pairhmm_batch(self.h, ctypes.byref(holder.c), int(use_double),
                                                _ptr(out, _lib._f64p), ctypes.byref(st)))
        return st.as_dict()

    def pair(self, hap, read, q, ins, dele, gcp, use_double: bool = False) -> float:
        arrs = [np.ascontiguousarray(np.frombuffer(x.encode() if isinstance(x, str) else bytes(
            bytearray(x)), dtype=np.uint8)) if not isinstance(x, np.ndarray) else
            np.ascontiguousarray(x, dtype=np.uint8) for x in (hap, read, q, ins, dele, gcp)]
        h, r, qq, ii, dd, cc = arrs
        if not (len(qq) == len(ii) == len(dd) == len(cc) == len(r)):
            raise RodvError(1, "quality arrays must match the read length")
        out = ctypes.c_double()
        self._check(self.lib.rodv_pairhmm_pair(
            self.h, _ptr(h, _lib._u8p), len(h), _ptr(r, _lib._u8p), _ptr(qq, _lib._u8p),
            _ptr(ii, _lib._u8p), _ptr(dd, _lib._u8p), _ptr(cc, _lib._u8p), len(r),
            int(use_double), ctypes.byref(out)))
        return out.value

    def upload(self, b: Batch) -> DeviceBatch:
        holder = _CBatchHolder(b)
        h = ctypes.c_void_p()
        self._check(self.lib.rodv_device_batch_upload(self.h, ctypes.byref(holder.c),
                                                      ctypes.byref(h)))
        return DeviceBatch(self, h, b)

    def plain(self, db: DeviceBatch):
        out = np.empty(db.num_pairs, dtype=np.float64)
        st = _lib.Stats()
        self._check(self.lib.rodv_pairhmm_plain(self.h, db.handle, _ptr(out, _lib._f64p),
                                                ctypes.byref(st)))
        return out, st.as_dict()

    def autotune(self, cache_path: Optional[str] = None, force: bool = False) -> List[int]:
        """Tunes the FP32 kernel's occupancy variant per work class; returns them."""
        v = (ctypes.c_int32 * 18)()
        self._check(self.lib.rodv_autotune(self.h, cache_path.encode() if cache_path else None,
                                           int(force), v))
        return list(v)

    def tuned_variants(self) -> dict:
        """The engine's current kernel variant per work class, FP32 and FP64."""
        a, b = (ctypes.c_int32 * 18)(), (ctypes.c_int32 * 18)()
        self._check(self.lib.rodv_tuned_variants(self.h, a, b))
        return {"fp32": list(a), "fp64": list(b)}

    def measure_peaks(self) -> dict:
        v = [ctypes.c_double() for _ in range(4)]
        self._check(self.lib.rodv_measure_peaks(self.h, *[ctypes.byref(x) for x in v]))
        return {"fp32_gflops": v[0].value, "fp32x2_gflops": v[1].value,
                "fp64_gflops": v[2].value, "sm_mhz": v[3].value}


class MultiEngine:
    """One batch over several devices (rodv_multi): regions sharded by cells,
    one engine and host thread per device, results merged in batch order;
    bitwise the results of :meth:`Engine.batch` on one device."""

    def __init__(self, devices: Sequence[int], force_fp64: bool = False, verbose: bool = False):
        self.lib = _lib.load()
        opts = _lib.Options()
        self.lib.rodv_default_options(ctypes.byref(opts))
        opts.force_fp64 = int(force_fp64)
        opts.verbose = int(verbose)
        devs = (ctypes.c_int32 * len(devices))(*devices)
        h = ctypes.c_void_p()
        st = self.lib.rodv_multi_create(ctypes.byref(opts), devs, len(devices), ctypes.byref(h))
        if st != _lib.RODV_OK:
            detail = self.lib.rodv_last_error(None) or b""
            raise RodvError(st, "multi-device engine creation failed: " +
                            detail.decode(errors="replace"))
        self.h = h
        self.devices = list(devices)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.rodv_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def batch(self, b: Batch, use_double: bool = False, stats: bool = False):
        holder = _CBatchHolder(b)
        out = np.empty(b.num_pairs, dtype=np.float64)
        st = _lib.Stats()
        rc = self.lib.rodv_multi_batch(self.h, ctypes.byref(holder.c), int(use_double),
                                       _ptr(out, _lib._f64p), ctypes.byref(st))
        if rc != _lib.RODV_OK:
            raise RodvError(rc, (self.lib.rodv_multi_last_error(self.h) or b"").decode(
                errors="replace"))
        return (out, st.as_dict()) if stats else out


class Service:
    """The streaming service (rodv_service): submit regions at any time, get
    each request's results by ticket.  Requests are batched continuously on
    the device; a region's results do not depend on what it was batched
    with."""

    def __init__(self, device: int = 0, force_fp64: bool = False, verbose: bool = False,
                 device_memory_budget: int = 0, max_inflight: int = 0, autotune: int = 0,
                 tune_cache: Optional[str] = None):
        self.lib = _lib.load()
        opts = _lib.Options()
        self.lib.rodv_default_options(ctypes.byref(opts))
        opts.device = device
        opts.force_fp64 = int(force_fp64)
        opts.verbose = int(verbose)
        opts.device_memory_budget = device_memory_budget
        opts.max_inflight = max_inflight
        opts.autotune = autotune
        self._tune_cache = tune_cache.encode() if tune_cache else None
        opts.tune_cache = self._tune_cache
        h = ctypes.c_void_p()
        st = self.lib.rodv_service_create(ctypes.byref(opts), ctypes.byref(h))
        if st != _lib.RODV_OK:
            detail = self.lib.rodv_last_error(None) or b""
            raise RodvError(st, "service creation failed: " + detail.decode(errors="replace"))
        self.h = h
        self._pairs = {}
        self._lock = threading.Lock()

    def close(self) -> None:
        """Finishes all submitted work, then stops the service."""
        if getattr(self, "h", None):
            self.lib.rodv_service_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _lib.RODV_OK:
            detail = self.lib.rodv_service_last_error(self.h) if self.h else b""
            raise RodvError(st, detail.decode(errors="replace") if detail else "")

    def submit(self, b: Batch) -> int:
        """Queues the regions of ``b``; returns the request's ticket."""
        holder = _CBatchHolder(b)
        t = ctypes.c_uint64()
        self._check(self.lib.rodv_submit_region(self.h, ctypes.byref(holder.c), ctypes.byref(t)))
        with self._lock:
            self._pairs[t.value] = b.num_pairs
        return t.value

    def _result(self, ticket: int, timeout_ms: Optional[int], stats: bool):
        with self._lock:
            n = self._pairs.get(ticket)
        out = np.empty(n if n is not None else 0, dtype=np.float64)
        rs = _lib.RequestStats()
        optr = _ptr(out, _lib._f64p) if n else None
        if timeout_ms == 0:
            st = self.lib.rodv_poll(self.h, ticket, optr, ctypes.byref(rs))
        else:
            st = self.lib.rodv_wait(self.h, ticket, -1 if timeout_ms is None else timeout_ms, optr,
                                    ctypes.byref(rs))
        if st == _lib.RODV_ERR_NOT_READY:
            return None
        if st != _lib.RODV_ERR_NOT_FOUND:
            with self._lock:
                self._pairs.pop(ticket, None)
        self._check(st)
        return (out, rs.as_dict()) if stats else out

    def poll(self, ticket: int, stats: bool = False):
        """The request's results (flat, hap-major per region), or None if not ready."""
        return self._result(ticket, 0, stats)

    def wait(self, ticket: int, timeout_ms: Optional[int] = None, stats: bool = False):
        """Blocks until the request is done; None if timeout_ms passes first."""
        return self._result(ticket, timeout_ms, stats)

    def stats(self) -> dict:
        ss = _lib.ServiceStats()
        self._check(self.lib.rodv_service_get_stats(self.h, ctypes.byref(ss)))
        return ss.as_dict()

    def reset_stats(self) -> None:
        self.lib.rodv_service_reset_stats(self.h)


_default: Optional[Engine] = None
_default_lock = threading.Lock()


def default_engine() -> Engine:
    """Process-wide engine on device 0 (what the reference-style calls use)."""
    global _default
    with _default_lock:
        if _default is None:
            _default = Engine(0)
        return _default


def schedule_pairhmm(haplotypes: Sequence, reads: Sequence, result: List,
                     quality: Sequence, insertion_qualities: Sequence,
                     deletion_qualities: Sequence, gap_contiguous_qualities: Sequence,
                     use_double: bool = False, max_idle_ratio_float: float = 0.1,
                     max_idle_ratio_double: float = 0.1, verbose: bool = False) -> bool:
    """Mirror of roDV's schedule_pairhmm (src/core/pairhmm_schedule.h:14-25).

    ``result`` is resized to ``[M][N]`` and filled hap-major with log10
    likelihoods.  Returns ``False`` when there are no haplotypes or no reads
    (pairhmm_schedule.cpp:130-132).  The idle ratios tune the reference's CPU
    SIMD grouping and have no effect here.  Invalid input raises
    :class:`RodvError` (the reference has no error path for it).
    """
    M, N = len(haplotypes), len(reads)
    if M == 0 or N == 0:
        return False
    b = Batch.from_regions([(haplotypes, reads, quality, insertion_qualities, deletion_qualities,
                             gap_contiguous_qualities)])
    out, st = default_engine().batch(b, use_double=use_double, stats=True)
    result[:] = [list(out[h * N:(h + 1) * N]) for h in range(M)]
    if verbose:
        import sys
        print(f"schedule_pairhmm: {st['pairs']} pairs, {st['fp64_pairs']} in FP64, "
              f"{st['total_ms']:.3f} ms", file=sys.stderr)
    return True


class TestCase(NamedTuple):
    """The reference's TestCase view (src/core/pairhmm/common/common.h:27-36)."""
    hap: bytes
    rs: bytes
    q: Sequence[int]
    i: Sequence[int]
    d: Sequence[int]
    c: Sequence[int]


TestCase.__test__ = False  # a data type, not a pytest test class


def compute_likelihoods(tc: TestCase, use_double: bool = False) -> float:
    """Mirror of computeLikelihoodsAVX512(tc, use_double) (pairhmm_api.h:17-20)."""
    return default_engine().pair(tc.hap, tc.rs, tc.q, tc.i, tc.d, tc.c, use_double=use_double)
