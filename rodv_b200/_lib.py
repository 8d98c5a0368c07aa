"""ctypes binding of librodv_pairhmm.so (the C ABI in include/rodv_pairhmm.h).

The library is loaded from this package directory.  If it is missing the
import fails with an error; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librodv_pairhmm.so")

RODV_OK = 0
RODV_ERR_NOT_FOUND = 10
RODV_ERR_NOT_READY = 11
STATUS_NAMES = {
    0: "RODV_OK", 1: "RODV_ERR_INVALID_ARG", 2: "RODV_ERR_EMPTY", 3: "RODV_ERR_INVALID_BASE",
    4: "RODV_ERR_NO_DEVICE", 5: "RODV_ERR_CUDA", 6: "RODV_ERR_OUT_OF_MEMORY",
    7: "RODV_ERR_TOO_LONG", 8: "RODV_ERR_DEVICE_CHECK", 9: "RODV_ERR_ADMISSION",
    10: "RODV_ERR_NOT_FOUND", 11: "RODV_ERR_NOT_READY", 12: "RODV_ERR_SHUTDOWN",
    13: "RODV_ERR_INTERNAL",
}


class RodvError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{name}: {detail}" if detail else name)


class Region(ctypes.Structure):
    _fields_ = [("hap_start", ctypes.c_uint32), ("num_haps", ctypes.c_uint32),
                ("read_start", ctypes.c_uint32), ("num_reads", ctypes.c_uint32)]


_u8p = ctypes.POINTER(ctypes.c_uint8)
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)


class CBatch(ctypes.Structure):
    _fields_ = [("num_regions", ctypes.c_uint32), ("regions", ctypes.c_void_p),
                ("num_haps", ctypes.c_uint32), ("hap_bases", _u8p), ("hap_offsets", _u64p),
                ("hap_lengths", _u32p), ("num_reads", ctypes.c_uint32), ("read_bases", _u8p),
                ("base_quals", _u8p), ("ins_quals", _u8p), ("del_quals", _u8p),
                ("gcp_quals", _u8p), ("read_offsets", _u64p), ("read_lengths", _u32p)]


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("force_fp64", ctypes.c_int32),
                ("device_memory_budget", ctypes.c_uint64), ("max_inflight", ctypes.c_uint32),
                ("verbose", ctypes.c_int32), ("autotune", ctypes.c_int32),
                ("tune_cache", ctypes.c_char_p)]


class Stats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_uint64), ("cells", ctypes.c_uint64),
                ("fp64_pairs", ctypes.c_uint64), ("fp64_cells", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint32), ("pad_", ctypes.c_uint32),
                ("total_ms", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("fp32_ms", ctypes.c_double), ("h2d_ms", ctypes.c_double),
                ("d2h_ms", ctypes.c_double), ("h2d_bytes", ctypes.c_uint64),
                ("d2h_bytes", ctypes.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad_"}


class RequestStats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_uint64), ("cells", ctypes.c_uint64),
                ("fp64_pairs", ctypes.c_uint64), ("batch_id", ctypes.c_uint64),
                ("batch_regions", ctypes.c_uint32), ("pad_", ctypes.c_uint32),
                ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad_"}


class ServiceStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("regions", ctypes.c_uint64), ("pairs", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("fp64_pairs", ctypes.c_uint64),
                ("latency_p50_ms", ctypes.c_double), ("latency_p99_ms", ctypes.c_double),
                ("latency_max_ms", ctypes.c_double), ("latency_mean_ms", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("wall_ms", ctypes.c_double),
                ("mean_batch_regions", ctypes.c_double), ("host_launch_ms", ctypes.c_double),
                ("host_finish_ms", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# (name, restype, argtypes) of every function declared in include/rodv_pairhmm.h
SIGNATURES = [
    ("rodv_default_options", None, [ctypes.POINTER(Options)]),
    ("rodv_engine_create", ctypes.c_int32, [ctypes.POINTER(Options),
                                            ctypes.POINTER(ctypes.c_void_p)]),
    ("rodv_engine_destroy", None, [ctypes.c_void_p]),
    ("rodv_pairhmm_batch", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(CBatch),
                                            ctypes.c_int32, _f64p, ctypes.POINTER(Stats)]),
    ("rodv_pairhmm_batch_raw", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(CBatch),
                                                ctypes.c_int32, _f64p, _u8p,
                                                ctypes.POINTER(Stats)]),
    ("rodv_batch_num_pairs", ctypes.c_uint64, [ctypes.POINTER(CBatch)]),
    ("rodv_batch_validate", ctypes.c_int32, [ctypes.POINTER(CBatch), ctypes.c_char_p,
                                             ctypes.c_size_t]),
    ("rodv_pairhmm_pair", ctypes.c_int32, [ctypes.c_void_p, _u8p, ctypes.c_uint32, _u8p, _u8p,
                                           _u8p, _u8p, _u8p, ctypes.c_uint32, ctypes.c_int32,
                                           _f64p]),
    ("rodv_device_batch_upload", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(CBatch),
                                                  ctypes.POINTER(ctypes.c_void_p)]),
    ("rodv_device_batch_run", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.POINTER(Stats)]),
    ("rodv_device_batch_download", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, _f64p]),
    ("rodv_device_batch_free", None, [ctypes.c_void_p, ctypes.c_void_p]),
    ("rodv_pairhmm_plain", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_void_p, _f64p,
                                            ctypes.POINTER(Stats)]),
    ("rodv_measure_peaks", ctypes.c_int32, [ctypes.c_void_p, _f64p, _f64p, _f64p, _f64p]),
    ("rodv_pairhmm_batch_noalloc", ctypes.c_int32, [ctypes.POINTER(CBatch), ctypes.c_int32,
                                                    ctypes.c_void_p, ctypes.c_void_p]),
    ("rodv_shard_plan", ctypes.c_int32, [ctypes.POINTER(CBatch), ctypes.c_uint32, _u32p,
                                         _u64p]),
    ("rodv_shard_merge", ctypes.c_int32, [ctypes.POINTER(CBatch), ctypes.c_uint32, _u32p,
                                          ctypes.POINTER(_f64p), _f64p]),
    ("rodv_multi_create", ctypes.c_int32, [ctypes.POINTER(Options),
                                           ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_void_p)]),
    ("rodv_multi_destroy", None, [ctypes.c_void_p]),
    ("rodv_multi_batch", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(CBatch),
                                          ctypes.c_int32, _f64p, ctypes.POINTER(Stats)]),
    ("rodv_multi_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("rodv_autotune", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_int32)]),
    ("rodv_tuned_variants", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_int32)]),
    ("rodv_service_create", ctypes.c_int32, [ctypes.POINTER(Options),
                                             ctypes.POINTER(ctypes.c_void_p)]),
    ("rodv_service_destroy", None, [ctypes.c_void_p]),
    ("rodv_submit_region", ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(CBatch), _u64p]),
    ("rodv_poll", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, _f64p,
                                   ctypes.POINTER(RequestStats)]),
    ("rodv_wait", ctypes.c_int32, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, _f64p,
                                   ctypes.POINTER(RequestStats)]),
    ("rodv_service_get_stats", ctypes.c_int32, [ctypes.c_void_p,
                                                ctypes.POINTER(ServiceStats)]),
    ("rodv_service_reset_stats", None, [ctypes.c_void_p]),
    ("rodv_service_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("rodv_fault_inject_alloc", ctypes.c_int32, [ctypes.c_int32, ctypes.c_int64]),
    ("rodv_debug_live_allocations", None, [_u64p, _u64p]),
    ("rodv_fault_inject_wait", ctypes.c_int32, [ctypes.c_int32]),
    ("rodv_debug_chain_plan", ctypes.c_int32, [_u32p, _u8p, ctypes.c_uint32,
                                               ctypes.POINTER(ctypes.c_int32), ctypes.c_int32,
                                               _u32p, ctypes.c_uint32, _u32p]),
    ("rodv_status_string", ctypes.c_char_p, [ctypes.c_int32]),
    ("rodv_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
]

_lib = None


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m rodv_b200.build`;"
                              " the engine has no CPU fallback")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib
