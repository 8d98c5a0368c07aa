#!/usr/bin/env python
"""Benchmark of the B200 PairHMM engine (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl rodv|reference]
                    [--workload uneven] [--scale 1.0]

A step is one pass of the PairHMM forward pass over every pair of the
workload.  The default workload is the uneven batch: 10,000 regions, 20-200
reads (50-250 bp) x 2-16 haplotypes (100-600 bp), seeded synthetic data with
those shapes (rodv_b200/workloads.py); about 10M pairs and 5e11 cells.

Reported (see the JSON keys):
  value      GCUPS with the batch resident in HBM (rodv_device_batch_run),
             device time from CUDA events on the engine's stream, summed over
             the K timed steps; the batch (about 1 GB) is larger than L2.
  e2e        GCUPS through rodv_pairhmm_batch with host buffers: packing,
             the H2D copy of the step's inputs from pinned memory, compute and
             the D2H copy of every result are inside the timed region.
  roofline   the FP32 forward kernels against the FP32 FMA peak measured on
             this GPU in this run (FMA-chain kernels, rodv_measure_peaks);
             12 algorithmic flops per cell (4 mul + 2 add for M, 2 mul + 1 add
             for I and for D); traffic is the DRAM bytes of those kernels per
             step, from an ncu capture of every FP32 launch of one step at a
             smaller scale on the same sources (profiles/), scaled by cells.
  plain_form the plain GPU form (one launch per pair) against the batched
             engine on the same sample.
  cpu_baseline  the reference's own schedule_pairhmm (oracle/_ref), threads
             over all host cores, on a bounded sample of the same workload.

Multi-GPU (torchrun): one process per GPU; every rank computes its own
workload of the same shape (seed + rank), no collective on the data path;
the barrier and max-over-ranks timing use torch.distributed.  ``scaling`` is
weak.  ``strong_scaling`` shards one batch of the workload over the ranks by
region (rodv_shard_plan) and times it the same way.  ``--impl reference``
times the reference's CPU path on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("PairHMM GCUPS on 1 B200 (batched vs plain GPU form, % FP32 peak) vs host AVX; "
          "p99 ms")
FLOPS_PER_CELL = 12
# every result must be within this many log10 units of the FP64 oracle and of
# the reference's own output
ACCURACY_TOL = 1e-3
TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "forward_kernels_dram_traffic_uneven.md")
# The device sources whose compiled code the traffic capture measured.
KERNEL_SOURCES = ["pairhmm_fwd.cuh", "pairhmm_pipe.cuh", "layout.h", "kernel_table.cuh",
                  "kernels.h", "pairhmm_kernels.cu", "kernels_r*.cu", "kernels_multi_r*.cu"]


def _code_only(text):
    """C++ source without its comments and blank or trailing space: what the
    compiler sees, so that editing a comment keeps a capture valid."""
    out, i, n = [], 0, len(text)
    while i < n:
        c = text[i]
        if c in "\"'":  # string or character literal, copied whole
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            out.append(text[i:j + 1])
            i = j + 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    lines = (ln.rstrip() for ln in "".join(out).splitlines())
    return "\n".join(ln for ln in lines if ln)


def kernel_source_sha():
    """sha256 (first 16 hex digits) of the forward kernels' sources, comments
    and blank lines left out."""
    import glob
    import hashlib
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "rodv_b200", "csrc")
    names = sorted({os.path.basename(p) for pat in KERNEL_SOURCES
                    for p in glob.glob(os.path.join(csrc, pat))})
    for name in names:
        with open(os.path.join(csrc, name), encoding="utf-8") as fh:
            h.update(name.encode() + b"\0" + _code_only(fh.read()).encode())
    return h.hexdigest()[:16]


def profile_fields(path=TRAFFIC_PROFILE):
    """The `key: value` lines of an ncu summary."""
    out = {}
    if os.path.exists(path):
        with open(path) as fh:
            for ln in fh:
                if ":" in ln and not ln.startswith(("#", "|", " ", "`", "*")):
                    k, v = ln.split(":", 1)
                    out[k.strip()] = v.strip()
    return out


def step_traffic_bytes(workload, scale):
    """DRAM bytes (read + write) of the FP32 kernels of one resident step of the
    full-size uneven workload: the capture of every FP32 launch of one step of
    the same workload at a smaller scale in TRAFFIC_PROFILE, scaled by the
    step's cells.  Returns (bytes or None, note).  A capture taken on other
    kernel sources than these is not reported (the note says so)."""
    if workload != "uneven" or scale != 1.0:
        return None, "captured for the full-size uneven workload only"
    f = profile_fields()
    if "fp32_step_traffic_bytes" not in f:
        return None, f"no traffic capture in {os.path.relpath(TRAFFIC_PROFILE, ROOT)}"
    if f.get("kernel_source_sha16") != kernel_source_sha():
        return None, ("STALE: the traffic capture measured kernel sources "
                      f"{f.get('kernel_source_sha16')}, this build has {kernel_source_sha()}")
    return int(f["fp32_step_traffic_bytes"]), f.get("traffic_note", "")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, path: str = ""):
        self.gpu = gpu_index
        self.proc = None
        self.path = path or os.path.join(tempfile.gettempdir(),
                                         f"rodv_clocks_gpu{gpu_index}_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        rows = []
        for ln in open(self.path):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for _, _, fl in rows for k, v in enumerate(fl)
                          if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_rate(batch, threads: int):
    """The reference's schedule_pairhmm over a batch; returns (GCUPS, seconds)."""
    import oracle
    t0 = time.perf_counter()
    oracle.ref_schedule(batch, threads=threads)
    dt = time.perf_counter() - t0
    return batch.cells() / dt / 1e9, dt


def sized_sample(name: str, seed: int, seconds: float, threads: int):
    """A seeded sample sized, from a short probe run, to take about `seconds`."""
    probe = sample_for_cpu(name, seed + 1, 2e9)
    rate, _ = reference_rate(probe, threads)  # also warms the reference's tables
    return sample_for_cpu(name, seed, rate * 1e9 * seconds)


def sample_for_cpu(name: str, seed: int, target_cells: float):
    """A seeded prefix of the workload holding about target_cells cells."""
    from rodv_b200 import workloads
    full_regions = {"uneven": 10_000, "uneven_windows": 10_000, "stream": 1_000, "long": 2_000,
                    "underflow": 200_000, "plain": 1, "tiny": 8}[name]
    probe = workloads.make_workload(name, seed=seed, scale=min(1.0, 50 / full_regions))
    per_region = probe.cells() / max(1, probe.num_regions)
    n = max(1, min(full_regions, int(target_cells / per_region)))
    return workloads.make_workload(name, seed=seed, scale=n / full_regions)


def run_reference(args, world, rank):
    """--impl reference: the reference's CPU path, rank 0 only."""
    if rank != 0:
        return
    import oracle
    threads = os.cpu_count() or 1
    config = {"workload": args.workload, "scale": args.scale, "sample": "bounded prefix",
              "l2": "n/a (CPU)"}
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libref_pairhmm.so was not built (reference tree absent "
                          "at build time)"}))
        return
    # each step is a sample sized to take about --ref-seconds on all host cores
    batch = sized_sample(args.workload, 7000, args.ref_seconds, threads)
    warm = sample_for_cpu(args.workload, 7002, batch.cells() / 10)
    for _ in range(max(1, args.warmup)):
        reference_rate(warm, threads)
    times = []
    for _ in range(args.steps):
        _, dt = reference_rate(batch, threads)
        times.append(dt)
    total = sum(times)
    value = batch.cells() * len(times) / total / 1e9
    sample = (f"{batch.num_regions} regions, {batch.num_pairs} pairs, {batch.cells():.3e} cells "
              f"of the {args.workload} workload per step")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total / len(times) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": config,
            "cpu_baseline": {"value": value, "unit": "GCUPS", "cores": threads,
                             "kind": "reference", "sample": sample, "cpu": cpu_model()},
            "e2e": {"value": value, "unit": "GCUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_engine(args, world, rank, local):
    import torch
    from rodv_b200 import Engine, workloads
    from rodv_b200.batch import Batch  # noqa: F401

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t_gen = time.perf_counter()
    batch = workloads.make_workload(args.workload, seed=workloads.SEEDS[args.workload] + rank,
                                    scale=args.scale)
    cells = batch.cells()
    if rank == 0:
        log(f"workload {args.workload}: {batch.num_regions} regions, {batch.num_pairs} pairs, "
            f"{cells:.3e} cells (generated in {time.perf_counter() - t_gen:.1f} s)")
    eng = Engine(local)
    t_tune = time.perf_counter()
    eng.autotune()
    variants = eng.tuned_variants()
    t_tune = time.perf_counter() - t_tune
    peaks = eng.measure_peaks()
    db = eng.upload(batch)

    # ---- value: device-resident batch ----
    for _ in range(args.warmup):
        db.run()
    barrier()
    dev_ms, fp32_ms, step_ms, launches, fp64_pairs = [], [], [], 0, 0
    with Clocks(local, args.clocks_out) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ts = time.perf_counter()
            st = db.run()
            step_ms.append((time.perf_counter() - ts) * 1e3)
            dev_ms.append(st["device_ms"])
            fp32_ms.append(st["fp32_ms"])
            launches += st["kernel_launches"]
            fp64_pairs = st["fp64_pairs"]
        barrier()
        wall = time.perf_counter() - t0
    clocks = clk.summary()
    dev_total = max_over_ranks(sum(dev_ms) / 1e3)
    value = world * cells * args.steps / dev_total / 1e9
    results = db.download()
    db.free()

    # ---- e2e: host buffers through rodv_pairhmm_batch ----
    from rodv_b200 import _CBatchHolder
    holder = _CBatchHolder(batch)
    out = np.empty(batch.num_pairs, dtype=np.float64)
    for _ in range(max(1, args.warmup // 2)):
        eng.batch_into(holder, out)
    barrier()
    e2e_ms, h2d, d2h = [], 0, 0
    for _ in range(args.e2e_steps or args.steps):
        t = time.perf_counter()
        st = eng.batch_into(holder, out)
        e2e_ms.append((time.perf_counter() - t) * 1e3)
        h2d, d2h = st["h2d_bytes"], st["d2h_bytes"]
    e2e_total = max_over_ranks(sum(e2e_ms) / 1e3)
    e2e_value = world * cells * len(e2e_ms) / e2e_total / 1e9
    same = float(np.abs(out - results).max())

    # ---- strong scaling (N > 1): one batch, its regions sharded over the ranks ----
    strong = None
    if world > 1 and not args.no_strong:
        from rodv_b200.sharding import shard_plan
        whole = (batch if rank == 0 else
                 workloads.make_workload(args.workload, seed=workloads.SEEDS[args.workload],
                                         scale=args.scale))
        assign, shard_cells = shard_plan(whole, world)
        sub = whole.subset(np.nonzero(assign == rank)[0].tolist())
        sdb = eng.upload(sub)
        for _ in range(args.warmup):
            sdb.run()
        barrier()
        s_ms = [sdb.run()["device_ms"] for _ in range(args.steps)]
        barrier()
        sdb.free()
        s_total = max_over_ranks(sum(s_ms) / 1e3)
        strong = {"value": whole.cells() * args.steps / s_total / 1e9, "unit": "GCUPS",
                  "what": "one batch of the workload, its regions sharded over the ranks by "
                          "rodv_shard_plan (cells, longest first); device time, max over ranks",
                  "ms_per_step": s_total / args.steps * 1e3,
                  "max_shard_cells_frac": float(shard_cells.max() / shard_cells.sum())}

    line = None
    if rank == 0:
        fp32_avg_s = sum(fp32_ms) / len(fp32_ms) / 1e3
        if fp32_avg_s <= 0:
            raise RuntimeError("the FP32 pass was not timed (fp32_ms = 0)")
        achieved = FLOPS_PER_CELL * cells / fp32_avg_s / 1e12
        peak = peaks["fp32_gflops"] / 1e3
        plain = plain_form(eng, args) if args.plain_pairs > 0 else None
        configs = config_lines(eng, args, value) if not args.no_configs else None
        cpu = None
        if not args.no_cpu_baseline:
            cpu = cpu_baseline(args)
        accuracy = accuracy_per_config(eng) if not args.no_accuracy else None
        traffic, traffic_note = step_traffic_bytes(args.workload, args.scale)
        stream = streaming_c5(args) if args.stream_requests > 0 else None
        line = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f32x2) + f64 rescue",
            "data": "synthetic",
            "config": {"workload": args.workload, "regions": batch.num_regions,
                       "pairs": batch.num_pairs, "cells": cells, "scale": args.scale,
                       "l2": "inputs larger than L2 (resident batch ~%.2f GB)" %
                             (batch.input_bytes() / 1e9),
                       "parallelism": f"dp{world} (regions sharded, no collective)",
                       "tuned_variants_fp32": variants["fp32"],
                       "tuned_variants_fp64": variants["fp64"], "tune_s": round(t_tune, 2)},
            "e2e": {"value": e2e_value, "unit": "GCUPS", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": len(e2e_ms),
                    "ms_per_step": e2e_total / len(e2e_ms) * 1e3,
                    "max_abs_diff_vs_resident_run": same},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                           "of every FP32 launch of one step at a smaller "
                                           "scale, scaled to this step by its cells (" +
                                           os.path.relpath(TRAFFIC_PROFILE, ROOT) + "); " +
                                           traffic_note,
                         "kernel_source_sha16": kernel_source_sha(),
                         "kernel": "forward_kernel<F32x2,...> (all FP32 classes of a step)",
                         "flops_per_cell": FLOPS_PER_CELL,
                         "peak_source": "FFMA-chain kernel measured in this run "
                                        "(rodv_measure_peaks); MEASURED_PEAKS.json has no "
                                        "FP32 entry",
                         "fp32x2_peak_tflops": peaks["fp32x2_gflops"] / 1e3,
                         "fp64_peak_tflops": peaks["fp64_gflops"] / 1e3,
                         "peak_sm_mhz": peaks["sm_mhz"]},
            "fp64_rescue": {"pairs": int(fp64_pairs),
                            "rate": fp64_pairs / max(1, batch.num_pairs)},
            "latency_ms": {"p50": float(np.percentile(step_ms, 50)),
                           "p99": float(np.percentile(step_ms, 99)),
                           "what": "per-step (whole batch) host-observed latency"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "wall_s_timed": wall,
        }
        if strong:
            line["strong_scaling"] = strong
        if plain:
            line["plain_form"] = plain
            line["config"]["C1_plain_speedup"] = plain["speedup"]
        if cpu:
            line["cpu_baseline"] = cpu
        if configs:
            line["configs"] = {k: v for c in configs for k, v in flat_config(c).items()}
            for c in configs:
                if c["config"] in ("C1", "C3", "C4", "C5"):
                    line["config"][c["config"] + "_gcups"] = c["gcups"]
        if accuracy:
            line["accuracy"] = {k: v for a in accuracy for k, v in flat_accuracy(a).items()}
            worst = []
            for key in ("vs_fp64_oracle", "vs_reference"):
                vals = [a[key]["max"] for a in accuracy if a[key]["max"] is not None]
                line["config"]["max_abs_dlog10_" + key] = max(vals) if vals else None
                worst += vals
            mism = sum(a[k]["non_finite_mismatches"] for a in accuracy
                       for k in ("vs_fp64_oracle", "vs_reference"))
            line["accuracy"]["tolerance_log10"] = ACCURACY_TOL
            line["accuracy"]["within_tolerance"] = bool(worst and max(worst) <= ACCURACY_TOL
                                                        and mism == 0)
        if stream:
            line["streaming"] = stream
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    eng.close()


def run_profile(args, local):
    """--mode profile: upload the workload, W untimed + K timed resident steps,
    nothing else launched (the command that ncu captures)."""
    from rodv_b200 import Engine, workloads
    batch = workloads.make_workload(args.workload, seed=workloads.SEEDS[args.workload],
                                    scale=args.scale)
    eng = Engine(local)
    if args.tune:
        # with --tune-cache, a first run tunes and writes the cache and later
        # runs (the one ncu profiles) only read it: no tuning launches
        eng.autotune(cache_path=args.tune_cache or None)
    db = eng.upload(batch)
    for _ in range(args.warmup):
        db.run()
    stats = [db.run() for _ in range(args.steps)]
    db.free()
    cells = batch.cells()
    dev = sum(s["device_ms"] for s in stats) / max(1, len(stats))
    fp32 = sum(s["fp32_ms"] for s in stats) / max(1, len(stats))
    print(json.dumps({"mode": "profile", "workload": args.workload, "scale": args.scale,
                      "pairs": batch.num_pairs, "cells": cells, "device_ms": dev,
                      "fp32_ms": fp32, "gcups": cells / dev / 1e6 if dev else None,
                      "fp64_pairs": stats[-1]["fp64_pairs"] if stats else None,
                      "launches_per_step": stats[-1]["kernel_launches"] if stats else None}),
          flush=True)
    eng.close()


def plain_form(eng, args):
    """Plain one-pair-per-launch GPU form vs the batched engine on one sample."""
    from rodv_b200 import workloads
    b = workloads.make_workload("plain")  # 1 region, 8 x 64 pairs
    db = eng.upload(b)
    db.run()
    reps = 5
    t_batched = []
    for _ in range(reps):
        t_batched.append(db.run()["device_ms"])
    _, st = eng.plain(db)
    db.free()
    cells = b.cells()
    batched = cells / (min(t_batched) / 1e3) / 1e9
    plain = cells / (st["device_ms"] / 1e3) / 1e9
    return {"sample": f"plain workload: 1 region, {b.num_pairs} pairs, {cells:.3e} cells",
            "plain_gcups": plain, "batched_gcups": batched, "speedup": batched / plain,
            "plain_launches": st["kernel_launches"]}


def streaming_c5(args):
    """C5: regions arrive one by one at the streaming service (rodv_service).

    A pool of synthetic C5 regions (1-32 haplotypes of 100-800 bases, 1-300
    reads of 50-250 bases) is cycled.  Saturation: requests submitted as fast
    as two host threads can; then Poisson arrivals at fractions of that rate.
    Per run: achieved GCUPS (cells of completed requests / wall time from the
    first submit to the last completion) and the service's latency
    percentiles (submit -> results available)."""
    import ctypes
    import threading
    from rodv_b200 import Service, _CBatchHolder, _lib, workloads

    pool_batch = workloads.make_workload("stream", seed=workloads.SEEDS["stream"],
                                         scale=args.stream_pool / 1000.0)
    pool = [pool_batch.subset([g]) for g in range(pool_batch.num_regions)]
    holders = [_CBatchHolder(b) for b in pool]
    cells = [b.cells() for b in pool]
    sv = Service(0, verbose=args.stream_verbose)
    lib, h = sv.lib, sv.h

    def run(n_req, rate):
        """n_req requests cycling the pool; rate None = as fast as possible."""
        tickets = [0] * n_req
        order = np.arange(n_req) % len(pool)
        lag = [0.0]

        def submitter(k0, step):
            t = ctypes.c_uint64()
            for k in range(k0, n_req, step):
                st = lib.rodv_submit_region(h, ctypes.byref(holders[order[k]].c), ctypes.byref(t))
                if st != 0:
                    raise RuntimeError(f"submit failed: {st}")
                tickets[k] = t.value

        def poisson():
            rng = np.random.default_rng(17)
            gaps = rng.exponential(1.0 / rate, n_req)
            t_next = time.perf_counter()
            t = ctypes.c_uint64()
            for k in range(n_req):
                t_next += gaps[k]
                while True:
                    dt = t_next - time.perf_counter()
                    if dt <= 0:
                        break
                    time.sleep(dt if dt > 2e-3 else 0)
                lag[0] = max(lag[0], time.perf_counter() - t_next)
                st = lib.rodv_submit_region(h, ctypes.byref(holders[order[k]].c), ctypes.byref(t))
                if st != 0:
                    raise RuntimeError(f"submit failed: {st}")
                tickets[k] = t.value

        sv.reset_stats()
        t0 = time.perf_counter()
        threads = ([threading.Thread(target=submitter, args=(i, 2)) for i in range(2)]
                   if rate is None else [threading.Thread(target=poisson)])
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        t_sub = time.perf_counter() - t0
        rs = _lib.RequestStats()
        for tk in tickets:
            st = lib.rodv_wait(h, tk, -1, None, ctypes.byref(rs))
            if st != 0:
                raise RuntimeError(f"request failed: {st}")
        ss = sv.stats()
        tot_cells = float(sum(cells[i] for i in order))
        res = {"requests": n_req, "offered_per_s": rate,
               "submitted_per_s": n_req / t_sub,
               "completed_per_s": n_req / (ss["wall_ms"] / 1e3),
               "gcups": tot_cells / (ss["wall_ms"] / 1e3) / 1e9,
               "device_gcups": tot_cells / (ss["device_ms"] / 1e3) / 1e9,
               "p50_ms": ss["latency_p50_ms"], "p99_ms": ss["latency_p99_ms"],
               "max_ms": ss["latency_max_ms"], "batches": ss["batches"],
               "mean_batch_regions": ss["mean_batch_regions"],
               "host_launch_ms": ss["host_launch_ms"], "host_finish_ms": ss["host_finish_ms"],
               "wall_ms": ss["wall_ms"], "device_ms": ss["device_ms"],
               "fp64_pairs": ss["fp64_pairs"]}
        if rate is not None:
            res["max_submit_lag_ms"] = lag[0] * 1e3
        return res

    run(len(pool), None)  # warm-up (buffers grow to size)
    sat = run(args.stream_requests, None)
    sat_rate = sat["completed_per_s"]
    runs = []
    for frac in (0.25, 0.5, 0.75, 0.9):
        rate = frac * sat_rate
        n = max(50, int(rate * args.stream_seconds))
        r = run(n, rate)
        r["fraction_of_saturation"] = frac
        runs.append(r)
    sv.close()
    mean_cells = float(np.mean(cells))
    return {"config": "C5 streaming: Poisson arrivals; per region 1-32 haplotypes of 100-800 "
                      "bases, 1-300 reads of 50-250 bases (synthetic, seeded)",
            "pool_regions": len(pool), "mean_cells_per_region": mean_cells,
            "saturation": sat, "saturation_regions_per_s": sat_rate, "poisson": runs}


# The configurations of the benchmark, by the workload generator that makes
# them: (name, workload, scale for the GPU throughput run, description).
CONFIGS = [
    ("C1", "plain", 1.0, "1 region: 8 haplotypes of 250-400 bases x 64 reads of 150 bases"),
    ("C2", "uneven", 1.0, "10,000 regions: 2-16 haplotypes of 100-600 bases x 20-200 reads "
                          "of 50-250 bases"),
    ("C3", "long", 1.0, "2,000 pairs: reads of 1,000-2,000 bases x haplotypes of "
                        "2,000-5,000 bases"),
    ("C4", "underflow", 1.0, "200,000 pairs: 250-base reads (base quals 2-8) x independent "
                             "400-base haplotypes; every pair rescued in FP64"),
    ("C5", "stream", 0.3, "300 regions of the streaming shape: 1-32 haplotypes of 100-800 "
                          "bases x 1-300 reads of 50-250 bases (resident, as one batch)"),
]


def real_regions_batch(copies: int = 1):
    """The 8 real chrY regions of roDV's assemble log (resouces/pairhmm_debug.txt,
    4,495 pairs), from the committed fixture, repeated `copies` times."""
    import gzip
    from rodv_b200.batch import Batch
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                        "assemble_regions.json.gz")
    with gzip.open(path, "rt") as fh:
        regs = json.load(fh)
    tup = [([h.encode() for h in r["haps"]], [x.encode() for x in r["reads"]],
            [np.array(v, np.uint8) for v in r["q"]], [np.array(v, np.uint8) for v in r["ins"]],
            [np.array(v, np.uint8) for v in r["del"]], [np.array(v, np.uint8) for v in r["gcp"]])
           for r in regs]
    return Batch.from_regions(tup * copies)


def config_lines(eng, args, c2_value):
    """GPU throughput of every configuration (resident batch, CUDA events) and
    its FP64 rescue rate; C2 is the headline line itself.  'real' is the 8
    logged chrY regions, as logged and repeated 500 times."""
    from rodv_b200 import workloads
    lines = []
    for copies in (1, 500):
        b = real_regions_batch(copies)
        db = eng.upload(b)
        db.run()
        sts = [db.run() for _ in range(3)]
        db.free()
        dev = min(x["device_ms"] for x in sts)
        lines.append({"config": f"real x{copies}", "what": "roDV assemble-log chrY regions "
                      "(8 regions, haplotypes 41-227, reads 10-150 bases)",
                      "regions": b.num_regions, "pairs": b.num_pairs, "cells": b.cells(),
                      "device_ms": dev, "gcups": b.cells() / (dev / 1e3) / 1e9,
                      "fp64_rescue_rate": sts[-1]["fp64_pairs"] / b.num_pairs})
    for name, wl, scale, desc in CONFIGS:
        if name == "C2":
            lines.append({"config": name, "what": desc, "gcups": c2_value, "see": "value"})
            continue
        b = workloads.make_workload(wl, seed=workloads.SEEDS[wl], scale=scale)
        db = eng.upload(b)
        db.run()
        sts = [db.run() for _ in range(3)]
        db.free()
        dev = min(x["device_ms"] for x in sts)
        lines.append({"config": name, "what": desc, "regions": b.num_regions,
                      "pairs": b.num_pairs, "cells": b.cells(), "device_ms": dev,
                      "gcups": b.cells() / (dev / 1e3) / 1e9,
                      "fp64_rescue_rate": sts[-1]["fp64_pairs"] / b.num_pairs})
    return lines


# Accuracy samples per configuration: (name, workload, scale of the sample the
# FP64 oracle computes, scale of the sample the reference computes).
ACCURACY_SAMPLES = [("C1", "plain", 1.0, 1.0), ("C2", "uneven", 0.001, 0.02),
                    ("C3", "long", 0.01, 0.1), ("C4", "underflow", 0.005, 0.1),
                    ("C5", "stream", 0.004, 0.05)]


def accuracy_per_config(eng):
    """|delta log10| of the engine's results against the FP64 oracle (FP64 DP
    with per-row rescaling, so no pair underflows: the exact value up to FP64
    rounding) and against the reference's schedule_pairhmm, on seeded samples
    of every configuration."""
    import oracle
    from rodv_b200 import workloads
    out = []
    for name, wl, s_oracle, s_ref in ACCURACY_SAMPLES:
        row = {"config": name}
        for key, scale in (("vs_fp64_oracle", s_oracle), ("vs_reference", s_ref)):
            b = workloads.make_workload(wl, seed=workloads.SEEDS[wl] + 99, scale=scale)
            got = eng.batch(b)
            ref = (oracle.batch_log10(b, oracle.SCALED) if key == "vs_fp64_oracle"
                   else oracle.ref_schedule(b))
            fin = np.isfinite(ref) & np.isfinite(got)
            d = np.abs(got[fin] - ref[fin])
            row[key] = {"pairs": int(b.num_pairs), "cells": b.cells(),
                        "max": float(d.max()) if d.size else None,
                        "mean": float(d.mean()) if d.size else None,
                        "non_finite_mismatches": int(np.sum(np.isfinite(ref) !=
                                                            np.isfinite(got)))}
        out.append(row)
    return out


def flat_config(c):
    """One configuration line as scalar keys prefixed by its name."""
    name = c["config"].replace(" ", "")
    return {f"{name}_{k}": v for k, v in c.items()
            if k != "config" and isinstance(v, (int, float, str))}


def flat_accuracy(a):
    """One configuration's accuracy as scalar keys: <config>_<vs>_<stat>."""
    out = {}
    for key, short in (("vs_fp64_oracle", "oracle"), ("vs_reference", "reference")):
        for stat in ("max", "mean", "pairs", "non_finite_mismatches"):
            out[f"{a['config']}_{short}_{stat}"] = a[key][stat]
    return out


def cpu_baseline(args):
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unit": "GCUPS", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref was not built"}
    threads = os.cpu_count() or 1
    batch = sized_sample(args.workload, 7000, args.cpu_seconds, threads)
    rate, dt = reference_rate(batch, threads)
    res = {"value": rate, "unit": "GCUPS", "cores": threads, "kind": "reference",
           "sample": f"{batch.num_regions} regions / {batch.num_pairs} pairs / "
                     f"{batch.cells():.3e} cells of the {args.workload} workload, "
                     f"{dt:.1f} s on {threads} threads",
           "cpu": cpu_model()}
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["rodv", "reference"], default="rodv")
    ap.add_argument("--mode", choices=["bench", "profile", "streaming"], default="bench",
                    help="profile: resident steps only, for ncu captures; streaming: the C5 "
                         "service measurement only")
    ap.add_argument("--workload", default="uneven")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--e2e-steps", type=int, default=0,
                    help="timed calls of the e2e measurement (0: the same as --steps)")
    ap.add_argument("--clocks-out", default="",
                    help="CSV of the nvidia-smi clock samples (default: a temporary file)")
    ap.add_argument("--plain-pairs", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-strong", action="store_true",
                    help="N > 1: skip the strong-scaling measurement")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the per-configuration accuracy samples")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the per-configuration throughput lines (C1, C3-C5)")
    ap.add_argument("--tune", action="store_true", help="profile mode: autotune first")
    ap.add_argument("--tune-cache", default="",
                    help="profile mode: tuning cache file (read if it has this device, else "
                         "written after tuning)")
    ap.add_argument("--ref-seconds", type=float, default=6.0,
                    help="reference arm: wall seconds of CPU work per step")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="cpu_baseline: wall seconds of CPU work")
    ap.add_argument("--stream-pool", type=int, default=300,
                    help="streaming (C5): regions in the cycled pool")
    ap.add_argument("--stream-requests", type=int, default=4000,
                    help="streaming (C5): requests of the saturation run (0: skip C5)")
    ap.add_argument("--stream-verbose", type=int, default=0,
                    help="streaming (C5): service verbosity (2: host time sections)")
    ap.add_argument("--stream-seconds", type=float, default=3.0,
                    help="streaming (C5): seconds of arrivals per Poisson rate")
    args = ap.parse_args()
    world, rank, local = dist_env()
    if args.mode == "profile":
        run_profile(args, local)
    elif args.mode == "streaming":
        print(json.dumps({"mode": "streaming", "streaming": streaming_c5(args)}), flush=True)
    elif args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_engine(args, world, rank, local)


if __name__ == "__main__":
    main()
