"""Builds rodv_b200/librodv_pairhmm.so from rodv_b200/csrc with nvcc for sm_100a.

Every translation unit is compiled with
``-gencode arch=compute_100a,code=sm_100a`` (device code exists for B200
only) and linked into one shared library with the CUDA runtime linked
statically, so the library does not depend on which libcudart a host process
(for example PyTorch) has already loaded.  Objects go to rodv_b200/_build/ and
are rebuilt when their source or any header is newer.

Usage: ``python -m rodv_b200.build [--force] [--jobs N]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "librodv_pairhmm.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: every fused multiply-add in the device code is an explicit FMA
# intrinsic; no other multiply and add may be fused by the compiler.  Fusing
# is not applied uniformly (the two copies of a 2-way unrolled loop can
# differ), which would make a result depend on the step parity at which its
# haplotype starts in a chain, i.e. on how the batch was cut.
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-ftz=true", "-fmad=false",
                     "-Xcompiler", "-fPIC,-O3", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _env():
    # nvcc uses gcc/g++ from PATH; the image's CC/CXX wrapper links libstdc++
    # statically, which must not leak into the host-compiler choice.
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    env.pop("NVCC_CCBIN", None)
    return env


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nvcc(), "-x", "cu"] + NVCC_FLAGS + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True, env=_env())
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, jobs: int = 0, verbose: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    # objects built with other flags are stale
    stamp = os.path.join(BUILD, "flags.txt")
    flags = " ".join(NVCC_FLAGS)
    if not os.path.exists(stamp) or open(stamp).read() != flags:
        force = True
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True, env=_env())
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(f"built {LIB}", file=sys.stderr)
    with open(stamp, "w") as fh:
        fh.write(flags)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=0)
    a = ap.parse_args()
    build(force=a.force, jobs=a.jobs)
