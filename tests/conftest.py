"""Shared pytest configuration: the ``gpu`` marker and golden-fixture loaders."""
from __future__ import annotations

import gzip
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_gkl():
    """The 104 golden cases: (hap, read, q, ins, del, gcp, expected, ref_intra, ref_fp64)."""
    cases = []
    with open(os.path.join(GOLDEN, "gkl_testdata.tsv")) as fh:
        next(fh)
        for ln in fh:
            f = ln.split()
            quals = [np.frombuffer(s.encode(), np.uint8) - 33 for s in f[2:6]]
            cases.append((f[0].encode(), f[1].encode(), *quals, float(f[6]), float(f[7]),
                          float(f[8])))
    return cases


def load_assemble():
    with gzip.open(os.path.join(GOLDEN, "assemble_regions.json.gz"), "rt") as fh:
        return json.load(fh)


def assemble_batch():
    from rodv_b200.batch import Batch
    regs = load_assemble()
    b = Batch.from_regions([(r["haps"], r["reads"], r["q"], r["ins"], r["del"], r["gcp"])
                            for r in regs])
    ref = np.concatenate([np.array(r["ref_schedule"]) for r in regs])
    return b, ref


def synthetic_batch():
    from rodv_b200.batch import Batch
    z = np.load(os.path.join(GOLDEN, "synthetic_ref.npz"))
    b = Batch(z["regions"], z["hap_bases"], z["hap_offsets"], z["hap_lengths"], z["read_bases"],
              z["base_quals"], z["ins_quals"], z["del_quals"], z["gcp_quals"], z["read_offsets"],
              z["read_lengths"])
    return b, z["ref_schedule"], z["ref_intra"]


@pytest.fixture(scope="session")
def gkl_cases():
    return load_gkl()


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def engine():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from rodv_b200 import Engine
    e = Engine(0)
    yield e
    e.close()
