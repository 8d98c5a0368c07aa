"""rodv_multi_batch: one batch sharded by region over several engines.

The run here has one GPU, so the engines share it (devices [0, 0]): the
plan, the per-device sub-batches, one host thread per engine and the merge
are exactly the multi-GPU path; only the device ordinals repeat.  Results
must be bitwise those of one engine on the whole batch (a pair's arithmetic
depends on its own region only)."""
import numpy as np
import pytest

from rodv_b200 import MultiEngine, workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("devices", [[0], [0, 0], [0, 0, 0]])
def test_multi_engine_matches_one_engine_bitwise(engine, devices):
    b = workloads.make_workload("uneven", scale=0.01)
    want = engine.batch(b)
    m = MultiEngine(devices)
    got, st = m.batch(b, stats=True)
    m.close()
    assert np.array_equal(got, want)
    assert st["pairs"] == b.num_pairs and st["cells"] == b.cells()


def test_multi_engine_fp64_and_uneven_shards(engine):
    # few regions of very different sizes: one shard may get a single region
    b = workloads.make_workload("stream", scale=0.004)
    want = engine.batch(b, use_double=True)
    m = MultiEngine([0, 0])
    got = m.batch(b, use_double=True)
    m.close()
    assert np.array_equal(got, want)
