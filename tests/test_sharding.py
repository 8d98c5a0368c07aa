"""Multi-GPU path on CPU: regions sharded over ranks, no collective on the
data path, results merged back in batch order.  The plan and the merge are
the library's host-only C entry points (rodv_shard_plan, rodv_shard_merge),
the same code rodv_multi_batch runs.  The ranks here are gloo processes on
127.0.0.1 and compute their shard with the CPU oracle (standing in for the
engine, which needs a GPU); the sharding, the per-rank sub-batch, the
max-over-ranks timing reduction and the merge are the code bench.py and a
multi-GPU caller use."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from rodv_b200 import workloads
from rodv_b200.sharding import merge_results, region_cells, shard_regions


def test_lpt_shards_cover_every_region_once_and_balance():
    b = workloads.make_workload("uneven", scale=0.01)
    cells = region_cells(b)
    assert int(cells.sum()) == b.cells()
    for world in (1, 2, 3, 8):
        shards = shard_regions(b, world)
        flat = sorted(g for s in shards for g in s)
        assert flat == list(range(len(b.regions)))
        loads = [int(cells[s].sum()) for s in shards]
        assert max(loads) - min(loads) <= int(cells.max())


def _lpt_reference(cells, world):
    """Longest processing time first, written out plainly: regions by
    decreasing cells (stable), each to the least-loaded shard (lowest index on
    a tie)."""
    load = [0] * world
    assign = [0] * len(cells)
    for g in sorted(range(len(cells)), key=lambda g: -int(cells[g])):
        k = min(range(world), key=lambda k: (load[k], k))
        assign[g] = k
        load[k] += int(cells[g])
    return assign, load


def test_c_plan_is_lpt_by_cells():
    """rodv_shard_plan (C ABI, host only) against a plain restatement of LPT."""
    from rodv_b200.sharding import shard_plan
    b = workloads.make_workload("stream", scale=0.05)
    cells = region_cells(b)
    for world in (1, 2, 5):
        assign, shard_cells = shard_plan(b, world)
        want, load = _lpt_reference(cells, world)
        assert assign.tolist() == want
        assert shard_cells.tolist() == load


def test_merge_restores_batch_order():
    b = workloads.make_workload("tiny", scale=3.0)
    off = b.out_offsets()
    full = np.arange(int(off[-1]), dtype=np.float64)
    shards = shard_regions(b, 3)
    parts = [np.concatenate([full[int(off[g]):int(off[g + 1])] for g in s]) if s else
             np.empty(0) for s in shards]
    assert np.array_equal(merge_results(b, shards, parts), full)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    import datetime
    import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        b = workloads.make_workload("uneven", scale=0.002)
        shards = shard_regions(b, world)
        sub = b.subset(shards[rank])
        import time
        dist.barrier()
        t0 = time.perf_counter()
        res = oracle.batch_log10(sub, oracle.REFERENCE, threads=1)
        dt = time.perf_counter() - t0
        import torch
        t = torch.tensor([dt], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        if rank == 0:
            merged = merge_results(b, shards, gathered)
            whole = oracle.batch_log10(b, oracle.REFERENCE, threads=1)
            q.put((bool(np.array_equal(merged, whole)), float(t.item()) >= dt,
                   [len(s) for s in shards]))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharded_batch_matches_whole_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    same, max_ok, sizes = q.get(timeout=5)
    assert same and max_ok and all(n > 0 for n in sizes)
