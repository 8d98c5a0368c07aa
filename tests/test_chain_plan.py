"""The packer's placement of a region's single-pass reads in chain items, on
the CPU through the library's host-only rodv_debug_chain_plan (the same
function the packer runs per region, chain_plan.cpp).  Checks the rules the
chain kernel relies on: every single-pass read is placed once (in a pair or
as the region's leftover), an item's pairs fit its class's lanes with a
pass-through row and, for uniform gaps, the sum row, per-row-gap reads stay
one pair per item in their own class, and multi-pass reads are left out."""
import ctypes

import numpy as np
import pytest

from rodv_b200 import _lib

NO = 0xFFFFFFFF
WARP = 32


def plan(lengths, uniform, ipw=(2, 2, 2, 2, 1, 1, 1, 1), stack=1):
    lib = _lib.load()
    n = len(lengths)
    lens = (ctypes.c_uint32 * max(n, 1))(*lengths)
    uni = (ctypes.c_uint8 * max(n, 1))(*[1 if u else 0 for u in uniform])
    ip = (ctypes.c_int32 * 8)(*ipw)
    cap = 4 + 4 * n + 2 * n
    out = (ctypes.c_uint32 * cap)()
    written = ctypes.c_uint32()
    st = lib.rodv_debug_chain_plan(lens, uni, n, ip, stack, out, cap, ctypes.byref(written))
    assert st == 0, st
    w = list(out[:written.value])
    items, leftover = w[0], w[1]
    pos, res = 2, []
    for _ in range(items):
        cls, pairs = w[pos], w[pos + 1]
        reads = w[pos + 2:pos + 2 + 2 * pairs]
        res.append((cls, [(reads[2 * k], reads[2 * k + 1]) for k in range(pairs)]))
        pos += 2 + 2 * pairs
    assert pos == len(w)
    return res, leftover


def rows_needed(length, uniform):
    return length + (2 if uniform else 1)


def single_pass(length, uniform):
    return rows_needed(length, uniform) <= WARP * 8


def class_of(length, uniform):
    R = -(-rows_needed(length, uniform) // WARP)
    return (R - 1) * 2 + (1 if uniform else 0)


def check(lengths, uniform, ipw=(2, 2, 2, 2, 1, 1, 1, 1), stack=1):
    items, leftover = plan(lengths, uniform, ipw, stack)
    seen = []
    for cls, pairs in items:
        assert 0 <= cls < 16
        R = cls // 2 + 1
        if cls % 2 == 0:  # per-row gaps: one pair, the class of the longer read
            assert len(pairs) == 1
            x, y = pairs[0]
            assert y != NO
            assert not (uniform[x] and uniform[y])
            assert cls == class_of(max(lengths[x], lengths[y]), False)
        else:             # uniform gaps: the pairs fit the class's lanes
            g = ipw[R - 1]
            lanes, rows = WARP // g, R * g
            used = 0
            for x, y in pairs:
                assert uniform[x] and (y == NO or uniform[y])
                longest = max(lengths[x], lengths[y] if y != NO else 0)
                used += (longest + 1) // rows + 1
            assert used <= lanes, (cls, pairs, used, lanes)
        for x, y in pairs:
            seen.append(x)
            if y != NO:
                seen.append(y)
    if leftover != NO:
        seen.append(leftover)
    expect = [r for r in range(len(lengths)) if single_pass(lengths[r], uniform[r])]
    assert sorted(seen) == expect
    return items, leftover


def test_small_regions():
    assert plan([], []) == ([], NO)
    items, left = check([100], [True])
    assert items == [] and left == 0
    items, left = check([100, 140], [True, True])
    assert len(items) == 1 and left == NO
    assert items[0][0] == class_of(140, True)


def test_class_edges_reserve_the_sum_row():
    # uniform gaps: 32R - 2 bases in class R, 32R - 1 in class R + 1, 255 multi-pass
    for R in range(1, 9):
        assert class_of(32 * R - 2, True) == (R - 1) * 2 + 1
        assert class_of(32 * R - 1, False) == (R - 1) * 2
    assert not single_pass(255, True) and single_pass(255, False)
    items, left = check([254, 255, 255, 256], [True, True, False, False])
    placed = {r for _, pairs in items for p in pairs for r in p if r != NO}
    assert 1 not in placed and 3 not in placed and left in (0, 2, NO)


@pytest.mark.parametrize("seed", range(12))
def test_random_regions_place_every_read_once(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 220))
    lengths = [int(v) for v in rng.integers(5, 300, n)]
    uniform = [bool(u) for u in rng.random(n) < (0.9 if seed % 3 else 0.5)]
    for ipw in ((2, 2, 2, 2, 1, 1, 1, 1), (1,) * 8, (2, 1, 2, 1, 1, 1, 1, 1)):
        for stack in (0, 1):
            items, _ = check(lengths, uniform, ipw, stack)
            if stack == 0:
                assert all(len(pairs) == 1 for _, pairs in items)


def test_short_uniform_reads_stack_into_few_items():
    # 40 reads of 50-60 bases: 7-8 lanes of 8 rows a pair, so several pairs
    # share an item when stacking is on
    lengths = [50 + (k % 11) for k in range(40)]
    items, left = check(lengths, [True] * 40)
    classic, _ = check(lengths, [True] * 40, stack=0)
    assert left == NO
    assert max(len(p) for _, p in items) >= 2
    assert len(items) < len(classic)


def test_plan_depends_on_the_region_only():
    rng = np.random.default_rng(5)
    lengths = [int(v) for v in rng.integers(20, 255, 90)]
    uniform = [True] * 90
    assert plan(lengths, uniform) == plan(lengths, uniform)


def test_bad_arguments_are_refused():
    lib = _lib.load()
    written = ctypes.c_uint32()
    ip = (ctypes.c_int32 * 8)(*([1] * 8))
    lens = (ctypes.c_uint32 * 1)(0)
    uni = (ctypes.c_uint8 * 1)(1)
    out = (ctypes.c_uint32 * 8)()
    assert lib.rodv_debug_chain_plan(lens, uni, 1, ip, 1, out, 8, ctypes.byref(written)) != 0
    lens[0] = 100
    bad_ip = (ctypes.c_int32 * 8)(*([3] * 8))
    assert lib.rodv_debug_chain_plan(lens, uni, 1, bad_ip, 1, out, 8, ctypes.byref(written)) != 0
    # too small an output buffer: refused, with the size it needs
    assert lib.rodv_debug_chain_plan(lens, uni, 1, ip, 1, out, 1, ctypes.byref(written)) != 0
    assert written.value == 2
