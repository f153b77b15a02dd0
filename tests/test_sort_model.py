"""One pass of the device radix sort, restated in sort_model.py in the
kernel's ranking order, is a stable sort by its 8-bit digit: on random keys,
on nearly sorted Morton-like keys (the order the sort sees from one step to
the next) and on sizes that leave a partial last tile."""
import numpy as np
import pytest

import sort_model as sm


@pytest.mark.parametrize("n,kind,shift", [(5000, "random", 0), (4097, "random", 8), (6000, "near", 0),
                                          (6000, "near", 24), (2048, "equal", 16), (1, "random", 0)])
def test_pass_is_a_stable_digit_sort(n, kind, shift):
    rng = np.random.default_rng(n + shift)
    if kind == "random":
        keys = rng.integers(0, 1 << 40, size=n, dtype=np.uint64)
    elif kind == "near":
        keys = np.sort(rng.integers(0, 1 << 32, size=n, dtype=np.uint64))
        swap = rng.integers(0, n - 1, size=n // 20)  # particles that moved a little
        keys[swap], keys[swap + 1] = keys[swap + 1].copy(), keys[swap].copy()
    else:
        keys = np.full(n, 0x123456, dtype=np.uint64)
    vals = np.arange(n, dtype=np.uint32)
    got_k, got_v = sm.onesweep_pass(keys, vals, shift)
    digit = (keys >> np.uint64(shift)) & np.uint64(0xFF)
    order = np.argsort(digit, kind="stable")
    assert np.array_equal(got_k, keys[order])
    assert np.array_equal(got_v, vals[order])


def test_passes_compose_to_a_full_sort():
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 1 << 32, size=3000, dtype=np.uint64)
    k, v = keys, np.arange(len(keys), dtype=np.uint32)
    for p in range(4):
        k, v = sm.onesweep_pass(k, v, 8 * p)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(k, keys[order]) and np.array_equal(v, order.astype(np.uint32))


@pytest.mark.parametrize("tiles,grid", [(1, 4), (37, 1), (200, 8), (977, 64), (1954, 444)])
def test_persistent_lookback_is_exact_and_ends(tiles, grid):
    """The pass's grid is the blocks resident at once, each taking tiles in
    ticket order until none is left (1,954 tiles of the 4m plasma on 444
    resident blocks).  Under random interleavings every tile's look-back ends
    with the exact count of its digit over all earlier tiles: a block waits
    only on tiles with earlier tickets, which running blocks hold."""
    rng = np.random.default_rng(tiles)
    counts = rng.integers(0, 9, size=tiles)
    for seed in range(3):
        excl, rounds = sm.lookback_schedule(counts, grid, seed)
        assert np.array_equal(excl, np.concatenate([[0], np.cumsum(counts)[:-1]]))
        assert rounds >= (1 if tiles > 1 else 0)
