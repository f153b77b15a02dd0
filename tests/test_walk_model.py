"""The fast walk's staging schedules, restated in walk_model.py: the leaf
gather finds each position's leaf as a search over the leaf starts would,
and the cell flushes evaluate every staged cell exactly once, in arrival
order, within the shared-memory cell buffer (104 entries)."""
import bisect

import numpy as np
import pytest

import walk_model as wm

FW_CELLS = 104


@pytest.mark.parametrize("seed", range(6))
def test_leaf_gather_matches_a_search_over_starts(seed):
    rng = np.random.default_rng(seed)
    for _ in range(50):
        nleaf = int(rng.integers(1, 64))  # a flush holds at most 63 leaves
        counts = [int(c) for c in rng.integers(1, 40 if seed % 2 else 17, size=nleaf)]
        starts = np.concatenate([[0], np.cumsum(counts)[:-1]]).tolist()
        want = [bisect.bisect_right(starts, g) - 1 for g in range(sum(counts))]
        assert wm.leaf_of_positions(counts) == want


@pytest.mark.parametrize("unit", [8, 16, 32])  # two targets per lane; one; one with a split list
def test_cell_flushes_evaluate_each_cell_once(unit):
    rng = np.random.default_rng(unit)
    for _ in range(200):
        sizes = rng.integers(0, 33, size=int(rng.integers(1, 40)))
        batches, nxt = [], 0
        for s in sizes:
            batches.append(list(range(nxt, nxt + int(s))))
            nxt += int(s)
        order, high = wm.cell_flushes(batches, unit)
        cells = [c for c in order if c is not None]
        assert cells == list(range(nxt))  # every cell once, in arrival order
        assert len(order) % unit == 0  # whole units only
        assert len(order) - nxt < unit  # padding only at the last flush, less than a unit
        assert high <= FW_CELLS
