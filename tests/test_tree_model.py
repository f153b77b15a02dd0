"""The GPU build's index arithmetic (numpy model in tree_model.py) against
the reference tree: cell ownership, pre-order numbering and children
reproduce the insertion octree of pot.c:1457-1643 exactly."""
import numpy as np
import pytest

import tree_model as tm
from common import SMALL, oracle_snapshot


@pytest.mark.parametrize("seed,N", [(1, 8193), (3, 3001)])
def test_model_tree_equals_reference_tree(seed, N):
    d = dict(SMALL, N=N)
    o = oracle_snapshot(d, seed=seed, mode="reference")
    P = o.particles()
    w = 2.0 * d["r"] * d["mpp"]
    keys = tm.morton_keys(P["x"], P["y"], P["z"], w)
    perm = np.argsort(keys, kind="stable")
    ks = keys[perm]
    tree = tm.build(ks, 1)
    ints, leaves = tm.canonical(ks, perm, tree)
    o.build_tree()
    od = o.tree_dump()
    assert ints == sorted(zip(od["int_level"].tolist(), od["int_path"].tolist()))
    assert leaves == sorted(zip(od["leaf_part"].tolist(), od["leaf_level"].tolist(), od["leaf_path"].tolist()))
    # parents precede children (pre-order), as the upward pass assumes
    par = tree["parent"]
    assert par[0] == -1 and np.all(par[1:] < np.arange(1, tree["M"])) and np.all(par[1:] >= 0)


def test_model_bucket_tree_partitions_particles():
    d = dict(SMALL, N=8193)
    o = oracle_snapshot(d, seed=2, mode="gpu")
    P = o.particles()
    keys = tm.morton_keys(P["x"], P["y"], P["z"], 2.0 * d["r"] * d["mpp"])
    perm = np.argsort(keys, kind="stable")
    for L in (8, 16):
        tree = tm.build(keys[perm], L)
        _, leaves = tm.canonical(keys[perm], perm, tree)
        assert sorted(l[0] for l in leaves) == list(range(d["N"]))
        counts = {}
        for part, lev, path in leaves:
            counts[(lev, path)] = counts.get((lev, path), 0) + 1
        assert max(counts.values()) <= L


def test_morton_key_matches_midpoint_descent():
    """Keys equal the comparisons of the reference's descent (pot.c:1522-1553)
    on points placed exactly on cell boundaries."""
    w = 1.41609e-06
    # boundaries by the reference's recursive halving
    lo, hi = 0.0, w
    pts = []
    for _ in range(10):
        mid = (lo + hi) / 2.0
        pts += [mid, np.nextafter(mid, -1), np.nextafter(mid, 2)]
        lo = mid
    x = np.array(pts)
    k = tm.morton_keys(x, x, x, w)
    for xi, ki in zip(x, k):
        l, h = 0.0, w
        want = 0
        for _ in range(21):
            m = (l + h) / 2.0
            b = 0 if xi < m else 1
            if b:
                l = m
            else:
                h = m
            want = (want << 3) | (b * 7)
        assert int(ki) == want


@pytest.mark.parametrize("N,L,seed", [(20000, 16, 1), (3001, 1, 2), (50000, 8, 3)])
def test_device_searches_find_cell_ends_and_children(N, L, seed):
    """The searches of k_finish_nodes (cell_end, child_starts), restated in
    tree_model.py, give every cell's last slot and child boundaries of the
    model tree, including clustered keys that make deep, lopsided cells."""
    rng = np.random.default_rng(seed)
    pts = rng.normal(0.5, 0.12, size=(N, 3)).clip(0.001, 0.999)
    keys = np.sort(tm.morton_keys(pts[:, 0], pts[:, 1], pts[:, 2], 1.0))
    tree = tm.build(keys, L)
    n = len(keys)
    for c in range(tree["M"]):
        f, l = int(tree["first"][c]), int(tree["level"][c])
        shift = 63 - 3 * l
        pfx = int(keys[f]) >> shift
        end = tm.cell_end(keys, f, n, shift, pfx)
        assert end == int(tree["last"][c]) + 1, c
        digits = (keys[f:end] >> np.uint64(shift - 3)) & np.uint64(7)
        want = [f + int(np.searchsorted(digits, np.uint64(d), side="left")) for d in range(1, 8)]
        assert tm.child_starts(keys, f, end, shift - 3) == want, c
