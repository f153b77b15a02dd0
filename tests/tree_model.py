"""numpy model of the GPU octree build (pot_b200/csrc/pot_tree.cu).

Test infrastructure: a vectorised restatement of the kernels' index
arithmetic -- Morton keys by midpoint descent, pair levels, pre-order cell
ownership, children by digit search -- so that the layout can be checked
against the reference tree on the CPU, before and independently of the GPU.
"""
from __future__ import annotations

import numpy as np

MAX_LEVELS = 21
SLOT_DIGITS = (4, 5, 0, 1, 2, 3, 6, 7)


def morton_keys(x, y, z, w):
    """63-bit keys from the comparisons x < mid, mid = (lo + hi) / 2
    (pot.c:1522-1553), level 1 in bits 62..60."""
    lo = [np.zeros_like(x) for _ in range(3)]
    hi = [np.full_like(x, w) for _ in range(3)]
    coords = (x, y, z)
    key = np.zeros(x.shape, np.uint64)
    for _ in range(MAX_LEVELS):
        digit = np.zeros(x.shape, np.uint64)
        for d in range(3):
            mid = (lo[d] + hi[d]) * 0.5
            b = ~(coords[d] < mid)
            lo[d] = np.where(b, mid, lo[d])
            hi[d] = np.where(b, hi[d], mid)
            digit |= b.astype(np.uint64) << np.uint64(2 - d)
        key = (key << np.uint64(3)) | digit
    return key


def lcp_levels(a, b):
    x = a ^ b
    out = np.full(a.shape, MAX_LEVELS, np.int64)
    nz = x != 0
    # number of leading zeros of a 64-bit value
    xv = x[nz]
    lz = np.zeros(xv.shape, np.int64)
    for shift in (32, 16, 8, 4, 2, 1):
        m = (xv >> np.uint64(64 - shift)) == 0
        lz = np.where(m, lz + shift, lz)
        xv = np.where(m, xv << np.uint64(shift), xv)
    out[nz] = (lz - 1) // 3
    return out


def build(keys_sorted, L=1):
    """Cells of the tree over sorted keys, as the kernels number them.

    Returns dict(first, last, level, child[M, 8] codes) with codes >= 0 a
    cell, -1 empty, -2 - slot a single-particle leaf (L = 1) or -2 - (8k + d)
    a bucket leaf with lrange[(8k + d)] = (start, count)."""
    k = keys_sorted
    n = len(k)
    P = n - L
    li = lcp_levels(k[:P], k[L:L + P])
    lvl = np.minimum(li, MAX_LEVELS - 1)
    prev = np.concatenate([[-1], lvl[:-1]])
    cnt = np.maximum(lvl - prev, 0)
    base = np.concatenate([[0], np.cumsum(cnt)[:-1]])
    M = int(cnt.sum())
    first = np.zeros(M, np.int64)
    level = np.zeros(M, np.int64)
    for i in np.nonzero(cnt)[0]:
        lo = 0 if i == 0 else lvl[i - 1] + 1
        for l in range(lo, lvl[i] + 1):
            idx = base[i] + (l - lo)
            first[idx] = i
            level[idx] = l
    last = np.zeros(M, np.int64)
    child = np.full((M, 8), -1, np.int64)
    parent = np.full(M, -1, np.int64)
    lrange = {}
    for c in range(M):
        f, l = first[c], level[c]
        shift = np.uint64(63 - 3 * l)
        pfx = k[f] >> shift
        same = (k >> shift) == pfx
        last[c] = f + np.argmin(same[f:]) - 1 if not same[f:].all() else n - 1
        rng = np.arange(f, last[c] + 1)
        digits = (k[rng] >> np.uint64(63 - 3 * (l + 1))) & np.uint64(7)
        for d in range(8):
            members = rng[digits == d]
            if len(members) == 0:
                continue
            sc = members[0]
            if len(members) <= L:
                if L == 1:
                    child[c, d] = -2 - sc
                else:
                    e = 8 * c + d
                    child[c, d] = -2 - e
                    lrange[e] = (sc, len(members))
            else:
                lo = 0 if sc == 0 else lvl[sc - 1] + 1
                kc = base[sc] + (l + 1 - lo)
                assert kc < M and kc > c and first[kc] == sc and level[kc] == l + 1
                child[c, d] = kc
                parent[kc] = c
    return dict(first=first, last=last, level=level, child=child, parent=parent, lrange=lrange, M=M)


def canonical(keys_sorted, perm, tree):
    """Internal cells (level, path) and leaves (original index, level, path)."""
    k = keys_sorted
    ints, leaves = [], []
    for c in range(tree["M"]):
        l = int(tree["level"][c])
        pfx = 0 if l == 0 else int(k[tree["first"][c]] >> np.uint64(63 - 3 * l))
        ints.append((l, pfx))
        for d in range(8):
            code = int(tree["child"][c, d])
            if code < -1:
                e = -2 - code
                if e in tree["lrange"]:
                    s0, cnt = tree["lrange"][e]
                else:
                    s0, cnt = e, 1
                for j in range(cnt):
                    leaves.append((int(perm[s0 + j]), l + 1, (pfx << 3) | d))
    return sorted(ints), sorted(leaves)


# ---- the device's searches over a cell's key range (k_finish_nodes) ----

def _first_fail8(k, a, b, pred):
    """first_fail8: seven probes per round keep one eighth of [a, b); the
    last eight or fewer are read at once."""
    while b - a > 8:
        span = b - a
        p = [a + ((span * (i + 1)) >> 3) for i in range(7)]
        ok = [pred(int(k[q])) for q in p]
        na, nb = a, b
        for i in range(7):
            if ok[i]:
                na = p[i] + 1
        for i in range(6, -1, -1):
            if not ok[i]:
                nb = p[i]
        a, b = na, nb
    return a + sum(1 for i in range(8) if a + i < b and pred(int(k[a + i])))


def cell_end(k, f, n, shift, pfx):
    """cell_end: f + 2^e probed for seven exponents per round until one
    leaves the cell (key >> shift != pfx), then the bracket searched."""
    same = lambda key: (key >> shift) == pfx
    a, b = f + 1, n
    for e0 in range(0, 32, 7):
        q = [f + (1 << (e0 + i)) for i in range(7)]
        ok = [qq < n and same(int(k[qq])) for qq in q]
        left = False
        for i in range(7):
            if ok[i]:
                a = q[i] + 1
        for i in range(6, -1, -1):
            if not ok[i]:
                b = min(q[i], n)
                left = True
        if left:
            break
    return _first_fail8(k, a, b, same)


def child_starts(k, f, e, shift):
    """child_starts: s[c] for c = 1..7, the first slot of [f, e) whose digit
    at shift is >= c, by seven bisections side by side."""
    lo, hi = [f] * 7, [e] * 7
    span = e - f
    while span > 0:
        for c in range(7):
            if lo[c] < hi[c]:
                m = lo[c] + ((hi[c] - lo[c]) >> 1)
                if ((int(k[m]) >> shift) & 7) < c + 1:
                    lo[c] = m + 1
                else:
                    hi[c] = m
        span >>= 1
    return lo
