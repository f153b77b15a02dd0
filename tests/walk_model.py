"""Restatement, in Python, of two staging schedules of the fast walk
(group_walk in pot_b200/csrc/pot_walk_fast.cu).  Test infrastructure: it
pins the bookkeeping, not the CUDA code.

* Leaf gather: the staged leaves' particle counts are scanned; chunk by
  chunk of 32 positions, the leaves that start inside the chunk set one bit
  each (a warp OR-reduction), and the position's leaf is the number of leaves
  started before the chunk plus the set bits at or below it, minus one.
* Cell flushes: cells arrive in batches of at most 32 per traversal round; a
  flush at 64 or more staged evaluates whole units of the unrolled loop and
  carries the rest to the front, and the last flush pads to a whole unit."""


def leaf_of_positions(counts):
    """The leaf index the gather reads for each position 0..sum(counts)-1."""
    assert all(c > 0 for c in counts), "no staged leaf is empty"
    starts, run = [], 0
    for c in counts:
        starts.append(run)
        run += c
    total = run
    out = []
    before = 0
    for base in range(0, total, 32):
        bits = 0
        for st in starts:
            if 0 <= st - base < 32:
                bits |= 1 << (st - base)
        for lane in range(32):
            g = base + lane
            if g < total:
                le = (2 << lane) - 1
                out.append(before + bin(bits & le).count("1") - 1)
        before += bin(bits).count("1")
    return out


def cell_flushes(batches, unit, flush_at=64):
    """Cell ids in evaluation order (None for padding) and the largest number
    staged at once, for cells arriving in the given batches (ids in order)."""
    staged, order, high = [], [], 0
    batches = list(batches)
    for r, batch in enumerate(batches + [[]]):
        done = r == len(batches)
        staged.extend(batch)
        high = max(high, len(staged))
        if len(staged) >= flush_at or (done and staged):
            n = len(staged)
            padded = (n + unit - 1) // unit * unit if done else n // unit * unit
            evaluated = staged[:padded] + [None] * max(0, padded - n)
            order.extend(evaluated)
            staged = staged[padded:] if padded < n else []
            high = max(high, padded)
    return order, high
