"""Restatement, in Python, of one pass of the device radix sort (k_os_pass
in pot_b200/csrc/pot_sort.cu) in the kernel's own order.  Test
infrastructure: it pins the ranking schedule, not the CUDA code.

A tile is 2,048 keys; warp w holds keys [256 w, 256 w + 256) of it, round r
the 32 at 256 w + 32 r.  Within a warp a key's rank is the warp's running
count of its digit before the round plus the lanes below it with the same
digit (the kernel's __match_any_sync); the warps' counts are then turned
into per-warp exclusive prefixes, the tile's digit starts are an exclusive
scan of its counts, and a key's staged position is digit start + warp
prefix + rank.  The digit's offset over earlier tiles is what the decoupled
look-back sums (counts and inclusive prefixes of earlier tiles), modelled
here by its value."""
import numpy as np

TILE, WARPS, ROUNDS, LANES, BINS = 2048, 8, 8, 32, 256


def onesweep_pass(keys, vals, shift):
    keys = np.asarray(keys, dtype=np.uint64)
    vals = np.asarray(vals, dtype=np.uint32)
    n = len(keys)
    digit = ((keys >> np.uint64(shift)) & np.uint64(0xFF)).astype(np.int64)
    goff = np.concatenate([[0], np.cumsum(np.bincount(digit, minlength=BINS))[:-1]])
    out_k = np.zeros(n, dtype=np.uint64)
    out_v = np.zeros(n, dtype=np.uint32)
    before_tiles = np.zeros(BINS, dtype=np.int64)  # the look-back's sum for this tile
    for base in range(0, n, TILE):
        wcnt = np.zeros((WARPS, BINS), dtype=np.int64)
        rank = {}
        for w in range(WARPS):
            for r in range(ROUNDS):
                start = base + w * ROUNDS * LANES + r * LANES
                d = [int(digit[i]) if i < n else BINS for i in range(start, start + LANES)]
                seen = {}
                for lane in range(LANES):
                    if d[lane] == BINS:
                        continue
                    lower = seen.get(d[lane], 0)  # lanes below with the same digit
                    rank[start + lane] = int(wcnt[w, d[lane]]) + lower
                    seen[d[lane]] = lower + 1
                for dd, c in seen.items():
                    wcnt[w, dd] += c
        wpre = np.cumsum(wcnt, axis=0) - wcnt
        cnt = wcnt.sum(axis=0)
        loc = np.concatenate([[0], np.cumsum(cnt)[:-1]])
        m = min(TILE, n - base)
        s_key = np.zeros(m, dtype=np.uint64)
        s_val = np.zeros(m, dtype=np.uint32)
        for i in range(base, base + m):
            t = i - base
            w = t // (ROUNDS * LANES)
            d = int(digit[i])
            p = int(loc[d] + wpre[w, d] + rank[i])
            s_key[p] = keys[i]
            s_val[p] = vals[i]
        for p in range(m):
            d = int((int(s_key[p]) >> shift) & 0xFF)
            o = int(goff[d] + before_tiles[d] + (p - loc[d]))
            out_k[o] = s_key[p]
            out_v[o] = s_val[p]
        before_tiles += cnt
    return out_k, out_v


AGG, PRE, LOOKBACK = 1, 2, 8  # status flags and tiles read per look-back round (OS_FLAG_*, OS_LOOKBACK)


def lookback_schedule(counts, grid, seed, max_events=10_000_000):
    """The pass's tile scheduling and decoupled look-back for one digit, with
    `grid` resident blocks interleaved at random.  A block takes the next
    ticket (tile), publishes its count (AGG; tile 0 publishes PRE), then reads
    LOOKBACK earlier status words per round, adding counts until it meets an
    inclusive prefix (PRE) and stopping the round at a word not yet published;
    it then publishes PRE with its inclusive prefix and takes the next ticket
    until none is left.  Each scheduling event advances one block by one
    step (a publish or one round of reads).  Returns each tile's exclusive
    prefix and the most rounds any tile spent looking back; raises if the
    blocks stop making progress."""
    rng = np.random.default_rng(seed)
    n = len(counts)
    st_flag = np.zeros(n, dtype=np.int64)
    st_val = np.zeros(n, dtype=np.int64)
    excl_out = np.full(n, -1, dtype=np.int64)
    ticket = 0
    blocks = [{"state": "take"} for _ in range(grid)]
    live = list(range(grid))
    max_rounds = 0
    events = 0
    while live:
        events += 1
        if events > max_events:
            raise RuntimeError("no progress")
        i = live[rng.integers(len(live))]
        b = blocks[i]
        if b["state"] == "take":
            if ticket >= n:
                live.remove(i)
                continue
            b.update(state="publish", tile=ticket, excl=0, j=ticket - 1, rounds=0)
            ticket += 1
        elif b["state"] == "publish":
            t = b["tile"]
            st_flag[t], st_val[t] = (PRE if t == 0 else AGG), counts[t]
            b["state"] = "done" if t == 0 else "look"
        elif b["state"] == "look":
            j = b["j"]
            reads = [(st_flag[j - q], st_val[j - q]) if j - q >= 0 else (0, 0) for q in range(LOOKBACK)]
            b["rounds"] += 1
            used, found = 0, False
            for flag, val in reads:
                if flag == 0:
                    break
                b["excl"] += val
                used += 1
                if flag == PRE:
                    found = True
                    break
            b["j"] = j - used
            if found:
                t = b["tile"]
                st_flag[t], st_val[t] = PRE, b["excl"] + counts[t]
                b["state"] = "done"
        if b["state"] == "done":
            excl_out[b["tile"]] = b["excl"]
            max_rounds = max(max_rounds, b.get("rounds", 0))
            b["state"] = "take"
    return excl_out, max_rounds
