"""The reinjection kernel's warp schedule for the orbit-angle integral
(restated lane by lane in reinject_model.py) against the oracle's sequential
integral (pot.c:433-492), bit for bit, on seeded inputs spanning the edge
potentials, speeds and domain sizes of the workloads."""
import struct

import numpy as np

import reinject_model as rm
from oracle.oracle import Oracle


def _bits(x):
    return struct.pack("<d", x)


def test_warp_schedule_matches_sequential_integral():
    L = Oracle.lib()
    rng = np.random.default_rng(20)
    stats = {}
    n = 0
    for rol in (5.0, 10.0, 20.0):
        for chi in (-2.0, -0.5, -0.05, 0.2, 1.0):
            for i in range(12):
                u = abs(rng.standard_normal()) + 0.3 * rng.random()
                u2 = u * u
                if u2 < chi:
                    continue
                b = float(np.sqrt(rng.random() * (1.0 - chi / u2)))
                mld = 0.01 if i % 2 else 0.1
                want = L.pto_integrate_for_alpha_dev(b, chi, u2, rol, mld)
                got = rm.warp_alpha(b, chi, u2, rol, mld, stats)
                # a NaN alpha (the orbit has no turning point; the reference draws
                # again, and so does the kernel) matches any NaN, whatever its sign
                assert _bits(got) == _bits(want) or (np.isnan(got) and np.isnan(want)), \
                    (rol, chi, u2, b, mld, got, want)
                n += 1
    assert n > 150
    # the guessed second interval was taken in a good share of the rounds
    assert stats["two"] > 0.25 * stats["rounds"], stats
