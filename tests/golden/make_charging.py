"""Write tests/golden/charging.npz: the grain's charging curve from the
reference program itself, for the GPU's ensemble tests of grain charging.

The reference pot.c -- compiled from its own sources by oracle/build.py with
the single-rank MPI stand-in, SCEPTIC reinjection on (the ``sceptic``
library) -- runs two plasmas of 8,193 particles (4,096 ions and 4,096
electrons in a sphere of 5 Debye lengths, Te = Ti, no flow, no field, theta
0.5, dt = 0.01 / omega_pe) for 2,000 steps from its own init_particles:

* ``small``    the grain of radius 0.1 Debye lengths (8 seeds, 1..8);
* ``grain05``  a grain of radius 0.5 Debye lengths, which collects about
  16 times more charge in the same time (16 seeds, 1..16).

WELL512 is seeded from splitmix64 of the seed.  After every step the grain
charge (e) is recorded: build_tree and move_particles exactly as run()
calls them (pot.c:4261-4386), grain update included (pot.c:2825-2867).

Each seed runs in its own process (the compiled reference keeps one run per
process), the seeds in parallel.

Usage (where the reference tree is present):
    python tests/golden/make_charging.py [--steps 2000]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SMALL = dict(N=8193, r=1000, dt=3.37727e-15, mpp=7.08046e-10, soft=1.41609e-09, Te=11600.0, Ti=11600.0,
             x_drift=0.0, a=1.41609e-08, settle=0.0, theta=0.5)
CASES = {"small": (SMALL, 8), "grain05": (dict(SMALL, a=7.08045e-08), 16)}


def one_seed(args):
    case, seed, steps = args
    sys.path.insert(0, ROOT)
    from oracle.oracle import RefLib, RunParams
    ref = RefLib("sceptic", build=False).setup(RunParams(**CASES[case][0]), seed=seed)
    q = np.zeros(steps, np.int32)
    t0 = time.perf_counter()
    for k in range(steps):
        ref.step()
        q[k] = ref.grain()["q"]
    return case, seed, q, time.perf_counter() - t0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--steps", type=int, default=2000)
    a = ap.parse_args(argv)
    from oracle import build as obuild
    obuild.build_ref(variants=("sceptic",))
    jobs = [(c, s_, a.steps) for c, (_, n) in CASES.items() for s_ in range(1, n + 1)]
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        res = pool.map(one_seed, jobs)
    arrays, meta = {}, {"variant": "sceptic", "steps": a.steps, "cases": {}}
    for c, (params, n) in CASES.items():
        rc = sorted((r for r in res if r[0] == c), key=lambda r: r[1])
        arrays["q_" + c] = np.stack([r[2] for r in rc])
        meta["cases"][c] = {"params": params, "seeds": [r[1] for r in rc],
                            "seconds_per_seed": [round(r[3], 1) for r in rc],
                            "window_mean_1001_2000": [float(r[2][1000:2000].mean()) for r in rc]
                            if a.steps >= 2000 else None}
    np.savez_compressed(os.path.join(HERE, "charging.npz"), **arrays)
    with open(os.path.join(HERE, "charging.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta))
    return 0


if __name__ == "__main__":
    sys.exit(main())
