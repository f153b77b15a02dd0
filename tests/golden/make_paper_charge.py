"""Write tests/golden/paper_charge.json: the grain charge of the reference's
published long run, as the distributional pin for the GPU's equilibrium
charge.

The reference ships the macroscopic time series of one 150,001-particle run
at pot.c's defaults (T = 220 K for both species, a = 2.5 um, R = 4e-4 m,
dt = 1e-12 s, the grain introduced after the 0.5 us settling time) in
``output/2016 TH PPCF paper/np-with-sph-macro.dat``; its analysis script
``gasma.R`` (lines 7-11 for the parameters, 127 for the pin) quotes the
equilibrium charge as -82.6761 e with variance 25.6239 e^2.  This script
reads the series (TIME and DGQ columns) and stores:

* the pin as gasma.R states it;
* the grain charge's mean and standard deviation over each microsecond from
  1 us to 6 us, and over t >= 2 us;
* the series itself from 0.5 us on, as integers, in two segments of evenly
  spaced rows (every 200 steps up to 1 us, every 2,000 after).

Usage (where the reference tree is present; its root from
$POT_REFERENCE_ROOT, else the directory named ``reference`` beside this
repository):
    python tests/golden/make_paper_charge.py
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SERIES = os.path.join("output", "2016 TH PPCF paper", "np-with-sph-macro.dat")


def reference_root() -> str:
    env = os.environ.get("POT_REFERENCE_ROOT")
    return env if env else os.path.join(os.path.dirname(ROOT), "reference")


def window_stats(t: np.ndarray, q: np.ndarray) -> dict:
    """Mean and sample standard deviation of the grain charge per
    microsecond [k, k + 1) for k = 1..5 and over t >= 2 us."""
    out = {}
    for k in range(1, 6):
        m = (t >= k * 1e-6) & (t < (k + 1) * 1e-6 - 1e-12)
        if k == 5:
            m = t >= 5e-6
        if m.sum() > 1:
            out["%d-%d us" % (k, k + 1)] = dict(rows=int(m.sum()), mean=float(q[m].mean()),
                                                  sd=float(q[m].std(ddof=1)))
    m = t >= 2e-6
    out["t >= 2 us"] = dict(rows=int(m.sum()), mean=float(q[m].mean()), sd=float(q[m].std(ddof=1)))
    return out


def main() -> None:
    path = os.path.join(reference_root(), SERIES)
    d = np.genfromtxt(path, names=True)
    t, q = d["TIME"], d["DGQ"]
    first = float(t[np.nonzero(q)[0][0]]) if np.any(q) else None
    segments = []
    for lo, hi in ((5e-7, 1e-6 + 1e-13), (1e-6 + 1e-13, 1.0)):
        m = (t >= lo) & (t < hi)
        ts = t[m]
        step = float(np.median(np.diff(ts)))
        assert np.allclose(np.diff(ts), step, rtol=1e-6, atol=1e-15), "rows not evenly spaced"
        segments.append(dict(t0_s=float(ts[0]), row_s=step, q_e=[int(round(x)) for x in q[m]]))
    out = {
        "source": SERIES,
        "params": dict(N=150001, T_e=220.0, T_i=220.0, a=2.5e-6, R=4e-4, dt=1e-12, settle=5e-7),
        "pin": dict(mean=-82.6761, variance=25.6239, sd=float(np.sqrt(25.6239)), where="gasma.R:127"),
        "first_charged_row_s": first,
        "windows": window_stats(t, q),
        "series": segments,
    }
    with open(os.path.join(HERE, "paper_charge.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print(json.dumps({k: out[k] for k in ("pin", "first_charged_row_s", "windows")}, indent=1))


if __name__ == "__main__":
    main()
