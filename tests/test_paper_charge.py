"""The reference's published long run as the pin for the equilibrium grain
charge (tests/golden/paper_charge.json, written by make_paper_charge.py from
the reference's ``output/2016 TH PPCF paper/np-with-sph-macro.dat``; the pin
is gasma.R:127).

``macro_windows`` reads a macroscopic file in the reference's format (the
one ``potgpu`` writes, pot.c's 35 columns) and returns the same per-
microsecond statistics as the fixture, so that a ``potgpu`` run at pot.c's
defaults compares with the published run window by window.
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "paper_charge.json")


def _load():
    with open(FIX) as f:
        return json.load(f)


def macro_windows(path_or_rows, first_us: int = 1, last_us: int = 6) -> dict:
    """Mean and sample standard deviation of DGQ per microsecond [k, k + 1)
    and over t >= 2 us, from a macroscopic file (or a (time, q) pair)."""
    if isinstance(path_or_rows, str):
        d = np.genfromtxt(path_or_rows, names=True)
        t, q = d["TIME"], d["DGQ"]
    else:
        t, q = (np.asarray(a, dtype=np.float64) for a in path_or_rows)
    out = {}
    for k in range(first_us, last_us):
        m = (t >= k * 1e-6) & (t < (k + 1) * 1e-6 - 1e-12)
        if k == last_us - 1:
            m = t >= k * 1e-6
        if m.sum() > 1:
            out["%d-%d us" % (k, k + 1)] = dict(rows=int(m.sum()), mean=float(q[m].mean()), sd=float(q[m].std(ddof=1)))
    m = t >= 2e-6
    if m.sum() > 1:
        out["t >= 2 us"] = dict(rows=int(m.sum()), mean=float(q[m].mean()), sd=float(q[m].std(ddof=1)))
    return out


def _series(fx):
    t, q = [], []
    for seg in fx["series"]:
        n = len(seg["q_e"])
        t.append(seg["t0_s"] + seg["row_s"] * np.arange(n))
        q.append(np.asarray(seg["q_e"], dtype=np.float64))
    return np.concatenate(t), np.concatenate(q)


def test_fixture_is_the_published_run():
    fx = _load()
    assert fx["params"]["N"] == 150001 and fx["params"]["dt"] == 1e-12
    assert fx["pin"]["mean"] == -82.6761 and abs(fx["pin"]["sd"] ** 2 - 25.6239) < 1e-9
    # the grain is introduced after the settling time, 0.5 us
    assert 5e-7 <= fx["first_charged_row_s"] < 5.1e-7
    t, q = _series(fx)
    assert t[-1] > 5.99e-6 and np.all(np.diff(t) > 0)
    assert np.all(q <= 0) and q[t >= 1.5e-6].max() < -60


def test_windows_recomputed_from_the_series():
    fx = _load()
    w = macro_windows(_series(fx))
    for k, v in fx["windows"].items():
        assert w[k]["rows"] == v["rows"]
        assert abs(w[k]["mean"] - v["mean"]) < 1e-9 and abs(w[k]["sd"] - v["sd"]) < 1e-9


def test_pin_agrees_with_the_equilibrium_windows():
    """Every microsecond from 2 us on lies within one of the pin's standard
    deviations of its mean, and so does the mean over t >= 2 us: the series
    is at equilibrium there, and the pin describes it."""
    fx = _load()
    pin, sd = fx["pin"]["mean"], fx["pin"]["sd"]
    for k in ("2-3 us", "3-4 us", "4-5 us", "5-6 us", "t >= 2 us"):
        assert abs(fx["windows"][k]["mean"] - pin) < sd, k
