"""Grain charging on the GPU against the reference program's own charging.

tests/golden/charging.npz holds the grain charge after each of 2,000 steps
of the reference pot.c itself (SCEPTIC reinjection, 8,193 particles, Te =
Ti, no flow, theta 0.5), written by tests/golden/make_charging.py for two
grains: radius 0.1 Debye lengths (the benchmark's small plasma, seeds 1..8)
and 0.5 Debye lengths (seeds 1..16; it collects about 16 times more charge,
so the comparison is sharper).  The GPU runs the same plasmas in both forms
from its own init_particles (Philox streams, so only the statistics can
agree), and the mean charge over steps 1,001-2,000 (from the device's
running charge sum) is compared with the reference's ensemble: the two
means must agree within 1 % of the reference's or three standard errors of
the difference, each standard error from the seed-to-seed spread.
"""
import json
import os

import numpy as np
import pytest

from common import SMALL, run_config
from pot_b200.gpu import Run

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "charging.npz")
CASES = {"small": (dict(SMALL), 12), "grain05": (dict(SMALL, a=7.08045e-08), 16)}


def _reference_window_means(case):
    q = np.load(GOLD)["q_" + case].astype(np.float64)
    return q[:, 1000:2000].mean(1)


def _gpu_window_means(params, form, seeds):
    cfg = run_config(params)
    kw = dict(leaf_size=8) if form == "fast" else {}
    out = []
    for s in seeds:
        with Run(cfg, form=form, seed=s, **kw) as r:
            r.init_particles()
            s1 = r.step(1000)
            s2 = r.step(1000)
            assert s2["status"] == 0 and s2["t_steps"] == 2000
            out.append((s2["q_sum"] - s1["q_sum"]) / 1000.0)
    return np.array(out)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["small", "grain05"])
@pytest.mark.parametrize("form", ["plain", "fast"])
def test_grain_charging_matches_reference_ensemble(case, form):
    params, n = CASES[case]
    ref = _reference_window_means(case)
    gpu = _gpu_window_means(params, form, range(101, 101 + n))
    m_r, m_g = ref.mean(), gpu.mean()
    se = np.sqrt(ref.var(ddof=1) / len(ref) + gpu.var(ddof=1) / len(gpu))
    tol = max(0.01 * abs(m_r), 3.0 * se)
    assert abs(m_g - m_r) <= tol, (case, form, m_g, m_r, se, gpu.tolist(), ref.tolist())


def test_charging_fixture_metadata():
    """The fixture holds the reference's 8,193-particle plasmas, 2,000 steps,
    and both grains charge negatively, the larger one more."""
    with open(os.path.join(HERE, "golden", "charging.json")) as f:
        meta = json.load(f)
    assert meta["steps"] == 2000 and meta["variant"] == "sceptic"
    d = np.load(GOLD)
    for case, (params, _) in CASES.items():
        m = meta["cases"][case]
        assert m["params"]["N"] == SMALL["N"] and m["params"]["a"] == params["a"]
        q = d["q_" + case]
        assert q.shape == (len(m["seeds"]), 2000)
        assert (q[:, -1] < 0).all()
    assert d["q_grain05"][:, 1000:].mean() < 5 * d["q_small"][:, 1000:].mean()
