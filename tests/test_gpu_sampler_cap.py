"""POT_OPT_CHI_CAP: the SCEPTIC sampler's edge potential capped for the
batch and serving family (off by default, where the reference's behaviour
holds).

* A run whose edge potential stays below the cap is bit-identical with and
  without the option (both forms).
* A run whose edge potential is far above it -- a grain given a large
  positive charge in cold ions, so the potential at the domain edge reads
  many kTi/e -- stops with POT_E_ITER and warn bit 64 without the option (the
  reference's inverse CDF is NaN there and it would retry without end,
  prng.c:171-214, pot.c:582-599), and runs on with it, warn bit 512 set,
  every particle inside the domain.
"""
import numpy as np
import pytest

from common import SMALL, run_config
from pot_b200.gpu import WARN_CHI_CAP, PotError, Run, RunConfig

pytestmark = pytest.mark.gpu


def _cold(N=20001):
    kb, eps0, qe, me = 1.38065e-23, 8.85419e-12, 1.6021766e-19, 9.109383e-31
    Te = 11600.0
    lam = 3.0 * (N - 1) * qe * qe / (4096.0 * 3.14159265358979 * eps0 * kb * Te)
    R = 8.0 * lam
    n = (N - 1) / (4.0 / 3.0 * 3.14159265358979 * R ** 3)
    wpe = np.sqrt(n / 2 * qe * qe / (eps0 * me))
    return RunConfig(N=N, r=1000, mpp=R / 1000, a=0.05 * lam, soft=0.01 * lam, dt=0.005 / wpe, Te=Te, Ti=Te / 10,
                     x_drift=0.3 * np.sqrt(kb * Te / (1836.15 * me)), theta=0.5)


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_cap_changes_nothing_below_it(form):
    cfg = run_config(dict(SMALL, N=20001))
    out = []
    for cap in (False, True):
        with Run(cfg, form=form, seed=21, chi_cap=cap) as r:
            r.init_particles()
            st = r.step(60)
            P, g = r.download()
        assert st["status"] == 0 and not (st["warn"] & WARN_CHI_CAP)
        out.append((P.tobytes(), g["q"], g["chi_b"], st["q_sum"]))
    assert out[0] == out[1]


@pytest.mark.parametrize("form", ["plain", "fast"])
def test_cap_keeps_a_run_going_where_the_sampler_is_undefined(form):
    cfg = _cold()
    with Run(cfg, form=form, seed=4) as r0:
        r0.init_particles()
        P, g = r0.download()
    g = dict(q=3000, pos=(P[0]["x"], P[0]["y"], P[0]["z"]))
    with Run(cfg, form=form, seed=4) as r:
        r.upload(P, g)
        with pytest.raises(PotError) as e:
            r.step(140)  # ions are reinjected from step 135 (tss_ion = 135)
        assert e.value.status == -8  # POT_E_ITER
        assert e.value.stats["warn"] & 64
    with Run(cfg, form=form, seed=4, chi_cap=True) as r:
        r.upload(P, g)
        st = r.step(140)
        Pc, gc = r.download()
    assert st["status"] == 0 and st["t_steps"] == 140 and st["chi_b"] > 1.0
    assert st["warn"] & WARN_CHI_CAP
    R = cfg.r * cfg.mpp
    rr = np.sqrt((Pc["x"] - R) ** 2 + (Pc["y"] - R) ** 2 + (Pc["z"] - R) ** 2)
    assert np.all(np.isfinite(rr)) and rr.max() <= R * (1 + 1e-12)
