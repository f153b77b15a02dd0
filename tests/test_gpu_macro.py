"""On-device macroscopic-summary sums (pot.c:3261-3508) against the same
two passes over the downloaded particles in long double, and the host
program's rows from either path."""
import os
import subprocess

import numpy as np
import pytest

from common import STRESS, run_config
from pot_b200.gpu import Run

pytestmark = pytest.mark.gpu


def host_sums(P, me, mi, cent):
    ld = np.longdouble
    Q = P[1:]
    v = np.sqrt(Q["vx"].astype(ld) ** 2 + Q["vy"].astype(ld) ** 2 + Q["vz"].astype(ld) ** 2)
    e = Q["species"] == 2
    i = ~e
    rx, ry, rz = Q["x"] - cent, Q["y"] - cent, Q["z"] - cent
    am = np.stack([ry * Q["vz"] - rz * Q["vy"], -(rx * Q["vz"] - rz * Q["vx"]), rx * Q["vy"] - ry * Q["vx"]], 1)
    vel = np.stack([Q["vx"], Q["vy"], Q["vz"]], 1).astype(ld)
    K = 0.5 * np.where(e, ld(me), ld(mi)) * v * v
    out = dict(n_e=e.sum(), n_i=i.sum(), K_e=K[e].sum(), s_e=v[e].sum(), s_i=v[i].sum(), v_e=vel[e].sum(0),
               v_i=vel[i].sum(0), am_e=am[e].astype(ld).sum(0), am_i=am[i].astype(ld).sum(0))
    Km, sme, smi = out["K_e"] / out["n_e"], out["s_e"] / out["n_e"], out["s_i"] / out["n_i"]
    ve, vi = out["v_e"] / out["n_e"], out["v_i"] / out["n_i"]
    out.update(sumsq_K_e=(K[e] ** 2).sum(), sum_x_e=Q["x"][e].astype(ld).sum(),
               sumsq_x_e=(Q["x"][e].astype(ld) ** 2).sum(),
               K_e_c=np.array([((K[e] - Km) ** k).sum() for k in (2, 3, 4)]),
               s_e_c=np.array([((v[e] - sme) ** k).sum() for k in (2, 3, 4)]),
               T_e=((vel[e] - ve) ** 2).sum(), sum_K_i=K[i].sum(), sumsq_K_i=(K[i] ** 2).sum(),
               s_i_c=np.array([((v[i] - smi) ** k).sum() for k in (2, 3, 4)]), T_i=((vel[i] - vi) ** 2).sum())
    return out


@pytest.mark.parametrize("form,A", [("fast", 0.0), ("plain", 3.0)])
def test_macro_sums_match_long_double(form, A):
    d = dict(STRESS, N=20001, a=3e-7, A=A)
    with Run(run_config(d), form=form, seed=3) as r:
        r.init_particles()
        r.step(7)
        m = r.macro()
        P, g = r.download()
        g2 = r.grain()
    me = 9.109383e-31
    mi = (1836.153 if A else 1836.15) * me
    h = host_sums(P, me, mi, d["r"] * d["mpp"])
    for k, v in h.items():
        got = np.asarray(m[k], dtype=np.float64)
        ref = np.asarray(v, dtype=np.longdouble)
        # odd central moments cancel: compare against the sum of magnitudes' scale
        scale = np.maximum(np.abs(ref).astype(np.float64), 1e-300)
        if k in ("K_e_c", "s_e_c", "s_i_c"):
            scale = np.maximum(scale, np.abs(ref).max().astype(np.float64))
        assert np.all(np.abs(got - ref.astype(np.float64)) <= 1e-11 * scale), (k, got, ref)
    assert g2["q"] == g["q"] and g2["t_steps"] == g["t_steps"] == 7


def test_host_program_rows_agree_between_paths(tmp_path):
    from pot_b200 import build
    exe = build.build_host()
    flags = ["-N", "8193", "-r", "1000", "-m", "7.08046e-10", "-a", "1.41609e-08", "-s", "1.41609e-09", "-d",
             "3.37727e-15", "-E", "11600", "-I", "11600", "-x", "0", "-e", "0", "-i", "30", "--seed", "9"]
    rows = {}
    for name, extra in (("device", []), ("host", ["--host-macro"])):
        out = tmp_path / name
        out.mkdir()
        p = subprocess.run([exe] + flags + extra + ["--output-dir", str(out)], capture_output=True, text=True,
                           timeout=300)
        assert p.returncode == 0, p.stderr
        rows[name] = [r.split() for r in (out / "pot-macroscopic.dat").read_text().splitlines()[1:]]
    assert len(rows["device"]) == len(rows["host"]) == 30
    A = np.array([[float(x) for x in r] for r in rows["device"]])
    B = np.array([[float(x) for x in r] for r in rows["host"]])
    assert np.array_equal(A[:, 9], B[:, 9]) and np.array_equal(A[:, 34], B[:, 34])  # grain charge, absorbed
    # printed to 6-7 significant digits, and means of velocities or moments of
    # skewness cancel: compare each column against its own scale
    scale = np.abs(B).max(0)
    assert np.all(np.abs(A - B) <= 1e-5 * scale + 1e-300), np.abs(A - B).max(0) / (scale + 1e-300)


def test_grain_charging_fast_matches_plain():
    """The FP32-walk fast form charges the grain like the plain FP64 form:
    over four seeds, the grain charge averaged over steps 1001-3000 (from the
    device-side charge sums) agrees within three standard errors of the
    seed-to-seed spread, or 1 %."""
    from pot_b200.configs import run_config as cfg_of
    cfg = cfg_of("1m", N=20001)
    means = {}
    for form in ("fast", "plain"):
        vals = []
        for seed in (11, 12, 13, 14):
            with Run(cfg, form=form, seed=seed) as r:
                r.init_particles()
                a = r.step(1000)["q_sum"]
                b = r.step(2000)["q_sum"]
            vals.append((b - a) / 2000.0)
        means[form] = np.array(vals)
    f, p = means["fast"], means["plain"]
    assert np.all(f < 0) and np.all(p < 0)
    se = np.sqrt(f.var(ddof=1) / len(f) + p.var(ddof=1) / len(p))
    assert abs(f.mean() - p.mean()) <= max(3 * se, 0.01 * abs(p.mean())), (f, p)


def _charging_config(N):
    """A plasma that charges its grain to near equilibrium in 20,000 steps:
    the serving jobs' recipe (domain 8 Debye lengths, dt = 0.005 / omega_pe,
    softening 0.01 lambda) with a grain of one Debye length, Te = Ti, no drift."""
    import math
    from pot_b200.gpu import RunConfig
    KB, EPS0, QE, ME = 1.38065e-23, 8.85419e-12, 1.6021766e-19, 9.109383e-31
    Te = 11600.0
    lam = 3.0 * (N - 1) * QE * QE / (4096.0 * math.pi * EPS0 * KB * Te)
    R = 8.0 * lam
    n_tot = (N - 1) / ((4.0 / 3.0) * math.pi * R ** 3)
    w_pe = math.sqrt((n_tot / 2.0) * QE * QE / (EPS0 * ME))
    return RunConfig(N=N, r=1000, dt=0.005 / w_pe, mpp=R / 1000.0, soft=0.01 * lam, Te=Te, Ti=Te, x_drift=0.0,
                     a=lam, settle=0.0, theta=0.5)


def test_late_grain_charge_fast_matches_plain():
    """Grain charge late in the charging, where it rises by under 1 % per
    thousand steps: the mean over steps 14,001-20,000 of four seeds per form
    agrees between the fast and plain forms within 1 % or three standard
    errors of the difference (the seed-to-seed spread is about 1 %)."""
    cfg = _charging_config(60001)
    means = {}
    for form in ("fast", "plain"):
        vals = []
        for seed in (1, 2, 3, 4):
            with Run(cfg, form=form, leaf_size=16 if form == "fast" else 0, seed=seed) as r:
                r.init_particles()
                a = r.step(14000)["q_sum"]
                b = r.step(6000)["q_sum"]
            vals.append((b - a) / 6000.0)
        means[form] = np.array(vals)
    f, p = means["fast"], means["plain"]
    assert np.all(f < -100) and np.all(p < -100)  # the grain did charge
    se = np.sqrt(f.var(ddof=1) / len(f) + p.var(ddof=1) / len(p))
    assert abs(f.mean() - p.mean()) <= max(3 * se, 0.01 * abs(p.mean())), (f, p)
