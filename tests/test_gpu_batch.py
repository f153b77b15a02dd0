"""Batches of independent runs (pot_batch_*), the autotuner and the
serving program.  The bar: a run's state after k steps in a batch -- with
other runs admitted and evicted around it, one CUDA-graph launch stepping
them all -- is bit-identical to the same run stepped alone."""
import json
import os
import subprocess

import numpy as np
import pytest

from pot_b200.gpu import Batch, Run, RunConfig, bytes_needed, tune

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SERVE = os.path.join(ROOT, "pot_b200", "potserve")


def job(N, a_rel=0.2, ratio=10.0, mach=1.0, B=0.0, A=0.0):
    """A run of the batched configurations' family (domain 8 Debye lengths)."""
    kb, eps0, qe, me = 1.38065e-23, 8.85419e-12, 1.6021766e-19, 9.109383e-31
    Te = 11600.0
    lam = 3.0 * (N - 1) * qe * qe / (4096.0 * 3.14159265358979 * eps0 * kb * Te)
    R = 8.0 * lam
    n = (N - 1) / (4.0 / 3.0 * 3.14159265358979 * R ** 3)
    wpe = np.sqrt(n / 2 * qe * qe / (eps0 * me))
    return RunConfig(N=N, r=1000, mpp=R / 1000, a=a_rel * lam, soft=0.01 * lam, dt=0.005 / wpe, Te=Te, Ti=Te / ratio,
                     x_drift=mach * np.sqrt(kb * Te / (1836.15 * me)), theta=0.5, B=(0.0, 0.0, B), A=A)


def test_bytes_needed_grows_with_n():
    a, b = bytes_needed(job(20001)), bytes_needed(job(200001))
    assert 0 < a < b
    assert bytes_needed(job(20001), form="plain") > a


@pytest.mark.gpu
@pytest.mark.parametrize("pack", [True, False])
def test_batch_matches_runs_alone(pack):
    cfgs = [job(12001, 0.3, 10, 1.0), job(30001, 0.05, 1, 0.0, B=0.4), job(20001, 0.5, 30, 2.0, A=3.0),
            job(16001, 0.1, 3, 0.5)]
    forms = ["fast", "fast", "plain", "fast"]
    seeds = [1001, 1002, 1003, 1004]
    with Batch(steps_per_launch=2, pack=pack) as b:
        s0 = b.admit(cfgs[0], forms[0], seed=seeds[0])
        s1 = b.admit(cfgs[1], forms[1], seed=seeds[1])
        b.step(10)
        s2 = b.admit(cfgs[2], forms[2], seed=seeds[2])  # joins after 10 steps: re-capture
        b.step(6)
        b.evict(s1)                                     # leaves after 16 steps
        s3 = b.admit(cfgs[3], forms[3], seed=seeds[3])
        b.step(8)
        b.sync()
        rows = {int(r["slot"]): r for r in b.summary()}
        got = {k: b.download(s) for k, s in ((0, s0), (2, s2), (3, s3))}
    steps = {0: 24, 2: 14, 3: 8}
    for k, (P, g) in got.items():
        with Run(cfgs[k], form=forms[k], seed=seeds[k]) as r:
            r.init_particles()
            qs = []
            for _ in range(steps[k]):
                qs.append(r.step(1)["grain_q"])
            Pa, ga = r.download()
        assert np.array_equal(P.view(np.uint8), Pa.view(np.uint8)), k
        assert g["q"] == ga["q"] and g["t_steps"] == steps[k]
        row = rows[{0: s0, 2: s2, 3: s3}[k]]
        assert row["t_steps"] == steps[k] and row["grain_q"] == ga["q"]
        assert row["q_sum"] == sum(qs)
        assert row["particles"] == cfgs[k].N


@pytest.mark.gpu
def test_large_run_pre_order_groups_match_packed():
    """From 2,000,000 particles on, a run alone builds its target groups in
    tree pre-order (three launches); the packed batch builds the same groups
    in one launch, in whatever order their cells finish.  The groups are the
    same set, so four steps of a 2,000,001-particle run, alone and as the
    one member of a packed batch, leave the same particles bit for bit."""
    cfg = job(2000001, 0.3, 10, 1.0, B=0.3)
    with Batch(steps_per_launch=2, pack=True) as b:
        s = b.admit(cfg, "fast", seed=77)
        b.step(4)
        b.sync()
        P, g = b.download(s)
    with Run(cfg, form="fast", seed=77) as r:
        r.init_particles()
        st = r.step(4)
        Pa, ga = r.download()
    assert st["status"] == 0 and st["n_groups"] > 0
    assert np.array_equal(P.view(np.uint8), Pa.view(np.uint8))
    assert g["q"] == ga["q"] and g["t_steps"] == 4


@pytest.mark.gpu
def test_packed_batch_of_many_runs_matches_runs_alone():
    """Twelve fast-form runs of 8k-70k particles -- leaf sizes 8, 16 and 32,
    groups of 32 and 64 (two packed classes), a spheroidal grain, a
    magnetic field -- stepped 12 steps in packed launches, one run admitted
    after 4 steps and one evicted after 8: each run's particles and grain
    bit for bit as stepped alone."""
    rng = np.random.default_rng(5)
    specs = []
    for i in range(12):
        N = int(np.exp(rng.uniform(np.log(8001), np.log(70001)))) | 1
        cfg = job(N, float(np.exp(rng.uniform(np.log(0.05), np.log(0.8)))), [1, 3, 10, 30][i % 4],
                  float(rng.uniform(0, 2)), B=0.6 if i == 3 else 0.0, A=3.0 if i == 5 else 0.0)
        specs.append((cfg, [8, 16, 32][i % 3], 64 if i % 4 == 1 else 32, 2000 + i))
    with Batch(steps_per_launch=2) as b:
        slots = {i: b.admit(c, "fast", leaf_size=L, group_size=G, seed=sd) for i, (c, L, G, sd) in enumerate(specs)
                 if i != 11}
        b.step(4)
        slots[11] = b.admit(specs[11][0], "fast", leaf_size=specs[11][1], group_size=specs[11][2], seed=specs[11][3])
        b.step(4)
        b.evict(slots.pop(7))
        b.step(4)
        b.sync()
        got = {i: b.download(s) for i, s in slots.items()}
    for i, (P, g) in got.items():
        c, L, G, sd = specs[i]
        with Run(c, form="fast", leaf_size=L, group_size=G, seed=sd) as r:
            r.init_particles()
            r.step(8 if i == 11 else 12)
            Pa, ga = r.download()
        assert np.array_equal(P.view(np.uint8), Pa.view(np.uint8)), i
        assert g["q"] == ga["q"] and g["t_steps"] == ga["t_steps"], i


@pytest.mark.gpu
def test_batch_admission_respects_hbm_reserve():
    import torch
    free, total = torch.cuda.mem_get_info()
    with Batch(reserve_bytes=free - bytes_needed(job(30001)) // 2) as b:
        assert b.try_admit(job(30001)) is None  # would cut into the reserve
        assert b.count()["runs"] == 0
    with Batch() as b:
        assert b.try_admit(job(30001)) is not None


@pytest.mark.gpu
def test_autotuner_picks_a_candidate():
    t = tune(job(40001), steps=4)
    assert (t["leaf_size"], t["group_size"]) in {(8, 32), (16, 32), (32, 32), (16, 64), (32, 64)}
    assert t["ms_per_step"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("mode,extra", [("sweep", ["--runs", "6"]),
                                        ("serve", ["--rate", "40", "--duration", "0.2", "--bmax", "1.0"])])
def test_serving_program(mode, extra):
    from pot_b200 import build
    build.build_host()
    p = subprocess.run([SERVE, "--mode", mode, "--nmin", "8001", "--nmax", "30001", "--max-steps", "600",
                        "--plain-sample", "2", "--tune"] + extra, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr
    d = json.loads(p.stdout)
    assert d["finished"] == d["jobs"] > 0
    assert d["particle_steps_per_s"] > 0 and d["latency_s"]["p50"] > 0
    assert d["latency_s"]["p99"] >= d["latency_s"]["p50"]
    assert d["plain_one_at_a_time"]["jobs"] == 2
