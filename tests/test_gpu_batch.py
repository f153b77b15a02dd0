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
def test_batch_matches_runs_alone():
    cfgs = [job(12001, 0.3, 10, 1.0), job(30001, 0.05, 1, 0.0, B=0.4), job(20001, 0.5, 30, 2.0, A=3.0),
            job(16001, 0.1, 3, 0.5)]
    forms = ["fast", "fast", "plain", "fast"]
    seeds = [1001, 1002, 1003, 1004]
    with Batch(steps_per_launch=2) as b:
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
