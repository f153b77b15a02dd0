"""The oracle (C restatement) against golden vectors written by the reference.

tests/golden/make_golden.py ran the reference pot.c itself (compiled from its
own sources) on these seeded inputs; here the oracle must reproduce it bit for
bit: whole particle arrays after init and after 60 / 150 steps (digests), the
tree, x87 long-double fields, potentials, absorption decisions and the
SCEPTIC sampler's inverse CDFs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.oracle import PARTICLE_DTYPE, Oracle, RunParams

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(parts):
    p = parts.copy()
    p["_pad"] = 0
    return hashlib.sha256(p.tobytes()).hexdigest()


def runs():
    with open(os.path.join(GOLD, "runs.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def snap():
    return np.load(os.path.join(GOLD, "small_snapshot.npz"))


@pytest.mark.parametrize("key", ["sceptic_small", "sceptic_stress", "sphere_small", "sphere_stress"])
def test_oracle_reproduces_reference_runs(key):
    rec = runs()[key]
    p = dict(rec["params"])
    if "B" in p:
        p["B"] = tuple(p["B"])
    o = Oracle(RunParams(**p), mode="reference", sceptic=key.startswith("sceptic"), seed=rec["seed"])
    assert digest(o.particles()) == rec["init_sha256"]
    o.run_steps(rec["steps"])
    assert digest(o.particles()) == rec["final_sha256"]
    g = o.grain()
    for k, v in rec["final_grain"].items():
        assert g[k] == v, k


def _small_oracle():
    rec = runs()["sceptic_small"]
    o = Oracle(RunParams(**rec["params"]), mode="reference", sceptic=True, seed=rec["seed"])
    o.set_grain(q=-317)
    o.build_tree()
    return o


def test_tree_matches_reference(snap):
    o = _small_oracle()
    d = o.tree_dump()
    for k in ("int_level", "int_path", "int_q", "int_aq", "int_c", "int_w", "leaf_part", "leaf_level",
              "leaf_path"):
        assert np.array_equal(d[k], snap[k]), k


def test_fields_and_potentials_match_reference(snap):
    o = _small_oracle()
    hi, lo = o.field_many(snap["field_idx"], snap["field_xyz"])
    assert np.array_equal(hi, snap["field_hi"])
    assert np.array_equal(lo, snap["field_lo"])
    phi = np.array([o.phi_at(*p) for p in snap["phi_pts"]])
    assert np.array_equal(phi, snap["phi"])
    assert o.measure_chi_b() == snap["chi_b"][0]


def test_absorption_decisions_match_reference(snap):
    g = np.zeros(1, PARTICLE_DTYPE)
    g["x"], g["y"], g["z"] = snap["cross_grain"]
    a = float(snap["cross_a"][0])
    o = _small_oracle()
    res = np.array([o.cross_grain(p, d, g[0], a) for p, d in zip(snap["cross_pts"], snap["cross_dpos"])])
    assert np.array_equal(res.astype(np.int8), snap["cross_res"])
    assert 0 < res.sum() < len(res)


def test_sceptic_sampler_matches_reference(snap):
    L = Oracle.lib()
    for i, U in enumerate(snap["icdf_U"]):
        for j, c in enumerate(snap["icdf_chi"]):
            got = [L.pto_u_icdf(U, c, q) for q in snap["icdf_q"]]
            np.testing.assert_allclose(got, snap["icdf"][i, j], rtol=1e-14, atol=0)
    for j, c in enumerate(snap["icdf_chi"]):
        got = [L.pto_u_no_flow_icdf(c, q) for q in snap["icdf_q"]]
        np.testing.assert_allclose(got, snap["icdf_noflow"][j], rtol=1e-14, atol=0)
    for s, chi, u2, Rol, alpha in snap["alpha_cases"]:
        got = L.pto_integrate_for_alpha(s, chi, u2, Rol)
        if np.isnan(alpha):
            assert np.isnan(got)
        else:
            assert got == pytest.approx(alpha, rel=1e-13, abs=0)


# ---- spheroidal grain (pot-spheroid.c) -------------------------------------

def spheroid_runs():
    with open(os.path.join(GOLD, "spheroid.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def sph():
    return np.load(os.path.join(GOLD, "spheroid.npz"))


@pytest.mark.parametrize("key", ["prolate_sceptic", "prolate", "oblate_sceptic"])
def test_oracle_reproduces_spheroid_runs(key):
    rec = spheroid_runs()[key]
    p = dict(rec["params"])
    p["B"] = tuple(p["B"])
    o = Oracle(RunParams(**p), mode="reference", sceptic=key.endswith("_sceptic"), seed=rec["seed"])
    o.set_grain(q=rec["grain_q0"])
    assert digest(o.particles()) == rec["init_sha256"]
    for _ in range(rec["steps"]):
        o.step(compute_epe=True)
    assert digest(o.particles()) == rec["final_sha256"]
    g = o.grain()
    for k, v in rec["final_grain"].items():
        assert g[k] == v, k
    assert o.last_step_stats()["epe"].tolist() == rec["final_epe"]


def _spheroid_oracle():
    rec = spheroid_runs()["prolate_sceptic"]
    p = dict(rec["params"])
    p["B"] = tuple(p["B"])
    o = Oracle(RunParams(**p), mode="reference", sceptic=True, seed=21)
    o.set_grain(q=-250)
    o.build_tree()
    return o


def test_spheroid_tree_fields_potentials_match_reference(sph):
    o = _spheroid_oracle()
    assert digest(o.particles()) == str(sph["snapshot_sha256"][0])
    d = o.tree_dump()
    for k in ("int_level", "int_path", "int_q", "int_aq", "int_c", "int_w", "leaf_part", "leaf_level",
              "leaf_path"):
        assert np.array_equal(d[k], sph[k]), k
    assert 0 not in set(d["leaf_part"].tolist())
    hi, lo = o.field_many(sph["field_idx"], sph["field_xyz"])
    assert np.array_equal(hi, sph["field_hi"])
    assert np.array_equal(lo, sph["field_lo"])
    phi = np.array([o.phi_at(*p) for p in sph["phi_pts"]])
    assert np.array_equal(phi, sph["phi"])
    pp = np.array([o.phi_particle_feels(int(i)) for i in sph["field_idx"][:64]])
    assert np.array_equal(pp, sph["phi_part"][:, 0])
    assert o.measure_chi_b() == sph["chi_b"][0]


def test_spheroid_absorption_decisions_match_reference(sph):
    o = _spheroid_oracle()
    g = o.particles()[0:1]
    res = np.array([o.cross_grain_run(p, dp, g[0]) for p, dp in zip(sph["cross_pts"], sph["cross_dpos"])])
    assert np.array_equal(res.astype(np.int8), sph["cross_res"])
    assert 0 < res.sum() < len(res)
