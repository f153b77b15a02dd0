"""GPU parity for the reference's other compile-time variants: OUT_BOUNCE,
POIS_POS_COLLECTION, velocity Verlet, Euler-Richardson and DIPOLES.

The oracle restates each variant bit for bit (pinned against the reference
compiled with the switch on, tests/test_oracle_variants_live.py).  Here the
CUDA path against the oracle in GPU semantics from the same state, step by
step: tallies, Poisson counts and grain charge exact; positions within
1e-12 of the domain radius and velocities within 1e-9 (FP64 against the
reference's long double), the same bars as the Boris step."""
import numpy as np
import pytest

from common import SMALL, STRESS, ld, oracle_snapshot
from test_gpu_parity import gpu_from_oracle

pytestmark = pytest.mark.gpu


def _compare_step(d, o, form="plain", **kw):
    """One step on the GPU and in the oracle from the oracle's state."""
    with gpu_from_oracle(d, o, form=form, **kw) as r:
        st = r.step(1)
        Pg, gg = r.download()
    o.step()
    return st, Pg, gg, o.last_step_stats(), o.particles(), o.grain()


def _assert_close(d, st, Pg, gg, so, Po, go, extra=0):
    R = d["r"] * d["mpp"]
    assert st["status"] == 0
    assert (st["dq"], st["de"], st["n_absorbed"]) == (so["dq"], so["de"], so["n_absorbed"])
    assert gg["q"] == go["q"] and gg["tot_absor_e"] == go["tot_absor_e"]
    d_pos = np.abs(np.stack([Pg["x"] - Po["x"], Pg["y"] - Po["y"], Pg["z"] - Po["z"]], 1)).max(1)
    d_vel = np.abs(np.stack([Pg["vx"] - Po["vx"], Pg["vy"] - Po["vy"], Pg["vz"] - Po["vz"]], 1)).max(1)
    vmax = max(np.abs(Po["vx"]).max(), np.abs(Po["vy"]).max(), np.abs(Po["vz"]).max())
    bad = np.nonzero((d_pos >= 1e-12 * R) | (d_vel >= 1e-9 * vmax))[0]
    # at most the ulp-level boundary coin flips of the known deviation 2
    assert len(bad) <= so["n_absorbed"] + extra, (len(bad), so["n_absorbed"])


@pytest.mark.parametrize("integrator", [1, 2], ids=["verlet", "euler_richardson"])
@pytest.mark.parametrize("d", [STRESS, dict(SMALL, N=8193, theta=0.8)], ids=["stress", "small"])
def test_integrators_plain_step_by_step(integrator, d):
    d = dict(d, integrator=integrator)
    o = oracle_snapshot(d, seed=13, mode="gpu", steps=2)
    o.set_grain(q=-500)
    for _ in range(6):
        _assert_close(d, *_compare_step(d, o))


@pytest.mark.parametrize("d", [STRESS, dict(STRESS, a=3.0e-7, A=3.0)], ids=["sphere", "prolate"])
def test_bounce_plain_step_by_step(d):
    d = dict(d, bounce=0.95)
    o = oracle_snapshot(d, seed=17, mode="gpu", steps=2)
    o.set_grain(q=-400)
    bounced = 0
    for _ in range(8):
        st, Pg, gg, so, Po, go = _compare_step(d, o)
        _assert_close(d, st, Pg, gg, so, Po, go)
        assert st["n_reinjected"] == st["n_absorbed"]  # nothing reinjected at the wall
        # a particle reinjected onto the sphere may sit an ulp outside it in
        # one result and not the other (known deviation 2), moving inwards
        assert abs(st["n_wall"] - o.variant_stats()["n_wall"]) <= so["n_absorbed"]
        bounced += st["n_bounced"]
    assert bounced > 0
    R = d["r"] * d["mpp"]
    rr = np.sqrt((Pg["x"] - R) ** 2 + (Pg["y"] - R) ** 2 + (Pg["z"] - R) ** 2)
    assert rr.max() <= R * (1 + 1e-9) or st["n_wall"] > 0


def test_poisson_collection_plain_exact():
    """The grain's Poisson charge gain: the same Philox draw and inversion as
    the oracle, so the count is exact step by step, and absorbed ions add
    no charge."""
    d = dict(STRESS, pois_ions=True)
    o = oracle_snapshot(d, seed=19, mode="gpu", steps=2)
    o.set_grain(q=-300)
    total = 0
    for k in range(10):
        if k == 5:
            o.set_ion_temp(3.0 * d["Ti"])
        with gpu_from_oracle(d, o) as r:
            if k >= 5:
                r.set_ion_temp(3.0 * d["Ti"])
            st = r.step(1)
            Pg, gg = r.download()
        o.step()
        so, Po, go = o.last_step_stats(), o.particles(), o.grain()
        _assert_close(d, st, Pg, gg, so, Po, go)
        assert st["n_collected"] == o.variant_stats()["n_pois"]
        total += st["n_collected"]
    assert total > 0


def test_poisson_ion_temperature_from_macro():
    """pot_gpu_macro leaves the ions' measured temperature as the cached
    one (pot.c:3442-3448); uploads keep it."""
    d = dict(SMALL, N=20001, pois_ions=True)
    o = oracle_snapshot(d, seed=2, mode="gpu", steps=1)
    P = o.particles()
    ions = P[P["species"] == 1]
    v = np.stack([ions["vx"], ions["vy"], ions["vz"]], 1).astype(np.longdouble)
    T_ref = float(((v - v.mean(0)) ** 2).sum() * (1836.15 * 9.109383e-31 / (3.0 * 1.38065e-23)) / len(ions))
    with gpu_from_oracle(d, o) as r:
        assert r.ion_temp() == d["Ti"]
        r.macro()
        T = r.ion_temp()
        r.upload(P, None)
        assert r.ion_temp() == T
    assert abs(T - T_ref) <= 1e-9 * T_ref


def test_dipoles_plain_fields_potentials_and_steps():
    d = dict(SMALL, N=8193, dipoles=True)
    o = oracle_snapshot(d, seed=23, mode="gpu", steps=2)
    o.set_grain(q=-350)
    o.build_tree()
    rng = np.random.default_rng(5)
    P = o.particles()
    idx = rng.choice(np.arange(1, d["N"]), 512, replace=False).astype(np.uint32)
    xyz = np.stack([P["x"][idx], P["y"][idx], P["z"][idx]], 1) * (1 + 1e-7 * rng.normal(size=(len(idx), 3)))
    hi, lo = o.field_many(idx, xyz)
    E_ref = ld(hi, lo).astype(np.float64)
    R = d["r"] * d["mpp"]
    pts = R + rng.uniform(-0.9 * R, 0.9 * R, size=(64, 3))
    phi_ref = np.array([o.phi_at(*p) for p in pts])
    with gpu_from_oracle(d, o) as r:
        r.build_tree()
        E = r.field_at(idx, xyz)
        phi = r.phi_at(pts)
    mag = np.sqrt((E_ref ** 2).sum(1))
    assert (np.abs(E - E_ref).max(1) / mag).max() < 1e-12
    assert np.max(np.abs(phi - phi_ref) / np.abs(phi_ref).max()) < 1e-12
    for _ in range(4):
        _assert_close(d, *_compare_step(d, o))
    with gpu_from_oracle(d, o) as r:
        st = r.step(1, epe=True)
    o.step(compute_epe=True)
    ref = o.last_step_stats()["epe"]
    assert np.all(np.abs(st["epe"] - ref) <= 1e-10 * np.abs(ref).max())


@pytest.mark.parametrize("variant", [dict(integrator=1), dict(integrator=2), dict(bounce=0.9),
                                     dict(pois_ions=True)], ids=["verlet", "er", "bounce", "pois"])
@pytest.mark.parametrize("group", [32, 64])
def test_fast_form_variants_run(variant, group):
    """The fast form with each variant: steps run, charge is conserved
    (grain charge = start + absorbed + collected) and no particle is left
    outside the domain unless the wall reported it."""
    d = dict(SMALL, N=20001, **variant)
    o = oracle_snapshot(d, seed=29, mode="gpu", steps=1)
    o.set_grain(q=-400)
    R = d["r"] * d["mpp"]
    with gpu_from_oracle(d, o, form="fast", leaf_size=16, group_size=group) as r:
        q0 = r.download()[1]["q"]
        tot = 0
        wall = 0
        for _ in range(12):
            st = r.step(1)
            assert st["status"] == 0
            tot += st["dq"] + st["n_collected"]
            wall += st["n_wall"]
        Pg, gg = r.download()
    assert gg["q"] == q0 + tot
    rr = np.sqrt((Pg["x"] - R) ** 2 + (Pg["y"] - R) ** 2 + (Pg["z"] - R) ** 2)
    assert rr.max() <= R * (1 + 1e-9) or wall > 0


@pytest.mark.parametrize("integrator", [1, 2], ids=["verlet", "euler_richardson"])
def test_fast_integrator_field_matches_plain(integrator):
    """One non-Boris step in the fast form against the plain form from the
    same state: the velocity change (dt times the mean of the two field
    evaluations' accelerations) agrees to the fast walk's field error."""
    d = dict(SMALL, N=30001, integrator=integrator)
    o = oracle_snapshot(d, seed=31, mode="gpu", steps=1)
    o.set_grain(q=-300)
    P0 = o.particles()
    out = {}
    for form, kw in (("plain", {}), ("fast", dict(leaf_size=16))):
        with gpu_from_oracle(d, o, form=form, **kw) as r:
            r.step(1)
            out[form] = r.download()[0]
    e = np.nonzero((P0["species"] == 2) & (np.abs(out["plain"]["x"] - P0["x"]) < 1e-3 * d["r"] * d["mpp"])
                   & (np.abs(out["fast"]["x"] - P0["x"]) < 1e-3 * d["r"] * d["mpp"]))[0]
    dv = {f: np.stack([out[f]["vx"] - P0["vx"], out[f]["vy"] - P0["vy"], out[f]["vz"] - P0["vz"]], 1)[e]
          for f in out}
    rel = np.sqrt(((dv["fast"] - dv["plain"]) ** 2).sum(1) / (dv["plain"] ** 2).sum(1))
    assert np.sqrt(np.mean(rel ** 2)) < 0.4


def _direct_rms(o, idx, xyz, E):
    hi, lo = o.field_direct_many(idx, xyz, soften_all=True)
    E_dir = ld(hi, lo).astype(np.float64)
    return float(np.sqrt(np.mean(((E - E_dir) ** 2).sum(1) / (E_dir ** 2).sum(1))))


@pytest.mark.parametrize("leaf", [1, 16])
def test_fast_dipoles_field_and_potential(leaf):
    """DIPOLES in the fast form: cell dipoles from prefix sums of q x, the
    dipole term in the FP32 walk.  Against an FP64 direct sum the field is
    more accurate than the same form's monopole field, and the edge
    potential and potential energies agree with the plain form's dipole
    results (FP64, the reference's arithmetic) to the FP32 walk's error."""
    d = dict(SMALL, N=30001)
    o = oracle_snapshot(d, seed=33, mode="gpu", steps=1)
    o.set_grain(q=-300)
    rng = np.random.default_rng(8)
    P = o.particles()
    idx = np.sort(rng.choice(np.arange(1, d["N"]), 2048, replace=False)).astype(np.uint32)
    xyz = np.stack([P["x"][idx], P["y"][idx], P["z"][idx]], 1)
    out = {}
    for dip in (False, True):
        dd = dict(d, dipoles=dip)
        with gpu_from_oracle(dd, o, form="fast", leaf_size=leaf, group_size=32) as r:
            r.build_tree()
            out[dip] = r.field_at(idx, xyz)
    err_mono, err_dip = _direct_rms(o, idx, xyz, out[False]), _direct_rms(o, idx, xyz, out[True])
    assert err_dip < 0.8 * err_mono, (err_dip, err_mono)
    dd = dict(d, dipoles=True)
    res = {}
    for form, kw in (("plain", {}), ("fast", dict(leaf_size=leaf, group_size=32))):
        with gpu_from_oracle(dd, o, form=form, **kw) as r:
            st = r.step(1, epe=True)
            res[form] = st
    assert res["fast"]["status"] == 0
    # the edge potential: the fast form's FP64 walk over its own (bucket-leaf) tree
    assert abs(res["fast"]["chi_b"] - res["plain"]["chi_b"]) <= 0.05 * abs(res["plain"]["chi_b"])
    ep, ef = res["plain"]["epe"], res["fast"]["epe"]
    assert np.all(np.abs(ef - ep) <= 0.1 * np.abs(ep).max()), (ef, ep)


def test_fast_dipoles_run_and_limits():
    """A fast-form run with dipoles steps and conserves charge; groups of 64
    (two targets per lane) are refused with dipoles."""
    from pot_b200.gpu import PotError, Run
    from common import run_config
    d = dict(SMALL, N=20001, dipoles=True)
    o = oracle_snapshot(d, seed=35, mode="gpu", steps=1)
    o.set_grain(q=-400)
    with gpu_from_oracle(d, o, form="fast", leaf_size=16, group_size=32) as r:
        q0 = r.download()[1]["q"]
        tot = 0
        for _ in range(10):
            st = r.step(1)
            assert st["status"] == 0
            tot += st["dq"]
        assert r.download()[1]["q"] == q0 + tot
    with pytest.raises(PotError):
        Run(run_config(d), form="fast", leaf_size=16, group_size=64)
