"""Write the golden fixtures of tests/golden/ from the reference program.

Runs the reference pot.c itself -- compiled from its own sources by
oracle/build.py with a single-rank MPI stand-in -- on seeded inputs and
stores what the tests need to pin the oracle without the reference tree:
SHA-256 digests of whole particle arrays after init and after N steps
(bit-for-bit pins), the canonical tree of a small snapshot, sampled fields
as double-double pairs of the reference's long double accumulators, edge
potentials, absorption decisions on crafted segments, the inverse CDFs and
orbit integral of the SCEPTIC sampler on a grid.

The spheroid fixtures (spheroid.json, spheroid.npz) come from the
reference's pot-spheroid.c compiled the same way.

Usage (where the reference tree is present):
    python tests/golden/make_golden.py [--ref-root /path/to/reference] [--spheroid-only]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import build as obuild  # noqa: E402
from oracle.oracle import PARTICLE_DTYPE, RefLib, RunParams  # noqa: E402

SMALL = dict(N=8193, r=1000, dt=3.37727e-15, mpp=7.08046e-10, soft=1.41609e-09, Te=11600.0, Ti=11600.0,
             x_drift=0.0, a=1.41609e-08, settle=0.0, theta=0.5)
STRESS = dict(N=4097, r=1000, dt=3.37727e-14, mpp=7.08046e-10, soft=1.41609e-09, Te=11600.0, Ti=1160.0,
              x_drift=3e4, a=1.5e-07, settle=0.0, theta=0.8, B=(0.3, 0.5, -0.2))


def digest(parts: np.ndarray) -> str:
    p = parts.copy()
    p["_pad"] = 0
    return hashlib.sha256(p.tobytes()).hexdigest()


def grain_json(g: dict) -> dict:
    return {k: (float(v) if isinstance(v, float) else int(v)) for k, v in g.items()}


def runs(ref_root: str) -> dict:
    obuild.build_ref(ref_root)
    out = {}
    for variant in ("sceptic", "sphere"):
        for name, d, seed, steps in (("small", SMALL, 1, 60), ("stress", STRESS, 7, 150)):
            ref = RefLib(variant, build=False).setup(RunParams(**d), seed=seed)
            rec = {"params": d, "seed": seed, "init_sha256": digest(ref.particles())}
            ref.run_steps(steps)
            rec["steps"] = steps
            rec["final_sha256"] = digest(ref.particles())
            rec["final_grain"] = grain_json(ref.grain())
            P = ref.particles()
            rec["final_head"] = {k: P[k][:4].tolist() for k in ("x", "y", "z", "vx", "vy", "vz", "species")}
            out["%s_%s" % (variant, name)] = rec
    return out


def tree_and_fields(ref_root: str):
    """Canonical tree, fields and potentials on the small config's initial
    snapshot with a charged grain (q = -317)."""
    ref = RefLib("sceptic", build=False).setup(RunParams(**SMALL), seed=1)
    ref.set_grain(q=-317)
    ref.build_tree()
    t = ref.tree_dump()
    P = ref.particles()
    rng = np.random.default_rng(1234)
    idx = np.concatenate([[0], rng.choice(np.arange(1, SMALL["N"]), 255, replace=False)]).astype(np.uint32)
    xyz = np.stack([P["x"][idx], P["y"][idx], P["z"][idx]], 1) + rng.normal(0, 1e-9, (len(idx), 3))
    hi, lo = ref.field_many(idx, xyz)
    R = SMALL["r"] * SMALL["mpp"]
    pts = R + rng.uniform(-0.95 * R, 0.95 * R, (32, 3))
    phi = np.array([ref.phi_at(*p) for p in pts])
    chi_b = ref.measure_chi_b()
    arrays = dict(int_level=t["int_level"], int_path=t["int_path"], int_q=t["int_q"], int_aq=t["int_aq"],
                  int_c=t["int_c"], int_w=t["int_w"], leaf_part=t["leaf_part"], leaf_level=t["leaf_level"],
                  leaf_path=t["leaf_path"], field_idx=idx, field_xyz=xyz, field_hi=hi, field_lo=lo,
                  phi_pts=pts, phi=phi, chi_b=np.array([chi_b]))
    return arrays


def absorption_cases(ref_root: str):
    """does_particle_cross_grain (pot.c:2287-2325) on crafted segments."""
    ref = RefLib("sceptic", build=False).setup(RunParams(**SMALL), seed=1, init=False)
    rng = np.random.default_rng(99)
    a = 1.41609e-08
    g = np.zeros(1, PARTICLE_DTYPE)
    g["x"] = g["y"] = g["z"] = 7.08046e-07
    n = 4000
    pts = np.zeros(n, PARTICLE_DTYPE)
    dpos = np.zeros((n, 3))
    res = np.zeros(n, np.int8)
    for k in range(n):
        # end points within a few grain radii, steps of comparable length,
        # some exactly on the sphere and some tangent
        c = rng.normal(0, 1.5 * a, 3)
        if k % 7 == 0:
            c = c / np.linalg.norm(c) * a
        pts[k]["x"], pts[k]["y"], pts[k]["z"] = g["x"][0] + c[0], g["y"][0] + c[1], g["z"][0] + c[2]
        dpos[k] = rng.normal(0, 2 * a, 3)
        res[k] = ref.cross_grain(pts[k], dpos[k], g[0], a)
    return dict(cross_pts=pts, cross_dpos=dpos, cross_res=res, cross_a=np.array([a]),
                cross_grain=np.array([g["x"][0], g["y"][0], g["z"][0]]))


def sampler_grid(ref_root: str):
    ref = RefLib("sceptic", build=False).setup(RunParams(**SMALL), seed=1, init=False)
    L = ref.lib
    qs = np.linspace(0.02, 0.98, 17)
    Us = np.array([0.05, 0.5, 1.0, 2.0, 3.0])
    chis = np.array([-3.0, -0.5, 0.0, 0.3])
    icdf = np.array([[[L.potref_u_icdf(U, c, q) for q in qs] for c in chis] for U in Us])
    nf = np.array([[L.potref_u_no_flow_icdf(c, q) for q in qs] for c in chis])
    rng = np.random.default_rng(5)
    ia = []
    for _ in range(64):
        u2 = rng.uniform(0.5, 6.0)
        chi = rng.uniform(-3.0, 0.4)
        s = np.sqrt(rng.uniform(0, max(1e-9, 1 - chi / u2)))
        Rol = rng.uniform(0.5, 6.0)
        ia.append((s, chi, u2, Rol, L.potref_integrate_for_alpha(s, chi, u2, Rol)))
    return dict(icdf_q=qs, icdf_U=Us, icdf_chi=chis, icdf=icdf, icdf_noflow=nf, alpha_cases=np.array(ia))


SPHEROID = dict(STRESS, a=3.0e-7)
SPHEROID_RUNS = (("prolate_sceptic", 3.0, 11, 120), ("prolate", 5.0, 12, 80),
                 ("oblate_sceptic", 0.4, 13, 120))


def spheroid(ref_root: str):
    """pot-spheroid.c (PROLATE / OBLATE programs): run digests with a
    charged grain, and for prolate A = 3 the grain-free tree, fields,
    potentials and absorption decisions on one snapshot."""
    obuild.build_ref(ref_root, variants=obuild.SPHEROID_VARIANTS)
    meta = {}
    for variant, A, seed, steps in SPHEROID_RUNS:
        ref = RefLib(variant, build=False).setup(RunParams(**SPHEROID, A=A), seed=seed)
        ref.set_grain(q=-400)
        rec = {"variant": variant, "params": dict(SPHEROID, A=A), "seed": seed, "grain_q0": -400,
               "init_sha256": digest(ref.particles())}
        ref.run_steps(steps, compute_epe=True)
        rec["steps"] = steps
        rec["final_sha256"] = digest(ref.particles())
        rec["final_grain"] = grain_json(ref.grain())
        rec["final_epe"] = [float(v) for v in ref.epe()]
        meta[variant] = rec
    ref = RefLib("prolate_sceptic", build=False).setup(RunParams(**SPHEROID, A=3.0), seed=21)
    ref.set_grain(q=-250)
    ref.build_tree()
    t = ref.tree_dump()
    P = ref.particles()
    rng = np.random.default_rng(4321)
    idx = np.concatenate([[0], rng.choice(np.arange(1, SPHEROID["N"]), 255, replace=False)]).astype(np.uint32)
    xyz = np.stack([P["x"][idx], P["y"][idx], P["z"][idx]], 1) + rng.normal(0, 1e-9, (len(idx), 3))
    hi, lo = ref.field_many(idx, xyz)
    R = SPHEROID["r"] * SPHEROID["mpp"]
    pts = R + rng.uniform(-0.95 * R, 0.95 * R, (32, 3))
    phi = np.array([ref.phi_at(*p) for p in pts])
    pp = np.array([ref.phi_particle_feels(int(i)) for i in idx[:64]])
    chi_b = ref.measure_chi_b()
    a = SPHEROID["a"]
    a_ax = a * 3.0 ** (2.0 / 3.0)
    g = P[0:1].copy()
    n = 2000
    cpts = np.zeros(n, PARTICLE_DTYPE)
    cd = np.zeros((n, 3))
    cres = np.zeros(n, np.int8)
    for k in range(n):
        end = np.array([g["x"][0], g["y"][0], g["z"][0]]) + rng.uniform(-2.0, 2.0, 3) * a_ax
        cpts[k]["x"], cpts[k]["y"], cpts[k]["z"] = end
        cd[k] = rng.normal(0, a_ax, 3)
        cres[k] = ref.cross_grain(cpts[k], cd[k], g[0], a)
    arrays = dict(int_level=t["int_level"], int_path=t["int_path"], int_q=t["int_q"], int_aq=t["int_aq"],
                  int_c=t["int_c"], int_w=t["int_w"], leaf_part=t["leaf_part"], leaf_level=t["leaf_level"],
                  leaf_path=t["leaf_path"], field_idx=idx, field_xyz=xyz, field_hi=hi, field_lo=lo,
                  phi_pts=pts, phi=phi, phi_part=pp, chi_b=np.array([chi_b]), cross_pts=cpts, cross_dpos=cd,
                  cross_res=cres, snapshot_sha256=np.array([digest(P)]))
    return meta, arrays


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=obuild.DEFAULT_REF_ROOT)
    ap.add_argument("--spheroid-only", action="store_true", help="write only spheroid.json / spheroid.npz")
    a = ap.parse_args(argv)
    meta_s, arrays_s = spheroid(a.ref_root)
    with open(os.path.join(HERE, "spheroid.json"), "w") as f:
        json.dump(meta_s, f, indent=1, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "spheroid.npz"), **arrays_s)
    if a.spheroid_only:
        print("wrote spheroid.json, spheroid.npz")
        return
    meta = runs(a.ref_root)
    with open(os.path.join(HERE, "runs.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    arrays = {}
    arrays.update(tree_and_fields(a.ref_root))
    arrays.update(absorption_cases(a.ref_root))
    arrays.update(sampler_grid(a.ref_root))
    np.savez_compressed(os.path.join(HERE, "small_snapshot.npz"), **arrays)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
