"""Shared helpers for the tests: configurations and oracle snapshots."""
from __future__ import annotations

import numpy as np

from oracle.oracle import Oracle, RunParams
from pot_b200.gpu import RunConfig

SMALL = dict(N=8193, r=1000, dt=3.37727e-15, mpp=7.08046e-10, soft=1.41609e-09, Te=11600.0, Ti=11600.0,
             x_drift=0.0, a=1.41609e-08, settle=0.0, theta=0.5)
# large grain, drift, magnetic field, theta 0.8: exercises absorption, SCEPTIC
# reinjection with flow, the Boris rotation and the self-inclusion of cells
STRESS = dict(N=4097, r=1000, dt=3.37727e-14, mpp=7.08046e-10, soft=1.41609e-09, Te=11600.0, Ti=1160.0,
              x_drift=3e4, a=1.5e-07, settle=0.0, theta=0.8, B=(0.3, 0.5, -0.2))


def params(d: dict, **over) -> RunParams:
    d = dict(d)
    d.update(over)
    return RunParams(**d)


def run_config(d: dict, sceptic=True, **over) -> RunConfig:
    d = dict(d)
    d.update(over)
    return RunConfig(sceptic=sceptic, **d)


def oracle_snapshot(d: dict, seed=1, mode="gpu", steps=0, sceptic=True, **over):
    """An oracle run initialised with `seed` and advanced `steps` steps."""
    o = Oracle(params(d, **over), mode=mode, sceptic=sceptic, seed=seed)
    if steps:
        o.run_steps(steps)
    return o


def canonical_dump(d: dict):
    ints = sorted(zip(d["int_level"].tolist(), d["int_path"].tolist()))
    leaves = sorted(zip(d["leaf_part"].tolist(), d["leaf_level"].tolist(), d["leaf_path"].tolist()))
    return ints, leaves


def by_cell(d: dict):
    """Map (level, path) -> (q, aq, cx, cy, cz, w) for internal cells."""
    out = {}
    for i in range(len(d["int_level"])):
        out[(int(d["int_level"][i]), int(d["int_path"][i]))] = (
            int(d["int_q"][i]), int(d["int_aq"][i]), float(d["int_c"][i, 0]), float(d["int_c"][i, 1]),
            float(d["int_c"][i, 2]), float(d["int_w"][i]))
    return out


def ld(hi, lo):
    """double-double -> float128-ish numpy longdouble."""
    return np.asarray(hi, np.longdouble) + np.asarray(lo, np.longdouble)
