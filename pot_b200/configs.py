"""Synthetic plasma configurations, in the reference's SI flag units.

Each entry is the reference command line (pot.c:4557-4850 flags) that
realises one benchmark plasma; Te = 11,600 K so that the Debye length
lambda = sqrt(eps0 k Te / ((n / 2) e^2)) (pot.c:3666) is fixed by N and the
domain radius R = r * mpp.

* ``small``  8,193 particles (grain + 4,096 ions + 4,096 electrons), grain
  radius 0.1 lambda, domain 5 lambda, Te = Ti, no flow, no field, softening
  0.01 lambda, dt = 0.01 / omega_pe, 2,000 steps, theta 0.5.
* ``1m``     1,000,001 particles (500,000 ions, 500,000 electrons), grain
  0.2 lambda, domain 10 lambda, Te/Ti = 10, ions drifting at Mach 1 (the ion
  sound speed sqrt(k Te / m_i)) along the reference's flow axis x,
  dt = 0.005 / omega_pe, 10,000 steps, theta 0.5, leaf size 16.
"""
from __future__ import annotations

from .gpu import RunConfig

CONFIGS = {
    "small": dict(N=8193, r=1000, mpp=7.08046e-10, a=1.41609e-08, soft=1.41609e-09, dt=3.37727e-15,
                  Te=11600.0, Ti=11600.0, x_drift=0.0, settle=0.0, theta=0.5, steps=2000, leaf_size=8),
    "1m": dict(N=1000001, r=1000, mpp=2.16079e-08, a=4.32157e-07, soft=2.16079e-08, dt=2.57665e-14,
               Te=11600.0, Ti=1160.0, x_drift=9785.26, settle=0.0, theta=0.5, steps=10000, leaf_size=16),
}


def run_config(name: str, N: int | None = None, **over) -> RunConfig:
    c = dict(CONFIGS[name])
    c.pop("steps")
    c.pop("leaf_size")
    c.pop("group_size", None)
    if N is not None:
        c["N"] = int(N)
    c.update(over)
    return RunConfig(**c)


def flags(name: str) -> str:
    """The reference command line for a configuration."""
    c = CONFIGS[name]
    return ("-N %d -r %d -m %g -a %g -s %g -d %g -E %g -I %g -x %g -e %g -i %d"
            % (c["N"], c["r"], c["mpp"], c["a"], c["soft"], c["dt"], c["Te"], c["Ti"], c["x_drift"],
               c["settle"], c["steps"]))
