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
* ``4m``     the spheroidal-grain program (pot-spheroid.c, PROLATE):
  4,000,001 particles, a prolate spheroid of semi-axes 0.3 / 0.1 / 0.1
  lambda (-a 7.21387e-07 -A 3: a is the volume-equivalent radius, the
  semi-axes a A^(2/3) and a A^(-1/3)) with its axis along the flow axis x,
  as the reference program has it (pot-spheroid.c:1689-1779, 2448-2537),
  Te/Ti = 10, Mach 0.5 drift, B = 0.9533 T along z (electron gyroradius
  sqrt(k Te / m_e) / omega_ce = 0.5 lambda), domain 12 lambda, theta 0.4,
  20,000 steps, seed 3.
* ``4m_tilt`` the same plasma with the spheroid tilted 30 degrees from the
  flow axis x towards y.  The reference cannot tilt its grain, so this one
  runs on the GPU only.

Keys beyond the run's flags: ``steps`` (run length), ``leaf_size`` (fast
form), ``seed`` and ``variant`` (the reference program that realises it:
pot.c with SCEPTIC reinjection, or pot-spheroid.c's prolate program).
"""
from __future__ import annotations

from .gpu import RunConfig

CONFIGS = {
    "small": dict(N=8193, r=1000, mpp=7.08046e-10, a=1.41609e-08, soft=1.41609e-09, dt=3.37727e-15,
                  Te=11600.0, Ti=11600.0, x_drift=0.0, settle=0.0, theta=0.5, steps=2000, leaf_size=8),
    "1m": dict(N=1000001, r=1000, mpp=2.16079e-08, a=4.32157e-07, soft=2.16079e-08, dt=2.57665e-14,
               Te=11600.0, Ti=1160.0, x_drift=9785.26, settle=0.0, theta=0.5, steps=10000, leaf_size=16),
    "4m": dict(N=4000001, r=1000, mpp=6.00218e-08, a=7.21387e-07, A=3.0, soft=5.00182e-08, dt=5.96447e-14,
               Te=11600.0, Ti=1160.0, x_drift=4892.63, settle=0.0, theta=0.4, B=(0.0, 0.0, 0.9533),
               steps=20000, leaf_size=16, group_size=64, seed=3, variant="prolate_sceptic"),
}
CONFIGS["4m_tilt"] = dict(CONFIGS["4m"], axis=(0.8660254037844387, 0.5, 0.0))

EXTRA_KEYS = ("steps", "leaf_size", "group_size", "seed", "variant")


def run_params(name: str, N: int | None = None, untilted: bool = False) -> dict:
    """The run's flags only (RunParams / RunConfig keywords); ``untilted``
    puts a spheroid's axis back on x, as the reference has it."""
    c = {k: v for k, v in CONFIGS[name].items() if k not in EXTRA_KEYS}
    if N is not None:
        c["N"] = int(N)
    if untilted and "axis" in c:
        c["axis"] = (1.0, 0.0, 0.0)
    return c


def variant(name: str) -> str:
    return CONFIGS[name].get("variant", "sceptic")


def run_config(name: str, N: int | None = None, **over) -> RunConfig:
    c = run_params(name, N)
    c.update(over)
    return RunConfig(**c)


def flags(name: str) -> str:
    """The reference command line for a configuration."""
    c = CONFIGS[name]
    s = ("-N %d -r %d -m %g -a %g -s %g -d %g -E %g -I %g -x %g -e %g -i %d"
         % (c["N"], c["r"], c["mpp"], c["a"], c["soft"], c["dt"], c["Te"], c["Ti"], c["x_drift"],
            c["settle"], c["steps"]))
    if c.get("A"):
        s += " -A %g" % c["A"]
    return s
