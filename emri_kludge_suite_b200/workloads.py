"""Seeded synthetic workloads of the benchmark and of the profiling runs.

* :func:`config2` -- the same with e0 ~ U(0.05, 0.7) and n_max = min(100, ceil(10 / (1 - e0)^1.5)).
* :func:`config1` -- the 512-source batch: log10 M ~ U(5, 7), mu ~ U(1, 100),
  a ~ U(0, 0.95), e0 ~ U(0.05, 0.5), cos iota ~ U(-1, 1) (|cos iota| < 0.05
  redrawn: the flux kludge is singular for polar orbits), isotropic sky and
  spin directions, phases ~ U(0, 2 pi), D = 1 Gpc, T ~ U(0.1, 1) yr at
  dt = 10 s, and p0 set so that the plunge falls after T (leading-order
  time to plunge from p_end = 10 + 3 e0, clipped to [9, 80]).

The small profiling workloads that use these draws are ``bench.py --profile``.
"""
from __future__ import annotations

import math

import numpy as np

YEAR = 31558149.8
MSUN_SEC = 6.67259e-11 * 1.98892e30 / 299792458.0**3
NMODES = 30
DT = 10.0
SEED = 20261203


def draw_source(rng, e_max: float = 0.5) -> dict:
    while True:
        logM = rng.uniform(5.0, 7.0)
        mu = rng.uniform(1.0, 100.0)
        a = rng.uniform(0.0, 0.95)
        e0 = rng.uniform(0.05, e_max)
        cosi = rng.uniform(-1.0, 1.0)
        thS = math.acos(rng.uniform(-1.0, 1.0))
        phS = rng.uniform(0.0, 2 * math.pi)
        thK = math.acos(rng.uniform(-1.0, 1.0))
        phK = rng.uniform(0.0, 2 * math.pi)
        gam, psi, alp = (rng.uniform(0.0, 2 * math.pi) for _ in range(3))
        T = rng.uniform(0.1, 1.0)
        if abs(cosi) < 0.05:  # the flux kludge is singular for polar orbits
            continue
        M = 10.0**logM
        rr = (M * MSUN_SEC) ** 2 / (mu * MSUN_SEC)  # radiation-reaction time [s]
        n = int(T * YEAR / DT)
        p_end = 10.0 + 3.0 * e0  # above the LSO for every spin / inclination
        p0 = (p_end**4 + 2.0 * (256.0 / 5.0) * n * DT / rr) ** 0.25
        p0 = min(max(p0, 9.0), 80.0)
        return dict(backint=False, LISA=True, length=n, dt=DT, p=p0, T=T, f=2e-3, T_fit=1.0, mu=mu, M=M, s=a, e=e0,
                    iota=math.acos(cosi), gamma=gam, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK, phi_K=phK,
                    alpha=alp, D=1.0)


def config1(seed: int, nsrc: int = 512):
    rng = np.random.default_rng(seed)
    return [draw_source(rng) for _ in range(nsrc)], rng


def config2(seed: int, nsrc: int = 512):
    """The configuration-1 draw with e0 ~ U(0.05, 0.7) and the harmonic cutoff
    n_max = min(100, ceil(10 / (1 - e0)^1.5)); returns (sources, nmodes)."""
    rng = np.random.default_rng(seed)
    src = [draw_source(rng, e_max=0.7) for _ in range(nsrc)]
    return src, [min(100, math.ceil(10.0 / (1.0 - p["e"]) ** 1.5)) for p in src]
