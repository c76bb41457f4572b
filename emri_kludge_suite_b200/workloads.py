"""Seeded synthetic workloads of the benchmark and of the profiling runs.

* :func:`config2` -- the same with e0 ~ U(0.05, 0.7) and n_max = min(100, ceil(10 / (1 - e0)^1.5)).
* :func:`config1` -- the 512-source batch: log10 M ~ U(5, 7), mu ~ U(1, 100),
  a ~ U(0, 0.95), e0 ~ U(0.05, 0.5), cos iota ~ U(-1, 1) (|cos iota| < 0.05
  redrawn: the flux kludge is singular for polar orbits), isotropic sky and
  spin directions, phases ~ U(0, 2 pi), D = 1 Gpc, T ~ U(0.1, 1) yr at
  dt = 10 s, and p0 set so that the plunge falls after T (leading-order
  time to plunge from p_end = 10 + 3 e0, clipped to [9, 80]).

Profiling workloads (run from the repository root on one GPU)::

    python -m emri_kludge_suite_b200.workloads waveform   # 16 of the 512 sources, FP64 and split, twice each
    python -m emri_kludge_suite_b200.workloads phase      # the phase product of the same 16 sources, twice
    python -m emri_kludge_suite_b200.workloads fisher     # two 14-parameter Fisher matrices, 28 x 3.2e6-sample templates
    python -m emri_kludge_suite_b200.workloads tdi        # frequency-domain TDI of the waveform workload's 16 sources, twice
    python -m emri_kludge_suite_b200.workloads mlp        # warm-start network: forward on 2^20 points, a training step
"""
from __future__ import annotations

import math
import sys

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


def profile_waveform():
    import torch

    from .aak import WaveBatch

    src, _ = config1(SEED, 512)
    wb = WaveBatch(0)
    wb.plan(src[::32][:16], nmodes=NMODES)
    wb.upload()
    n = wb.total_samples
    hI = torch.empty(n, dtype=torch.float64, device="cuda")
    hII = torch.empty_like(hI)
    for precision in (0, 1):
        for _ in range(2):
            wb.run(hI.data_ptr(), hII.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    print("waveform workload:", n, "samples")


def profile_phase():
    """The phase product of the same 16 sources as the waveform workload, twice
    (64 B/sample of outputs: 1.8 GB, above the 126 MB L2)."""
    import torch

    from .aak import WaveBatch

    src, _ = config1(SEED, 512)
    wb = WaveBatch(0)
    wb.plan(src[::32][:16], nmodes=NMODES)
    wb.upload()
    n = wb.total_samples
    out = torch.empty(8 * n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        wb.run_phase(out.data_ptr(), n)
    torch.cuda.synchronize()
    assert wb.device_status() == 0
    print("phase workload:", n, "samples")


def profile_fisher():
    """Two Fisher-matrix calls at the configuration-4 fiducial point: 28
    templates of 3.2e6 samples (1.43 GB of spectra, above the 126 MB L2)."""
    from .gpuAAK import GPUAAK

    length, dt = 3_200_000, 10.0
    x0 = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.8, 2.0, 1.0])
    g = GPUAAK(1.0, 100, length, 100.0, dt, True, False)
    X = np.tile(x0, (28, 1))
    for i in range(14):
        X[2 * i, i] += 1e-6 * max(abs(x0[i]), 1.0)
        X[2 * i + 1, i] -= 1e-6 * max(abs(x0[i]), 1.0)
    for _ in range(2):
        G, st = g.fisher_gram(X, 1.0, return_status=True)
        assert np.all(st == 0) and np.all(np.isfinite(G))
    print("fisher workload: 28 x", length, "samples")


def profile_tdi():
    """The frequency-domain TDI of the same 16 sources as the waveform workload, twice."""
    from .aak import WaveBatch

    src, _ = config1(SEED, 512)
    wb = WaveBatch(0)
    for _ in range(2):
        rows, offs, st = wb.tdi_host(src[::32][:16])
    assert np.all(st == 0) and np.all(np.isfinite(rows))
    print("tdi workload:", int(offs[-1]), "bins")


def profile_mlp():
    import torch

    from . import parmap_mlp as P

    d = P.make_dataset(1 << 16, 5)
    m = P.ParMapMLP(0, seed=1)
    m.fit_norm(d["x"][d["valid"]], d["y"][d["valid"]])
    n = 1 << 20
    x = torch.tensor(np.tile(d["x"], (16, 1)).astype(np.float32), device="cuda")
    y = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    yt = torch.tensor(np.tile(np.nan_to_num(d["y"]), (16, 1)).astype(np.float32), device="cuda")
    for _ in range(2):
        m.forward_device(x.data_ptr(), y.data_ptr(), n)
        m.train_step_device(x.data_ptr(), yt.data_ptr(), 16384, 1e-3)
    torch.cuda.synchronize()
    print("mlp workload done")


if __name__ == "__main__":
    {"waveform": profile_waveform, "phase": profile_phase, "fisher": profile_fisher,
     "tdi": profile_tdi, "mlp": profile_mlp}[sys.argv[1] if len(sys.argv) > 1 else "waveform"]()
