"""Likelihoods at the full configuration-4 length (3,200,000 samples, the
5-smooth FFT length that holds one year at dt = 10 s) against the numpy
likelihood oracle (oracle/oracle.py: inner_products) on FP64 oracle waveforms.

Data: the fiducial configuration-0 source observed for 1.014 yr (it plunges
after 0.79 yr, so the taper and the frozen tail are in the window) plus seeded
LISA-coloured noise, weighted by S_n^{-1/2} sqrt(dt/N) as pyGPUAAK does
(pygpuAAK.py:67-96).  Templates: the fiducial itself and three perturbations
of it (1e-5 relative in M, mu, p0; 1e-3 rad in the angles), the reference's
harmonic rule.  Every precision of the batched path is compared with the
oracle: FP64 (0), split waveforms with the FP64 transform (1), split waveforms
with the FP32 transform and compensated FP32 products (2)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.gpuAAK import GPUAAK  # noqa: E402
from emri_kludge_suite_b200.LISAnoise import LISA_Noise, generate_noise_frequencies, generate_noise_single_channel  # noqa: E402
from oracle import oracle as O  # noqa: E402

LENGTH, DT = 3_200_000, 10.0
# gpu_gen_AAK order: iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D
FIDUCIAL = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.8, 2.0, 1.0])
# bars on |d<h|d>|, |d<h|h>| and |dlogL|, relative to <h|h> of the template
# (<h|d> of a perturbed template can be near zero, and the noise part of <d|d>
# cancels in dlogL).  FP64: the bar of the full-length FP64 waveforms (the
# oracle's sequential FP64 phase sum alone rounds by ~sqrt(N) eps Phi, ~4e-8 rad
# at this length); split and FP32: the split harmonic sums' level.
TOL = {0: 1e-7, 1: 2e-5, 2: 2e-5}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    O.set_threads(os.cpu_count() or 1)
    yield
    O.set_threads(1)


def _pars(x):
    iota, s, p, e, M, mu, gamma, psi, alph, thS, phS, thK, phK, D = x
    return dict(backint=False, LISA=True, length=LENGTH, dt=DT, p=p, T=LENGTH * DT / O.YEAR, f=0.0, T_fit=1.0, mu=mu,
                M=M, s=s, e=e, iota=iota, gamma=gamma, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK, phi_K=phK,
                alpha=alph, D=D)


def _oracle_wave(x):
    pars = _pars(x)
    m = E.front_end(pars)  # host front end (pinned against the reference in test_front_end.py)
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    _, hI, hII, i_plunge, _ = O.oracle_genwave(pars, mt, 0)
    return hI, hII, i_plunge


def _templates():
    rng = np.random.default_rng(404)
    X = np.tile(FIDUCIAL, (4, 1))
    for j in (2, 4, 5):
        X[1:, j] *= 1.0 + 1e-5 * rng.standard_normal(3)
    for j in (0, 6, 7, 8, 9, 10, 11, 12):
        X[1:, j] += 1e-3 * rng.standard_normal(3)
    return X


def test_config4_length_likelihoods_against_oracle():
    freqs = generate_noise_frequencies(LENGTH * DT, 1 / DT)
    freqs[0] = freqs[1] / 10.0
    w = O.noise_weights(LENGTH, DT, dur=1)
    sI, sII, i_plunge = _oracle_wave(FIDUCIAL)
    assert 0 < i_plunge < LENGTH - 1  # the fiducial plunges inside the window
    rng = np.random.default_rng(2024)
    df = 1.0 / (LENGTH * DT)
    n1 = generate_noise_single_channel(LISA_Noise, [], {"dur": 1}, df, freqs, rng)
    n2 = generate_noise_single_channel(LISA_Noise, [], {"dur": 1}, df, freqs, rng)
    D1, D2 = w * (np.fft.rfft(sI) + n1), w * (np.fft.rfft(sII) + n2)
    d_d = 4.0 * float(np.sum(np.abs(D1) ** 2) + np.sum(np.abs(D2) ** 2))

    X = _templates()
    ref = []
    for x in X:
        hI, hII, _ = _oracle_wave(x)
        ref.append(O.inner_products(hI, hII, D1, D2, w, w))
    ref = np.array(ref)

    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    g.input_data(D1, D2, w, w)
    worst = {}
    for precision in (0, 1, 2):
        g.set_precision(precision)
        out, st = g.likelihood_batch(X, max_batch=2, return_status=True)
        assert np.all(st == 0), (precision, st)
        scale = ref[:, 1]
        dhd = np.abs(out[:, 0] - ref[:, 0]) / scale
        dhh = np.abs(out[:, 1] - ref[:, 1]) / scale
        dlogl = 0.5 * np.abs((out[:, 1] - 2 * out[:, 0]) - (ref[:, 1] - 2 * ref[:, 0])) / scale
        worst[precision] = (float(dhd.max()), float(dhh.max()), float(dlogl.max()))
        print(f"precision {precision}: / <h|h>: max |d<h|d>| {dhd.max():.2e}, max |d<h|h>| {dhh.max():.2e}, "
              f"max |dlogL| {dlogl.max():.2e} (<h|h> ~ {scale.mean():.1f}, d_d = {d_d:.4e})")
    g.set_precision(0)
    for precision, w3 in worst.items():
        assert max(w3) <= TOL[precision], (precision, w3)
