"""GPU likelihood (GPUAAK / pyGPUAAK call shapes) against the numpy likelihood
oracle (oracle/oracle.py: inner_products) on oracle waveforms."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.gpuAAK import GPUAAK  # noqa: E402
from emri_kludge_suite_b200.LISAnoise import LISA_Noise  # noqa: E402
from emri_kludge_suite_b200.pygpuAAK import pyGPUAAK  # noqa: E402
from oracle import oracle as O  # noqa: E402

LENGTH, DT = 40000, 10.0
# gpu_gen_AAK order: iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D
INJ = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.3, 0.2, 0.4, 0.5, 1.0, 0.8, 2.0, 1.0])


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _pars(x, length=LENGTH, dt=DT):
    iota, s, p, e, M, mu, gamma, psi, alph, thS, phS, thK, phK, D = x
    return dict(backint=False, LISA=True, length=length, dt=dt, p=p, T=length * dt / O.YEAR, f=0.0, T_fit=1.0, mu=mu,
                M=M, s=s, e=e, iota=iota, gamma=gamma, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK, phi_K=phK,
                alpha=alph, D=D)


def _oracle_wave(x):
    pars = _pars(x)
    m = E.front_end(pars)  # host front end (pinned against the reference in test_front_end.py)
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    _, hI, hII, _, _ = O.oracle_genwave(pars, mt, 0)
    return hI, hII


def _weights():
    w = O.noise_weights(LENGTH, DT, dur=1)
    return w, w.copy()


def test_single_template_likelihood_matches_oracle():
    w1, w2 = _weights()
    dI, dII = _oracle_wave(INJ * np.r_[1, 1, 1.001, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1])
    D1 = np.fft.rfft(dI) * w1
    D2 = np.fft.rfft(dII) * w2
    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    g.input_data(D1, D2, w1, w2)
    g.gpu_gen_AAK(*INJ)
    t, hI, hII = g.GetWaveform()
    oI, oII = _oracle_wave(INJ)
    assert len(hI) == LENGTH + 2
    assert np.abs(hI[:LENGTH] - oI).max() <= 1e-8 * np.abs(oI).max()
    like = g.Likelihood()
    ref = O.inner_products(oI, oII, D1, D2, w1, w2)
    np.testing.assert_allclose(like, ref, rtol=1e-8)
    # after Likelihood the rows hold the weighted half spectra, as in the reference
    _, sI, sII = g.GetWaveform(is_Fourier=True)
    spec = sI[0::2][: LENGTH // 2 + 1] + 1j * sI[1::2][: LENGTH // 2 + 1]
    want = np.fft.rfft(oI) * w1
    assert np.abs(spec - want).max() <= 1e-8 * np.abs(want).max()


def test_batch_equals_single_template_calls():
    w1, w2 = _weights()
    dI, dII = _oracle_wave(INJ)
    D1, D2 = np.fft.rfft(dI) * w1, np.fft.rfft(dII) * w2
    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    g.input_data(D1, D2, w1, w2)
    rng = np.random.default_rng(4)
    X = np.tile(INJ, (7, 1))
    X[:, 2] *= 1 + 1e-4 * rng.standard_normal(7)
    X[:, 6:11] += 1e-2 * rng.standard_normal((7, 5))
    X[3, 3] = -0.5  # invalid eccentricity: zero template, status reported
    out, st = g.likelihood_batch(X, max_batch=3, return_status=True)
    assert st[3] != 0 and np.all(out[3] == 0.0)
    for k in range(7):
        if k == 3:
            continue
        g.gpu_gen_AAK(*X[k])
        one = g.Likelihood()
        np.testing.assert_allclose(out[k], one, rtol=1e-13)


def test_pygpuaak_nll_is_zero_at_injection_without_noise():
    keys = ["iota", "s", "p", "e", "M", "mu", "gamma", "psi", "alpha", "theta_S", "phi_S", "theta_K", "phi_K", "D"]
    inj = dict(zip(keys, INJ))
    like = pyGPUAAK({"injection_params": inj}, LENGTH, DT, 100.0, keys, backint=False)
    x = np.tile(INJ, (3, 1)).T.copy()
    x[2, 1] *= 1.0001
    nll = like.getNLL(x)
    assert abs(nll[0]) <= 1e-9 * like.d_d
    assert nll[1] > nll[0]
    # the injected SNR^2 equals <h|h>
    snr_d, snr_h = like.NLL(*INJ, return_snr=True)
    assert snr_h[0] ** 2 == pytest.approx(like.d_d, rel=1e-9)


def test_fp32_transform_and_compensated_products_against_fp64_oracle():
    """Precision 2: split templates in FP32 rows, an FP32 R2C transform and the
    Kahan-compensated FP32 inner products, against the FP64 oracle's inner
    products of the FP64 oracle waveforms.  Bar: 2e-5 relative on <h|d> and
    <h|h>, and |dlogL| <= 2e-5 (d_d + h_h) (the FP32 transform's rounding)."""
    w1, w2 = _weights()
    dI, dII = _oracle_wave(INJ * np.r_[1, 1, 1.0001, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1])
    D1, D2 = np.fft.rfft(dI) * w1, np.fft.rfft(dII) * w2
    d_d = 4.0 * float(np.sum(np.abs(D1) ** 2) + np.sum(np.abs(D2) ** 2))
    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    g.input_data(D1, D2, w1, w2)
    rng = np.random.default_rng(11)
    X = np.tile(INJ, (5, 1))
    X[:, 2] *= 1 + 1e-5 * rng.standard_normal(5)
    X[:, 6:11] += 1e-3 * rng.standard_normal((5, 5))
    g.set_precision(2)
    out32, st = g.likelihood_batch(X, max_batch=4, return_status=True)
    g.set_precision(0)
    out64 = g.likelihood_batch(X, max_batch=4)
    assert np.all(st == 0)
    worst = 0.0
    for k in range(len(X)):
        oI, oII = _oracle_wave(X[k])
        ref = O.inner_products(oI, oII, D1, D2, w1, w2)
        np.testing.assert_allclose(out64[k], ref, rtol=1e-8)
        np.testing.assert_allclose(out32[k], ref, rtol=2e-5)
        dl = 0.5 * abs((out32[k, 1] - 2 * out32[k, 0]) - (ref[1] - 2 * ref[0]))
        worst = max(worst, dl / (d_d + ref[1]))
    print("fp32 likelihood: max |dlogL| / (d_d + h_h) =", worst)
    assert worst <= 2e-5


def test_warm_started_batch_equals_single_template_calls():
    """With a learned warm start, a likelihood batch does each chunk's front end
    (coarse inspirals, one prediction launch, map solves) two chunks ahead of
    its planning; the templates must come out as single-template calls, whose
    planner runs the warm-started front end itself."""
    from emri_kludge_suite_b200 import parmap_mlp as PM

    train = PM.make_dataset(1 << 14, seed=41)
    m = PM.ParMapMLP(0, seed=2)
    m.train(train["x"][train["valid"]], train["y"][train["valid"]], epochs=10, batch=4096, lr=1e-2)
    w1, w2 = _weights()
    dI, dII = _oracle_wave(INJ)
    D1, D2 = np.fft.rfft(dI) * w1, np.fft.rfft(dII) * w2
    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    g.input_data(D1, D2, w1, w2)
    g.set_warm_start(m)
    rng = np.random.default_rng(5)
    X = np.tile(INJ, (9, 1))
    X[:, 2] *= 1 + 1e-4 * rng.standard_normal(9)
    X[:, 6:11] += 1e-2 * rng.standard_normal((9, 5))
    X[4, 3] = -0.5  # invalid eccentricity: zero template, status reported
    out, st = g.likelihood_batch(X, max_batch=2, return_status=True)  # five chunks: the front ends run ahead
    assert st[4] != 0 and np.all(out[4] == 0.0)
    for k in range(9):
        if k == 4:
            continue
        assert st[k] == 0
        g.gpu_gen_AAK(*X[k])
        np.testing.assert_allclose(out[k], g.Likelihood(), rtol=1e-13)
