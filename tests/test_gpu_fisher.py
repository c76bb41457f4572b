"""GPU Fisher-matrix batch (pyGPUAAK.get_Fisher, pygpuAAK/pygpuAAK.py:269-300):
the device Gram reduction against the numpy oracle (oracle/oracle.py:
fisher_gram, fisher_reference_form) on the same spectra and on oracle
waveforms.  Calls go through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.gpuAAK import GPUAAK  # noqa: E402
from emri_kludge_suite_b200.pygpuAAK import pyGPUAAK  # noqa: E402
from oracle import oracle as O  # noqa: E402

LENGTH, DT = 40000, 10.0
# gpu_gen_AAK order: iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D
INJ = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.3, 0.2, 0.4, 0.5, 1.0, 0.8, 2.0, 1.0])
# central-difference steps large enough that the derivatives stand well above
# the 1e-8 relative agreement of two FP64 waveform evaluations
STEP = np.array([1e-3, 1e-3, 1e-3, 1e-3, 1e3, 1e-2, 1e-3, 1e-3, 1e-3, 1e-3, 1e-3, 1e-3, 1e-3, 1e-3])
# sampler coordinates of the get_Fisher test: log masses, as a sampler would use them
KEYS = ["iota", "s", "p", "e", "ln_M", "ln_mu", "gamma", "psi", "alpha", "theta_S", "phi_S", "theta_K", "phi_K", "D"]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rows(nd=14, base=INJ):
    X = np.tile(base, (2 * nd, 1))
    for i in range(nd):
        X[2 * i, i] += STEP[i]
        X[2 * i + 1, i] -= STEP[i]
    return X


def _generator():
    w = O.noise_weights(LENGTH, DT, dur=1)
    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    z = np.zeros(LENGTH // 2 + 1, dtype=np.complex128)
    g.input_data(z, z, w, w.copy())
    return g, w


def _spectra(g, X):
    """Weighted spectra of each row through the single-template path."""
    rows = [[], []]
    for x in X:
        g.gpu_gen_AAK(*x)
        g.Likelihood()
        _, sI, sII = g.GetWaveform(is_Fourier=True)
        n = LENGTH // 2 + 1
        rows[0].append(sI[0::2][:n] + 1j * sI[1::2][:n])
        rows[1].append(sII[0::2][:n] + 1j * sII[1::2][:n])
    return np.array(rows[0]), np.array(rows[1])


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_fisher_gram_matches_oracle_on_the_same_spectra():
    """One batched call (generate 28 templates, FFT, device Gram) equals the
    numpy Gram of the same templates' spectra taken one at a time."""
    g, _ = _generator()
    X = _rows()
    scale = 0.5
    G, st = g.fisher_gram(X, scale, return_status=True)
    assert np.all(st == 0)
    assert G.shape == (2, 14, 14)
    assert np.array_equal(G, np.transpose(G, (0, 2, 1)))
    sI, sII = _spectra(g, X)
    ref = O.fisher_gram(sI, sII, scale)
    # batched and single-template transforms may round differently; the
    # differences divide by steps of ~1e-3 relative
    assert _rel(G, ref) < 1e-10
    # deterministic: the same call again gives the same bits
    assert np.array_equal(g.fisher_gram(X, scale), G)


def test_fisher_gram_against_oracle_waveforms():
    """The device Gram against numpy on the oracle's waveforms (C restatement of
    the reference waveform) of the same 2 nd points, six derivatives."""
    g, w = _generator()
    nd = 6
    X = _rows(nd, base=np.r_[INJ[:3], 0.25, INJ[4:]])  # e = 0.25: another source than the other tests'
    G = g.fisher_gram(X, 1.0)
    H = [[], []]
    for x in X:
        iota, s, p, e, M, mu, gamma, psi, alph, thS, phS, thK, phK, D = x
        pars = dict(backint=False, LISA=True, length=LENGTH, dt=DT, p=p, T=LENGTH * DT / O.YEAR, f=0.0, T_fit=1.0,
                    mu=mu, M=M, s=s, e=e, iota=iota, gamma=gamma, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK,
                    phi_K=phK, alpha=alph, D=D)
        m = E.front_end(pars)
        mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
        _, hI, hII, _, _ = O.oracle_genwave(pars, mt, 0)
        H[0].append(np.fft.rfft(hI) * w)
        H[1].append(np.fft.rfft(hII) * w)
    ref = O.fisher_gram(np.array(H[0]), np.array(H[1]), 1.0)
    # two FP64 waveform evaluations agree to ~1e-11 relative; the differences
    # divide that by steps of ~1e-3 (measured: 3e-9 at worst)
    for c in range(2):
        d = np.sqrt(np.diag(ref[c]))
        assert np.abs(np.diag(G[c]) / np.diag(ref[c]) - 1).max() < 1e-6
        assert np.abs(G[c] / np.outer(d, d) - ref[c] / np.outer(d, d)).max() < 1e-6


def test_get_fisher_reference_and_full_forms():
    """pyGPUAAK.get_Fisher (one batched device call) against the reference's own
    procedure on this project's spectra: getNLL(return_TDI=True) of the 2 ndim
    points, then the reference's pairing of the derivative spectra."""
    x = INJ.copy()
    x[4:6] = np.log(x[4:6])
    inj = dict(zip(KEYS, x))
    like = pyGPUAAK({"injection_params": inj}, LENGTH, DT, 100.0, KEYS, backint=False, eps=1e-4)
    M_ref_form = like.get_Fisher(x)
    M_full = like.get_Fisher(x, form="full")
    x_in = np.tile(x, (2 * like.ndim, 1))
    for i in range(like.ndim):
        x_in[2 * i, i] += like.eps
        x_in[2 * i + 1, i] -= like.eps
    hI, hII = like.getNLL(x_in.T, return_TDI=True)
    G = O.fisher_gram(hI, hII, 1.0 / (2 * like.eps))
    # batch vs single-template transforms, divided by steps of 1e-4
    assert _rel(M_ref_form, O.fisher_reference_form(G)) < 1e-8
    assert _rel(M_full, G[0] + G[1]) < 1e-8
    assert np.array_equal(M_full, M_full.T) and np.all(np.diag(M_full) > 0)


def test_fisher_reports_failed_templates():
    g, _ = _generator()
    X = _rows(3)
    X[4, 3] = -0.5  # invalid eccentricity in one evaluation
    G, st = g.fisher_gram(X, 1.0, return_status=True)
    assert st[4] != 0 and np.all(np.delete(st, 4) == 0)
    assert np.all(np.isfinite(G))


def test_fisher_batch_equals_single_point_calls():
    """GPUAAK.fisher_gram_batch (aak_gpu_fisher_batch: the next point planned
    while the device reduces the current one, two planning contexts in turn)
    against one fisher_gram call per point; five points, so both result slots
    are reused, and one invalid template in the third point."""
    g, _ = _generator()
    rng = np.random.default_rng(17)
    pts = np.tile(INJ, (5, 1))
    pts[:, 2] *= 1 + 1e-3 * rng.standard_normal(5)
    pts[:, 6:11] += 1e-2 * rng.standard_normal((5, 5))
    rows = np.stack([_rows(14, p) for p in pts])
    rows[2, 7, 3] = -0.5  # invalid eccentricity: that template reported, the others unaffected
    G, st = g.fisher_gram_batch(rows, 0.5, return_status=True)
    assert G.shape == (5, 2, 14, 14) and st.shape == (5, 28)
    assert st[2, 7] != 0 and np.count_nonzero(st) == 1
    for k in range(5):
        Gk, sk = g.fisher_gram(rows[k], 0.5, return_status=True)
        assert np.array_equal(sk, st[k])
        assert np.abs(G[k] - Gk).max() <= 1e-12 * np.abs(Gk).max(), k
    # pyGPUAAK.get_Fisher_batch: the same matrices as get_Fisher point by point
    x = INJ.copy()
    x[4:6] = np.log(x[4:6])
    like = pyGPUAAK({"injection_params": dict(zip(KEYS, x))}, LENGTH, DT, 100.0, KEYS, backint=False, eps=1e-4)
    X = np.tile(x, (3, 1))
    X[:, 6:9] += 1e-2 * rng.standard_normal((3, 3))
    for form in ("reference", "full"):
        M = like.get_Fisher_batch(X, form=form)
        for k in range(3):
            Mk = like.get_Fisher(X[k], form=form)
            assert np.abs(M[k] - Mk).max() <= 1e-12 * np.abs(Mk).max(), (form, k)
