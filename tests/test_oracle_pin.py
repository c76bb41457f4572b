"""Pin the oracle restatement (oracle/aak_oracle.c) to the reference.

Against the committed fixtures (made by the reference itself, see
tests/golden/make_golden.py) and, where the reference build exists, live.
"""
import numpy as np
import pytest
import scipy.special as sp

from conftest import golden_mapped, golden_names, load_golden, mismatch
from oracle import oracle as O


@pytest.mark.parametrize("name", golden_names())
def test_oracle_waveform_matches_reference_fixture(name):
    g = load_golden(name)
    pars = g["pars"]
    mt = O.MappedTrajectory(int(g["steps"]), g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"],
                            float(g["Phi0"]), 2)
    t, hI, hII, ip, ib = O.oracle_genwave(pars, mt, int(g["nmodes"]))
    scale = max(np.abs(g["genwave_hI"]).max(), np.abs(g["genwave_hII"]).max())
    # identical algorithm, independent Bessel evaluation: agreement to ~1e-13
    assert np.array_equal(t, g["genwave_t"])
    assert np.abs(hI - g["genwave_hI"]).max() / scale < 1e-11
    assert np.abs(hII - g["genwave_hII"]).max() / scale < 1e-11
    assert mismatch(hI, hII, g["genwave_hI"], g["genwave_hII"]) < 1e-14


@pytest.mark.parametrize("name", [n for n in golden_names() if "dense_t" in load_golden(n)])
def test_oracle_dense_trajectory_matches_reference_fixture(name):
    g = load_golden(name)
    pars = g["pars"]
    mt = O.MappedTrajectory(int(g["steps"]), g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"],
                            float(g["Phi0"]), 2)
    arrs, ip, ib = O.oracle_pnevolution(pars, mt)
    assert ip == int(g["i_plunge"]) and ib == int(g["i_buffer"])
    for k, a in zip("t e v M S gim Phi alp nu gimdot".split(), arrs):
        ref = g["dense_" + k]
        rel = np.max(np.abs(a - ref) / np.maximum(np.abs(ref), 1e-300))
        assert rel < 1e-12, (k, rel)


@pytest.mark.parametrize("name", golden_names())
def test_oracle_phases_match_reference_fixture(name):
    """GenPhase restatement against the reference AAKphase outputs."""
    g = load_golden(name)
    pars = g["pars"]
    mt = O.MappedTrajectory(int(g["steps"]), g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"],
                            float(g["Phi0"]), 2)
    out = O.oracle_genphase(pars, mt)
    assert np.array_equal(out[0], g["aakwave_t"])
    for k, a in zip(O.PHASE_KEYS[1:], out[1:8]):
        ref = g["aakphase_" + k]
        # the phases grow to ~1e5 rad: compare them against their largest value;
        # the rates and e sample by sample
        den = np.abs(ref).max() if k.startswith("phase") else np.maximum(np.abs(ref), 1e-300)
        rel = np.max(np.abs(a - ref) / den)
        assert rel < 1e-13, (k, rel)


def test_oracle_phase_freeze_after_plunge_buffer():
    """The phases of the samples after i_plunge + i_buffer + 1 hold their values at
    i_plunge (AAKPhase.cc:253-257); the rates and e run on."""
    g = load_golden("plunge")
    pars = g["pars"]
    mt = O.MappedTrajectory(int(g["steps"]), g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"],
                            float(g["Phi0"]), 2)
    t, pr, pt, pp, wr, wt, wp, e, ip, ib = O.oracle_genphase(pars, mt)
    first = ip + ib + 2
    assert first < len(t)
    for a in (pr, pt, pp):
        assert np.all(a[first:] == a[ip])
        assert a[first - 1] != a[ip]
    assert not np.all(wr[first:] == wr[ip])


def _tdi_scale(rows):
    return max(np.abs(r).max() for r in rows) or 1.0


@pytest.mark.parametrize("name", golden_names())
def test_oracle_tdi_matches_reference_fixture(name):
    """GenTDI restatement (phase grid + stationary-phase sum) against the
    reference AAKTDI outputs.  The SPA phase faza - Om xi cancels ~1e5-1e6 rad
    to a few rad, so rounding of the phases shows at ~1e-10 of the largest bin."""
    g = load_golden(name)
    pars = g["pars"]
    mt = O.MappedTrajectory(int(g["steps"]), g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"],
                            float(g["Phi0"]), 2)
    out = O.oracle_gentdi(pars, mt)
    n = (int(pars["length"]) + 1) // 2
    assert np.array_equal(out[0], np.arange(n) * (1.0 / ((int(pars["length"]) - 1) * pars["dt"])))
    ref = [g["aaktdi_" + k] for k in O.TDI_KEYS[1:]]
    sc = _tdi_scale(ref)
    for k, a, b in zip(O.TDI_KEYS[1:], out[1:7], ref):
        assert np.array_equal(a != 0, b != 0), k
        assert np.abs(a - b).max() / sc < 1e-9, k


@pytest.mark.parametrize("extra", [dict(length=400000), dict(length=300000, e=0.4, dt=30.0),
                                   dict(length=100000, p=6.0, mu=100.0, dt=100.0, backint=True)])
def test_oracle_tdi_matches_reference_live(ref_available, extra):
    """Longer spans (1e5-4e5 bins), run through the reference build itself."""
    if not ref_available:
        pytest.skip("reference build (oracle/_ref) not present")
    from tests.golden.make_golden import BASE
    pars = dict(BASE)
    pars.update(extra)
    pars["T"] = pars["length"] * pars["dt"] / O.YEAR
    mt = O.ref_front(pars)
    ref = O.ref_gentdi(pars, mt)
    out = O.oracle_gentdi(pars, mt)
    sc = _tdi_scale(ref[1:])
    assert np.count_nonzero(ref[1]) > 1000
    for a, b in zip(out[1:7], ref[1:]):
        assert np.abs(a - b).max() / sc < 1e-9


def test_oracle_bessel_against_scipy():
    rng = np.random.default_rng(7)
    for _ in range(200):
        n = int(rng.integers(1, 101))
        e = float(rng.uniform(0.001, 0.95))
        x = n * e
        lo = max(n - 2, 0)
        got = O.oracle_bessel(lo, n + 2, x)
        want = sp.jv(np.arange(lo, n + 3), x)
        scale = np.abs(want).max()
        assert np.abs(got - want).max() <= 1e-13 * scale + 1e-300


def test_oracle_pn_rates_match_reference(ref_available):
    if not ref_available:
        pytest.skip("reference build (oracle/_ref) not present")
    L = O.oracle_lib()
    rng = np.random.default_rng(3)
    for _ in range(100):
        v, e, Y, q = rng.uniform(0.1, 0.45), rng.uniform(0.01, 0.8), rng.uniform(-1, 1), rng.uniform(-0.95, 0.95)
        m, M = 1e-4, 5.0
        ref = O.ref_pn_rates(v, e, Y, q, m, M)
        ours = [L.oracle_dtdm(v, e, Y, q), L.oracle_drdm(v, e, Y, q), L.oracle_dthetadm(v, e, Y, q),
                L.oracle_dphidm(v, e, Y, q), L.oracle_dvdt(v, e, Y, m, M, q), L.oracle_dedt(v, e, Y, m, M, q)]
        np.testing.assert_allclose(ours, ref, rtol=1e-14, atol=0)


def test_oracle_kerr_stability_matches_reference(ref_available):
    if not ref_available:
        pytest.skip("reference build (oracle/_ref) not present")
    rng = np.random.default_rng(11)
    for _ in range(150):
        p, e, ci, a = rng.uniform(3.0, 15.0), rng.uniform(0.05, 0.8), rng.uniform(-0.99, 0.99), rng.uniform(0, 0.95)
        if abs(ci) < 0.05:
            continue
        ref = O.ref_iekg(p, e, ci, a)
        ours = O.oracle_kerr_constants(p, e, ci, a)
        # deep inside the unstable region the constants are not unique; only the flag is used there
        if ref[3] == 1:
            np.testing.assert_allclose(ours[:3], ref[:3], rtol=1e-12, atol=1e-14)
        if ref[3] in (-1, 0, 1):
            assert ours[3] == ref[3]


def test_fisher_oracle_forms_against_pairwise_sums():
    """The vectorised Fisher oracle against pair-by-pair sums over bins, in the
    reference's pairing (pygpuAAK/pygpuAAK.py:286-298) and the full one."""
    rng = np.random.default_rng(9)
    nd, nb = 5, 257
    hI = rng.standard_normal((2 * nd, nb)) + 1j * rng.standard_normal((2 * nd, nb))
    hII = rng.standard_normal((2 * nd, nb)) + 1j * rng.standard_normal((2 * nd, nb))
    eps = 1e-3
    G = O.fisher_gram(hI, hII, 1.0 / (2 * eps))
    M = O.fisher_reference_form(G)
    for i in range(nd):
        di = [(h[2 * i + 1] - h[2 * i]) / (2 * eps) for h in (hI, hII)]
        for j in range(nd):
            dj = [(h[2 * j + 1] - h[2 * j]) / (2 * eps) for h in (hI, hII)]
            for c in range(2):
                want = 4 * np.real(np.sum(np.conj(di[c]) * dj[c]))
                assert abs(G[c, i, j] - want) <= 1e-12 * abs(want) + 1e-9
            a, b = min(i, j), max(i, j)
            da = [(h[2 * a + 1] - h[2 * a]) / (2 * eps) for h in (hI, hII)]
            db = [(h[2 * b + 1] - h[2 * b]) / (2 * eps) for h in (hI, hII)]
            want = 4 * np.real(np.sum(np.conj(db[0]) * db[0]) + np.sum(np.conj(da[1]) * db[1]))
            assert abs(M[i, j] - want) <= 1e-12 * abs(want)
