"""GPU parity of the frequency-domain AAK TDI (AAKTDI / GenTDI,
src/suite/AAKTDI.cc:27-829; AAKwrapper.tdi, AAKwrapper/AAKwrapper.pyx:135-177)
against the reference fixtures and the oracle restatement.  Calls go through
the C ABI."""
import numpy as np
import pytest

from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from oracle import oracle as O  # noqa: E402

BASE = dict(backint=False, LISA=True, length=1000, dt=10.0, p=8.0, T=0.25, f=2e-3, T_fit=1.0, mu=10.0, M=1e6, s=0.5,
            e=0.2, iota=0.785, gamma=0.0, psi=0.0, theta_S=0.5, phi_S=1.0, theta_K=0.8, phi_K=2.0, alpha=0.0, D=1.0)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _err(rows, ref):
    """Largest difference over the six rows relative to the largest reference bin."""
    sc = max(np.abs(r).max() for r in ref) or 1.0
    return max(np.abs(a - b).max() for a, b in zip(rows, ref)) / sc


def _oracle(pars):
    m = E.front_end(pars)  # the same host front end as the GPU path
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    return O.oracle_gentdi(pars, mt)


@pytest.mark.parametrize("name", golden_names())
def test_tdi_matches_oracle_and_reference_fixture(name):
    """AAKwrapper.tdi call shape: against the oracle on the same mapped
    trajectory (the stationary-phase phases cancel ~1e5 rad to a few rad, so
    rounding shows at ~1e-10 of the largest bin), and against the reference's
    own outputs (its front end differs from this one at 1e-13, which the phases
    integrate)."""
    g = load_golden(name)
    pars = g["pars"]
    out = E.tdi(pars)
    assert len(out) == 8 and out[7] > 0
    n = (int(pars["length"]) + 1) // 2
    assert np.array_equal(out[0], np.arange(n) * (1.0 / ((int(pars["length"]) - 1) * pars["dt"])))
    ora = _oracle(pars)
    assert _err(out[1:7], ora[1:7]) < 1e-9
    ref = [g["aaktdi_" + k] for k in O.TDI_KEYS[1:]]
    assert _err(out[1:7], ref) < 1e-6


@pytest.mark.parametrize("extra", [dict(length=3200000), dict(length=1000000, e=0.4),
                                   dict(length=800000, mu=30.0, M=3e5, p=10.5, s=0.7, iota=2.0),
                                   dict(length=100000, p=6.0, mu=100.0, dt=100.0, backint=True)])
def test_tdi_long_spans_against_oracle(extra):
    """A year of configuration 0 (1.6e6 bins), a higher-eccentricity source
    (12 harmonics), a retrograde source around a lighter, faster-spinning black
    hole, and a backint source that plunges inside the span."""
    pars = dict(BASE)
    pars.update(extra)
    pars["T"] = pars["length"] * pars["dt"] / O.YEAR
    out = E.tdi(pars)
    ora = _oracle(pars)
    assert np.count_nonzero(ora[1]) > 1000
    assert _err(out[1:7], ora[1:7]) < 1e-8


def test_tdi_batch_equals_single_source_calls():
    """aak_tdi_batch_host over five sources (one invalid) equals the single
    calls bin for bin up to the order of the atomic adds."""
    rng = np.random.default_rng(17)
    params = []
    for _ in range(5):
        p = dict(BASE)
        p.update(e=float(rng.uniform(0.15, 0.4)), p=float(rng.uniform(8, 12)), length=int(rng.integers(20000, 200000)),
                 iota=float(rng.uniform(0.2, 2.8)), theta_S=float(rng.uniform(0.3, 2.8)), phi_S=float(rng.uniform(0, 6)))
        params.append(p)
    params[2] = dict(params[2], e=-0.1)
    wb = E.WaveBatch(0)
    rows, offs, st = wb.tdi_host(params)
    assert st[2] != 0 and np.all(np.delete(st, 2) == 0)
    assert np.all(rows[:, offs[2]:offs[3]] == 0.0)
    for s in (0, 1, 3, 4):
        one = E.tdi(params[s])
        seg = rows[:, offs[s]:offs[s + 1]]
        assert _err(list(seg), list(one[1:7])) < 1e-13
