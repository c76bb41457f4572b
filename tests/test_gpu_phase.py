"""GPU parity of the AAK phase product (GenPhase, src/suite/AAKPhase.cc:315-374;
AAKwrapper.phase, AAKwrapper/AAKwrapper.pyx:90-133) against the reference
fixtures and the oracle restatement.  Calls go through the C ABI."""
import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.aak import PHASE_ROWS  # noqa: E402
from oracle import oracle as O  # noqa: E402

BASE = dict(backint=False, LISA=True, length=1000, dt=10.0, p=8.0, T=0.25, f=2e-3, T_fit=1.0, mu=10.0, M=1e6, s=0.5,
            e=0.2, iota=0.785, gamma=0.0, psi=0.0, theta_S=0.5, phi_S=1.0, theta_K=0.8, phi_K=2.0, alpha=0.0, D=1.0)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def _run_phase(params, mapped=None):
    """Plan (optionally on given mapped trajectories), upload, phase product into
    a device buffer; returns (rows (8, N) on host, batch)."""
    wb = E.WaveBatch(0)
    wb.plan(params, mapped=mapped)
    N = wb.total_samples
    out = torch.full((8, N), float("nan"), dtype=torch.float64, device="cuda")
    wb.upload()
    wb.run_phase(out.data_ptr(), N)
    torch.cuda.synchronize()
    assert wb.launches() == 3  # tile parameters, phase pass, freeze
    assert wb.device_status() == 0
    return out.cpu().numpy(), wb


def _check_rows(rows, ref, phase_tol, rate_tol, e_tol):
    """rows/ref: the eight arrays of PHASE_ROWS.  Time bit-exact; the phases
    (which grow to ~1e5 rad) against their largest value; the rates and e
    sample by sample."""
    assert np.array_equal(rows[0], ref[0])
    for k in (1, 2, 3):
        err = np.max(np.abs(rows[k] - ref[k])) / max(1.0, np.abs(ref[k]).max())
        assert err < phase_tol, (PHASE_ROWS[k], err)
    for k in (4, 5, 6):
        err = np.max(np.abs(rows[k] - ref[k]) / np.abs(ref[k]))
        assert err < rate_tol, (PHASE_ROWS[k], err)
    err = np.max(np.abs(rows[7] - ref[7]) / np.abs(ref[7]))
    assert err < e_tol, ("eccentricity", err)


@pytest.mark.parametrize("name", golden_names())
def test_phase_on_reference_mapped_trajectory_matches_reference(name):
    """Same mapped trajectory as the reference AAKphase: the phase product
    agrees with its outputs to FP64 rounding of the reassociated phase sums."""
    g = load_golden(name)
    rows, wb = _run_phase([g["pars"]], mapped=[golden_mapped(g)])
    assert wb.status[0] == 0
    ref = [g["aakwave_t"]] + [g["aakphase_" + k] for k in PHASE_ROWS[1:]]
    _check_rows(rows, ref, phase_tol=1e-12, rate_tol=1e-12, e_tol=1e-13)


@pytest.mark.parametrize("name", golden_names())
def test_phase_end_to_end_matches_reference_aakphase(name):
    """AAKwrapper.phase call shape: host front end + GPU phase product.  The
    front end (Newton map of the coarse Kerr inspiral) differs from the
    reference's at the 1e-13 level, which the phases integrate; after a
    plunge the fitted e extrapolates it to ~4e-11."""
    g = load_golden(name)
    out = E.phase(g["pars"])
    assert len(out) == 9 and out[8] > 0
    ref = [g["aakwave_t"]] + [g["aakphase_" + k] for k in PHASE_ROWS[1:]]
    _check_rows(out[:8], ref, phase_tol=1e-9, rate_tol=1e-10, e_tol=1e-10)


def test_phase_batch_matches_oracle_and_freezes_after_plunge_buffer():
    """Every golden source in one batch (plus an invalid one): each source's rows
    equal the oracle's GenPhase on the same mapped trajectory; the failed source
    is zero; the frozen phases equal their values at i_plunge exactly."""
    names = golden_names()
    gs = [load_golden(n) for n in names]
    params = [g["pars"] for g in gs] + [dict(BASE, e=-0.3)]
    mapped = [golden_mapped(g) for g in gs] + [golden_mapped(gs[0])]
    rows, wb = _run_phase(params, mapped=mapped)
    assert wb.status[-1] != 0 and np.all(wb.status[:-1] == 0)
    o = wb.offsets
    assert np.all(rows[:, o[-2]:o[-1]] == 0.0)
    froze = 0
    for s, g in enumerate(gs):
        mt = O.MappedTrajectory(int(g["steps"]), g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"],
                                float(g["Phi0"]), 2)
        ref = O.oracle_genphase(g["pars"], mt)
        assert wb.i_plunge[s] == ref[8] and wb.i_buffer[s] == ref[9]
        r = rows[:, o[s]:o[s + 1]]
        _check_rows(r, ref[:8], phase_tol=1e-12, rate_tol=1e-12, e_tol=1e-13)
        first = int(wb.i_plunge[s]) + int(wb.i_buffer[s]) + 2
        if first < r.shape[1]:
            froze += 1
            for k in (1, 2, 3):
                assert np.all(r[k, first:] == r[k, wb.i_plunge[s]])
    assert froze >= 1


def test_phase_long_backward_chain_against_oracle():
    """backint, 400,000 samples with t = 0 near the end: ~380 tiles chain
    backward.  The device sums the AB2 increments by block scans and
    double-double carries, the oracle one by one."""
    pars = dict(load_golden("plunge_backint")["pars"])
    pars.update(length=400000, T=400000 * pars["dt"] / O.YEAR, p=7.0)
    m = E.front_end(pars)
    rows, wb = _run_phase([pars], mapped=[m])
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    ref = O.oracle_genphase(pars, mt)
    assert rows[0][1] < 0.0 < rows[0][-1]
    _check_rows(rows, ref[:8], phase_tol=1e-11, rate_tol=1e-12, e_tol=1e-13)


def test_phase_host_batch_equals_device_batch():
    """aak_phase_batch_host (plan + upload + phase product + copy back) equals
    the device-buffer call, and single-source aak_phase equals its batch row."""
    rng = np.random.default_rng(5)
    params = []
    for _ in range(6):
        p = dict(BASE)
        p.update(e=float(rng.uniform(0.1, 0.4)), p=float(rng.uniform(8, 12)), length=int(rng.integers(3000, 30000)),
                 iota=float(rng.uniform(0.2, 2.8)), mu=float(rng.uniform(5, 60)), backint=bool(rng.integers(0, 2)))
        params.append(p)
    wh = E.WaveBatch(0)
    host, off, st = wh.phase_host(params)
    assert np.all(st == 0)
    dev, wd = _run_phase(params)
    assert np.array_equal(wd.offsets, off)
    assert np.array_equal(host, dev)
    single = E.phase(params[3])
    for k in range(8):
        assert np.array_equal(single[k], host[k, off[3]:off[4]])
