"""GPU parity of the dense AAK kernels (FP64 path) against the reference
fixtures and the oracle restatement.  Calls go through the C ABI."""
import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden, mismatch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200._lib import AAKValueError  # noqa: E402
from oracle import oracle as O  # noqa: E402

BASE = dict(backint=False, LISA=True, length=1000, dt=10.0, p=8.0, T=0.25, f=2e-3, T_fit=1.0, mu=10.0, M=1e6, s=0.5,
            e=0.2, iota=0.785, gamma=0.0, psi=0.0, theta_S=0.5, phi_S=1.0, theta_K=0.8, phi_K=2.0, alpha=0.0, D=1.0)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()


def _maxrel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", golden_names())
def test_genwave_matches_reference_fixture(name):
    """Same mapped trajectory in: waveform() semantics, harmonic-count override."""
    g = load_golden(name)
    t, hI, hII = E.genwave(g["pars"], golden_mapped(g), int(g["nmodes"]))
    assert np.array_equal(t, g["genwave_t"])
    # FP64 path vs the reference: phase sums reassociated, Bessel by recurrence
    assert _maxrel(hI, g["genwave_hI"]) < 1e-8
    assert _maxrel(hII, g["genwave_hII"]) < 1e-8
    assert mismatch(hI, hII, g["genwave_hI"], g["genwave_hII"]) < 1e-12


@pytest.mark.parametrize("name", golden_names())
def test_wave_end_to_end_matches_reference_aakwave(name):
    """AAKwrapper.wave call shape: host front end + GPU dense path, reference harmonic rule."""
    g = load_golden(name)
    t, hI, hII, secs = E.wave(g["pars"])
    assert secs > 0
    assert np.array_equal(t, g["aakwave_t"])
    assert mismatch(hI, hII, g["aakwave_hI"], g["aakwave_hII"]) < 1e-10
    assert _maxrel(hI, g["aakwave_hI"]) < 1e-6


@pytest.mark.parametrize("name", [n for n in golden_names() if "dense_t" in load_golden(n)])
def test_dense_trajectory_matches_reference(name):
    """Spline + AB2 phases (diagnostic trajectory output) vs PNevolution of the reference."""
    g = load_golden(name)
    pars = g["pars"]
    wb = E.WaveBatch(0)
    wb.plan([pars], nmodes=int(g["nmodes"]), mapped=[golden_mapped(g)])
    assert wb.status[0] == 0
    assert wb.i_plunge[0] == int(g["i_plunge"]) and wb.i_buffer[0] == int(g["i_buffer"])
    N = wb.total_samples
    hI = torch.zeros(N, dtype=torch.float64, device="cuda")
    hII = torch.zeros_like(hI)
    traj = torch.zeros(9 * N, dtype=torch.float64, device="cuda")
    wb.upload()
    wb.run(hI.data_ptr(), hII.data_ptr(), traj_ptr=traj.data_ptr(), traj_stride=N)
    torch.cuda.synchronize()
    tr = traj.view(9, N).cpu().numpy()
    n_out = min(N, int(g["i_plunge"]) + int(g["i_buffer"]))
    for row, k in enumerate(["e", "v", "M", "S"]):
        ref = g["dense_" + k][:n_out]
        rel = np.max(np.abs(tr[row, :n_out] - ref) / np.abs(ref))
        assert rel < 1e-13, (k, rel)
    for row, k in zip((4, 5, 6), ("gim", "Phi", "alp")):
        ref = g["dense_" + k][:n_out]
        # the trajectory bar, 1e-10 relative to the phase's largest value
        # (the sums are regrouped: tile scans with double-double carries)
        rel = np.max(np.abs(tr[row, :n_out] - ref)) / max(1.0, np.abs(ref).max())
        print(name, k, "max|dPhase|/max|Phase|", rel)
        assert rel < 1e-10, (k, rel)
    for row, k in zip((7, 8), ("nu", "gimdot")):
        ref = g["dense_" + k][:n_out]
        assert np.max(np.abs(tr[row, :n_out] - ref) / np.abs(ref)) < 1e-12, k


def test_batch_equals_single_source_calls():
    """Batched generation of mixed sources (one invalid) equals per-source calls."""
    names = golden_names()
    gs = [load_golden(n) for n in names]
    params = [g["pars"] for g in gs]
    bad = dict(BASE)
    bad.update(e=0.0, length=3000)
    params.insert(2, bad)
    maps = [golden_mapped(g) for g in gs]
    nmodes = [int(g["nmodes"]) for g in gs]
    wb = E.WaveBatch(0)
    # mapped path for the good ones: plan them together with one failing full-front-end source
    wb.plan(params, nmodes=[*nmodes[:2], 0, *nmodes[2:]])
    assert wb.status[2] != 0 and all(wb.status[i] == 0 for i in range(len(params)) if i != 2)
    N = wb.total_samples
    hI = torch.full((N,), 7.0, dtype=torch.float64, device="cuda")
    hII = torch.full((N,), 7.0, dtype=torch.float64, device="cuda")
    wb.upload()
    wb.run(hI.data_ptr(), hII.data_ptr())
    torch.cuda.synchronize()
    hI, hII = hI.cpu().numpy(), hII.cpu().numpy()
    o = wb.offsets
    assert np.all(hI[o[2]:o[3]] == 0.0) and np.all(hII[o[2]:o[3]] == 0.0)
    k = 0
    for i, p in enumerate(params):
        if i == 2:
            continue
        m = E.front_end(p)
        t1, a1, b1 = E.genwave(p, m, nmodes[k])
        assert np.array_equal(a1, hI[o[i]:o[i + 1]])
        assert np.array_equal(b1, hII[o[i]:o[i + 1]])
        k += 1


def test_configuration0_full_length_against_oracle():
    """M=1e6, mu=10, a=0.5, p0=8, e0=0.2, T=0.25 yr, dt=10 s, n=1..30: 788,953 samples."""
    pars = dict(BASE)
    pars["length"] = int(0.25 * O.YEAR / 10.0)
    m = E.front_end(pars)
    t, hI, hII = E.genwave(pars, m, 30)
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    to, oI, oII, ip, ib = O.oracle_genwave(pars, mt, 30)
    assert np.array_equal(t, to)
    mm = mismatch(hI, hII, oI, oII)
    assert mm < 1e-6, mm
    assert _maxrel(hI, oI) < 1e-4


def test_distance_scaling_is_exact_linear():
    """h is proportional to 1/D (zeta = mu/D): a size-independent check on long sources."""
    rng = np.random.default_rng(5)
    params = []
    for _ in range(3):
        p = dict(BASE)
        p.update(e=float(rng.uniform(0.1, 0.4)), p=float(rng.uniform(9, 12)), length=int(rng.integers(200000, 400000)))
        params.append(p)
    params2 = [dict(p, D=2.0 * p["D"]) for p in params]
    outs = []
    for ps in (params, params2):
        wb = E.WaveBatch(0)
        hI, hII, off, st = wb.generate_host(ps, nmodes=12)
        assert np.all(st == 0)
        outs.append((hI, hII))
    np.testing.assert_allclose(outs[1][0] * 2.0, outs[0][0], rtol=1e-12, atol=1e-40)
    np.testing.assert_allclose(outs[1][1] * 2.0, outs[0][1], rtol=1e-12, atol=1e-40)


def test_invalid_source_raises_value_error():
    p = dict(BASE)
    p.update(e=-0.1)
    with pytest.raises(AAKValueError):
        E.wave(p)


def test_lookback_wait_gives_up_and_device_stays_usable():
    """The phase scan's bounded look-back wait: on a flag that nothing sets it
    gives up after about a millisecond of SM clocks and reports it; kernels
    launched afterwards run normally."""
    from emri_kludge_suite_b200._lib import lib
    assert lib().aak_selftest_lookback_timeout(2_000_000) == 0
    pars = dict(BASE)
    pars["length"] = 5000
    m = E.front_end(pars)
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    t, hI, hII = E.genwave(pars, m, 30)
    to, oI, oII, _, _ = O.oracle_genwave(pars, mt, 30)
    assert mismatch(hI, hII, oI, oII) < 1e-10


def test_lookback_chains_forward_and_backward_report_no_timeout():
    """Batches with forward (t = 0 at the start) and backward (t = 0 at the
    plunge) phase chains, both precisions and the graph replay: the device
    status stays clear and the replay equals the direct launch."""
    names = golden_names()
    gs = [load_golden(n) for n in names]
    assert any(g["pars"]["backint"] for g in gs)
    wb = E.WaveBatch(0)
    wb.plan([g["pars"] for g in gs], nmodes=[int(g["nmodes"]) for g in gs], mapped=[golden_mapped(g) for g in gs])
    assert np.all(wb.status == 0)
    N = wb.total_samples
    wb.upload()
    out = {}
    for prec in (0, 1):
        a = torch.zeros(N, dtype=torch.float64, device="cuda")
        b = torch.zeros_like(a)
        wb.run(a.data_ptr(), b.data_ptr(), precision=prec)
        a2 = torch.zeros_like(a)
        b2 = torch.zeros_like(a)
        wb.run_graph(a2.data_ptr(), b2.data_ptr(), precision=prec)
        torch.cuda.synchronize()
        assert torch.equal(a, a2) and torch.equal(b, b2)
        out[prec] = (a.cpu().numpy(), b.cpu().numpy())
    assert wb.device_status() == 0
    o = wb.offsets
    for s in range(len(gs)):
        sl = slice(o[s], o[s + 1])
        assert mismatch(out[1][0][sl], out[1][1][sl], out[0][0][sl], out[0][1][sl]) < 1e-6


def test_backward_chain_full_length_against_oracle():
    """backint with the plunge inside the window: t = 0 at sample 388,582 of
    400,000 (dt = 100 s), so ~380 tiles chain backward and ~11 forward."""
    pars = dict(load_golden("plunge_backint")["pars"])
    pars.update(length=400000, T=400000 * pars["dt"] / O.YEAR, p=7.0)
    m = E.front_end(pars)
    t, hI, hII = E.genwave(pars, m, 30)
    mt = O.MappedTrajectory(m.steps, m.e_traj, m.v_map, m.M_map, m.s_map, m.dt_map, m.Phi0, 2)
    to, oI, oII, ip, ib = O.oracle_genwave(pars, mt, 30)
    assert np.array_equal(t, to)
    assert t[1] < 0.0 < t[-1]
    mm = mismatch(hI, hII, oI, oII)
    assert mm < 1e-6, mm
    assert _maxrel(hI, oI) < 1e-4


@pytest.mark.parametrize("precision", [0, 1])
def test_streamed_host_batch_matches_device_batch(precision):
    """aak_wave_batch_host on 40 sources (planned on host threads while groups
    of finished sources are uploaded, generated and copied back) equals plan +
    upload + run into device buffers, and leaves the context with the whole
    batch's plan."""
    rng = np.random.default_rng(11)
    params = []
    for _ in range(40):
        p = dict(BASE)
        p.update(e=float(rng.uniform(0.1, 0.4)), p=float(rng.uniform(9, 12)), length=int(rng.integers(5000, 60000)),
                 iota=float(rng.uniform(0.2, 1.3)), phi_S=float(rng.uniform(0, 6)), mu=float(rng.uniform(5, 60)))
        params.append(p)
    params[7] = dict(params[7], e=-0.2)  # one invalid source: zeros and a status
    wh = E.WaveBatch(0)
    wh.set_precision(precision)
    hI = hII = None
    for _ in range(2):  # twice: the second call reuses the contexts' buffers
        hI, hII, off, st = wh.generate_host(params, nmodes=20)
    assert st[7] != 0 and np.all(np.delete(st, 7) == 0)
    assert np.all(hI[off[7]:off[8]] == 0.0)
    assert np.array_equal(wh.offsets, off) and np.array_equal(wh.status, st)
    wd = E.WaveBatch(0)
    wd.plan(params, nmodes=20)
    assert np.array_equal(wd.offsets, off) and np.array_equal(wd.i_plunge, wh.i_plunge)
    N = wd.total_samples
    a = torch.zeros(N, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    wd.upload()
    wd.run(a.data_ptr(), b.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    a, b = a.cpu().numpy(), b.cpu().numpy()
    scale = max(np.abs(a).max(), np.abs(b).max())
    assert np.max(np.abs(hI - a)) <= 1e-13 * scale
    assert np.max(np.abs(hII - b)) <= 1e-13 * scale
