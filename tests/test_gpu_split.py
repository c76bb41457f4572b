"""Split precision (FP64 phases and angle reductions, FP32 Bessel/trig/response)
against the FP64 path: overlap mismatch <= 1e-6 per source (the bar of the
benchmark's configuration 2) and a bound on max|dh|/max|h|."""
import math

import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden, mismatch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402

YEAR = 31558149.8


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _run(wb, precision):
    N = wb.total_samples
    hI = torch.zeros(N, dtype=torch.float64, device="cuda")
    hII = torch.zeros_like(hI)
    wb.upload()
    wb.run(hI.data_ptr(), hII.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    return hI.cpu().numpy(), hII.cpu().numpy()


def _compare(wb, tol_mm=1e-6, tol_rel=1e-3):
    a = _run(wb, 0)
    b = _run(wb, 1)
    o = wb.offsets
    worst_mm, worst_rel = 0.0, 0.0
    for s in range(wb.nsrc):
        if wb.status[s] != 0:
            continue
        sl = slice(o[s], o[s + 1])
        mm = mismatch(b[0][sl], b[1][sl], a[0][sl], a[1][sl])
        scale = max(np.abs(a[0][sl]).max(), np.abs(a[1][sl]).max())
        rel = max(np.abs(b[0][sl] - a[0][sl]).max(), np.abs(b[1][sl] - a[1][sl]).max()) / scale
        worst_mm, worst_rel = max(worst_mm, mm), max(worst_rel, rel)
        assert mm <= tol_mm, (s, mm)
        assert rel <= tol_rel, (s, rel)
    return worst_mm, worst_rel


def test_split_precision_golden_cases():
    gs = [load_golden(n) for n in golden_names()]
    wb = E.WaveBatch(0)
    wb.plan([g["pars"] for g in gs], nmodes=[int(g["nmodes"]) for g in gs], mapped=[golden_mapped(g) for g in gs])
    mm, rel = _compare(wb)
    print(f"golden: worst mismatch {mm:.2e}, worst max|dh|/max|h| {rel:.2e}")


def _config2_source(rng, length):
    while True:
        M = 10 ** rng.uniform(5, 7)
        mu = rng.uniform(1, 100)
        e0 = rng.uniform(0.05, 0.7)
        cosi = rng.uniform(-1, 1)
        if abs(cosi) < 0.05:
            continue
        rr = (M * 4.925490947641267e-06) ** 2 / (mu * 4.925490947641267e-06)
        p0 = min(max((( 10 + 3 * e0) ** 4 + 102.4 * length * 10.0 / rr) ** 0.25, 9.0), 80.0)
        return dict(backint=False, LISA=True, length=length, dt=10.0, p=p0, T=length * 10.0 / YEAR, f=0.0, T_fit=1.0,
                    mu=mu, M=M, s=rng.uniform(0, 0.95), e=e0, iota=math.acos(cosi), gamma=rng.uniform(0, 6.28),
                    psi=rng.uniform(0, 6.28), theta_S=math.acos(rng.uniform(-1, 1)), phi_S=rng.uniform(0, 6.28),
                    theta_K=math.acos(rng.uniform(-1, 1)), phi_K=rng.uniform(0, 6.28), alpha=rng.uniform(0, 6.28), D=1.0)


def test_split_precision_configuration2_sample():
    rng = np.random.default_rng(20261203 + 2)
    params = [_config2_source(rng, int(rng.integers(100_000, 400_000))) for _ in range(24)]
    nmodes = [min(100, math.ceil(10.0 / (1.0 - p["e"]) ** 1.5)) for p in params]
    wb = E.WaveBatch(0)
    wb.plan(params, nmodes=nmodes)
    assert np.sum(wb.status == 0) >= 20
    mm, rel = _compare(wb)
    print(f"configuration-2 sample: worst mismatch {mm:.2e}, worst max|dh|/max|h| {rel:.2e}")


def test_graph_replay_matches_direct_launches():
    gs = [load_golden(n) for n in golden_names()]
    wb = E.WaveBatch(0)
    wb.plan([g["pars"] for g in gs], nmodes=[int(g["nmodes"]) for g in gs], mapped=[golden_mapped(g) for g in gs])
    for precision in (0, 1):
        ref = _run(wb, precision)
        N = wb.total_samples
        hI = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
        hII = torch.full_like(hI, float("nan"))
        for _ in range(2):  # capture, then replay
            wb.run_graph(hI.data_ptr(), hII.data_ptr(), precision=precision)
            torch.cuda.synchronize()
            assert np.array_equal(hI.cpu().numpy(), ref[0]) and np.array_equal(hII.cpu().numpy(), ref[1])
    # a new upload is picked up by the next replay
    wb.plan([gs[0]["pars"]], nmodes=[int(gs[0]["nmodes"])], mapped=[golden_mapped(gs[0])])
    ref = _run(wb, 1)
    hI = torch.zeros(wb.total_samples, dtype=torch.float64, device="cuda")
    hII = torch.zeros_like(hI)
    wb.run_graph(hI.data_ptr(), hII.data_ptr(), precision=1)
    torch.cuda.synchronize()
    assert np.array_equal(hI.cpu().numpy(), ref[0])
