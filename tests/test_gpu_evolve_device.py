"""The coarse AK evolution on the GPU (aak_ctx_set_evolve_device): plans and
waveforms against the host's grouped recurrences on the same sources."""
import numpy as np
import pytest

from conftest import mismatch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.workloads import NMODES, SEED, config1  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _run(wb):
    N = wb.total_samples
    a = torch.zeros(N, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    wb.upload()
    wb.run(a.data_ptr(), b.data_ptr())
    torch.cuda.synchronize()
    return a.cpu().numpy(), b.cpu().numpy()


def test_device_evolution_matches_host_planning():
    src, _ = config1(SEED, 24)
    src = [dict(p, length=min(int(p["length"]), 400_000)) for p in src]
    src[3] = dict(src[3], backint=True)  # a backward extension after the device pass
    host = E.WaveBatch(0)
    host.plan(src, nmodes=NMODES)
    dev = E.WaveBatch(0)
    dev.set_evolve_device(True)
    dev.plan(src, nmodes=NMODES)
    ms = dev.plan_ms()
    assert ms["total"] > 0 and ms["device_evolution"] > 0
    assert np.array_equal(host.status, dev.status)
    assert np.array_equal(host.offsets, dev.offsets)
    assert np.array_equal(host.i_plunge, dev.i_plunge) and np.array_equal(host.i_buffer, dev.i_buffer)
    hI, hII = _run(host)
    dI, dII = _run(dev)
    o = host.offsets
    worst_mm, worst_rel = 0.0, 0.0
    for s in range(len(src)):
        sl = slice(o[s], o[s + 1])
        if host.status[s] != 0:
            continue
        worst_mm = max(worst_mm, mismatch(hI[sl], hII[sl], dI[sl], dII[sl]))
        scale = max(np.abs(hI[sl]).max(), np.abs(hII[sl]).max())
        worst_rel = max(worst_rel, max(np.abs(hI[sl] - dI[sl]).max(), np.abs(hII[sl] - dII[sl]).max()) / scale)
    print("device vs host evolution: max mismatch", worst_mm, "max |dh|/max|h|", worst_rel, "plan ms", ms)
    # the recurrences differ only where log() rounds differently (about 1e-16 per step)
    assert worst_mm <= 1e-10 and worst_rel <= 1e-6
