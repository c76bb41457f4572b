"""The plain FP64 per-source path (the baseline of the batched paths) agrees
with the batched FP64 path: same trajectory kernels on one-source views, the
harmonic sum evaluated per harmonic with jn() as the reference's CUDA port does."""
import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden, mismatch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_plain_path_matches_batched_fp64():
    gs = [load_golden(n) for n in golden_names()]
    wb = E.WaveBatch(0)
    wb.plan([g["pars"] for g in gs], nmodes=[int(g["nmodes"]) for g in gs], mapped=[golden_mapped(g) for g in gs])
    N = wb.total_samples
    hI = torch.zeros(N, dtype=torch.float64, device="cuda")
    hII = torch.zeros_like(hI)
    pI = torch.full_like(hI, float("nan"))
    pII = torch.full_like(hI, float("nan"))
    traj = torch.zeros(9 * N, dtype=torch.float64, device="cuda")
    wb.upload()
    wb.run(hI.data_ptr(), hII.data_ptr())
    wb.run_plain(pI.data_ptr(), pII.data_ptr(), traj.data_ptr(), N)
    torch.cuda.synchronize()
    a = (hI.cpu().numpy(), hII.cpu().numpy())
    b = (pI.cpu().numpy(), pII.cpu().numpy())
    assert np.all(np.isfinite(b[0])) and np.all(np.isfinite(b[1]))
    o = wb.offsets
    for s in range(wb.nsrc):
        sl = slice(o[s], o[s + 1])
        mm = mismatch(b[0][sl], b[1][sl], a[0][sl], a[1][sl])
        scale = max(np.abs(a[0][sl]).max(), np.abs(a[1][sl]).max())
        rel = max(np.abs(b[0][sl] - a[0][sl]).max(), np.abs(b[1][sl] - a[1][sl]).max()) / scale
        print(f"source {s}: mismatch {mm:.2e}, max|dh|/max|h| {rel:.2e}")
        assert mm < 1e-12
        assert rel < 1e-8
