"""aak_batch_run_noalloc: the allocation-free entry point.

It serves callers that cannot call cudaMalloc (their device memory belongs to
a host framework or a pre-reserved pool).  This test plays such a caller: it
owns every device buffer (allocated here through torch), calls the entry
point through the C ABI twice in a row in each precision, and compares each
result with the regular aak_batch_run on the same batch.  The file is named so
that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200 import _lib  # noqa: E402

# agreement with aak_batch_run, relative to the largest |h| of the batch: the
# same kernels on the same plan (the look-back sums may regroup, which moves a
# phase carry at the 1e-32 level of its double-double)
TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _planned_batch():
    names = golden_names()
    gs = [load_golden(n) for n in names]
    wb = E.WaveBatch(0)
    wb.plan([g["pars"] for g in gs], nmodes=[int(g["nmodes"]) for g in gs], mapped=[golden_mapped(g) for g in gs])
    assert np.all(wb.status == 0)
    return wb


def _regular(wb, precision):
    N = wb.total_samples
    a = torch.zeros(N, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    wb.upload()
    wb.run(a.data_ptr(), b.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    return a.cpu().numpy(), b.cpu().numpy()


def _noalloc(L, wb, base, need, N):
    hI = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
    hII = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
    st = L.aak_batch_run_noalloc(wb._ctx, ctypes.c_void_p(base), need, None, ctypes.c_void_p(hI.data_ptr()),
                                 ctypes.c_void_p(hII.data_ptr()), None)
    assert st == 0, _lib.STATUS_NAMES.get(st)
    torch.cuda.synchronize()
    return hI.cpu().numpy(), hII.cpu().numpy()


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_batch_run_on_two_calls(precision):
    L = _lib.lib()
    wb = _planned_batch()
    N = wb.total_samples
    ref_I, ref_II = _regular(wb, precision)

    need = ctypes.c_int64(0)
    assert L.aak_batch_run_noalloc(wb._ctx, None, 0, ctypes.byref(need), None, None, None) == 0
    assert need.value > 0
    # caller-owned buffers; 256-byte aligned plan buffer
    plan = torch.empty(int(need.value) + 256, dtype=torch.uint8, device="cuda")
    base = (plan.data_ptr() + 255) // 256 * 256
    wb.set_precision(precision)
    scale = np.abs(ref_I).max()
    for call in range(2):
        a, b = _noalloc(L, wb, base, need.value, N)
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(b)), call
        assert np.abs(a - ref_I).max() <= TOL * scale, call
        assert np.abs(b - ref_II).max() <= TOL * scale, call
    assert wb.device_status() == 0
    wb.set_precision(0)


def test_noalloc_call_after_a_wait_gave_up():
    """A call whose look-back waits give up at once (a one-clock bound) leaves
    the report word set; the next call with the normal bound is unaffected and
    matches aak_batch_run, and the report is read once."""
    L = _lib.lib()
    wb = _planned_batch()
    N = wb.total_samples
    ref_I, ref_II = _regular(wb, 0)
    need = ctypes.c_int64(0)
    L.aak_batch_run_noalloc(wb._ctx, None, 0, ctypes.byref(need), None, None, None)
    plan = torch.empty(int(need.value) + 256, dtype=torch.uint8, device="cuda")
    base = (plan.data_ptr() + 255) // 256 * 256
    assert wb.device_status() == 0
    assert L.aak_ctx_set_lookback_bound(wb._ctx, 1) == 0
    _noalloc(L, wb, base, need.value, N)  # results not checked: the carries may be zero
    assert L.aak_ctx_set_lookback_bound(wb._ctx, 0) == 0
    a, b = _noalloc(L, wb, base, need.value, N)
    scale = np.abs(ref_I).max()
    assert np.abs(a - ref_I).max() <= TOL * scale
    assert np.abs(b - ref_II).max() <= TOL * scale
    first = wb.device_status()  # the give-up of the first call, if one of its waits had to wait at all
    assert first in (0, 9)  # AAK_OK or AAK_ERR_DEVICE_TIMEOUT
    assert wb.device_status() == 0


def test_noalloc_rejects_small_buffer_and_large_batch():
    L = _lib.lib()
    wb = _planned_batch()
    need = ctypes.c_int64(0)
    L.aak_batch_run_noalloc(wb._ctx, None, 0, ctypes.byref(need), None, None, None)
    buf = torch.empty(int(need.value), dtype=torch.uint8, device="cuda")
    out = torch.empty(wb.total_samples, dtype=torch.float64, device="cuda")
    st = L.aak_batch_run_noalloc(wb._ctx, ctypes.c_void_p(buf.data_ptr()), need.value - 256, None,
                                 ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(out.data_ptr()), None)
    assert st == 8  # AAK_ERR_CAPACITY
    # more than 32768 tiles of 1024 samples
    base = dict(load_golden("cfg0_short")["pars"])
    big = []
    for k in range(9):
        p = dict(base)
        p["length"] = 3_800_000
        p["T"] = p["length"] * p["dt"] / 31558149.8
        big.append(p)
    wb2 = E.WaveBatch(0)
    wb2.plan(big, nmodes=4)
    assert wb2.total_samples > 32768 * 1024
    L.aak_batch_run_noalloc(wb2._ctx, None, 0, ctypes.byref(need), None, None, None)
    buf2 = torch.empty(int(need.value), dtype=torch.uint8, device="cuda")
    st = L.aak_batch_run_noalloc(wb2._ctx, ctypes.c_void_p(buf2.data_ptr()), need.value, None,
                                 ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(out.data_ptr()), None)
    assert st == 8
