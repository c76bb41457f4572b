"""aak_batch_run_noalloc: the allocation-free entry point.

It serves callers that cannot call cudaMalloc (their device memory belongs to
a host framework or a pre-reserved pool).  This test plays such a caller: it
owns every device buffer (allocated here through torch), calls the entry
point through the C ABI twice in a row, and compares each result with the
regular aak_batch_run on the same batch.  The file is named so that pytest
collects it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200 import _lib  # noqa: E402


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


def test_noalloc_matches_batch_run_on_two_calls():
    L = _lib.lib()
    wb = _planned_batch()
    N = wb.total_samples
    # the regular entry point (context-owned device buffers)
    ref_I = torch.zeros(N, dtype=torch.float64, device="cuda")
    ref_II = torch.zeros_like(ref_I)
    wb.upload()
    wb.run(ref_I.data_ptr(), ref_II.data_ptr())
    torch.cuda.synchronize()
    ref_I, ref_II = ref_I.cpu().numpy(), ref_II.cpu().numpy()

    need = ctypes.c_int64(0)
    assert L.aak_batch_run_noalloc(wb._ctx, None, 0, ctypes.byref(need), None, None, None) == 0
    assert need.value > 0
    # caller-owned buffers; 256-byte aligned plan buffer
    plan = torch.empty(int(need.value) + 256, dtype=torch.uint8, device="cuda")
    base = (plan.data_ptr() + 255) // 256 * 256
    for call in range(2):
        hI = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
        hII = torch.full((N,), float("nan"), dtype=torch.float64, device="cuda")
        st = L.aak_batch_run_noalloc(wb._ctx, ctypes.c_void_p(base), need.value, None, ctypes.c_void_p(hI.data_ptr()),
                                     ctypes.c_void_p(hII.data_ptr()), None)
        assert st == 0, _lib.STATUS_NAMES.get(st)
        torch.cuda.synchronize()
        a, b = hI.cpu().numpy(), hII.cpu().numpy()
        scale = np.abs(ref_I).max()
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(b)), call
        assert np.abs(a - ref_I).max() <= 1e-12 * scale, call
        assert np.abs(b - ref_II).max() <= 1e-12 * scale, call


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
