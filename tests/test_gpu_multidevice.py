"""The one-process, several-device wrappers of shard.py (MultiDeviceWaveBatch,
MultiDeviceGPUAAK) against one device: the LPT split, the per-device host
threads and the reassembly in the caller's order.  With one GPU per run the
"devices" are two contexts on device 0, driven from two host threads at once;
each launch's waits (the phase scan's look-back) are on tiles of that launch
only, taken from its own work queue, so two launches in flight on one GPU do
not wait on each other."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.gpuAAK import GPUAAK  # noqa: E402
from emri_kludge_suite_b200.shard import MultiDeviceGPUAAK, MultiDeviceWaveBatch  # noqa: E402
from emri_kludge_suite_b200.workloads import config1  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_split_wave_batch_equals_one_device():
    src, _ = config1(9, 64)
    params = []
    for p in src:
        q = dict(p)
        q["length"] = min(int(p["length"]), 200000)
        params.append(q)
    params[4] = dict(params[4], e=-0.2)  # invalid: reported in its place
    one = E.WaveBatch(0)
    hI, hII, offs, st = one.generate_host(params, nmodes=30)
    md = MultiDeviceWaveBatch([0, 0])
    mI, mII, moffs, mst = md.generate_host(params, nmodes=30)
    md.close()
    one.close()
    assert st[4] != 0 and np.array_equal(st, mst) and np.array_equal(offs, moffs)
    assert np.array_equal(hI, mI) and np.array_equal(hII, mII)


def test_split_likelihood_and_fisher_batches_equal_one_device():
    from test_gpu_fisher import _rows
    from test_gpu_likelihood import DT, INJ, LENGTH, _oracle_wave, _weights

    w1, w2 = _weights()
    dI, dII = _oracle_wave(INJ)
    D1, D2 = np.fft.rfft(dI) * w1, np.fft.rfft(dII) * w2
    one = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    md = MultiDeviceGPUAAK([0, 0], 1.0, 100, LENGTH, 100.0, DT, True, False)
    one.input_data(D1, D2, w1, w2)
    md.input_data(D1, D2, w1, w2)
    rng = np.random.default_rng(8)
    X = np.tile(INJ, (7, 1))
    X[:, 2] *= 1 + 1e-4 * rng.standard_normal(7)
    X[:, 6:11] += 1e-2 * rng.standard_normal((7, 5))
    a, sa = one.likelihood_batch(X, max_batch=2, return_status=True)
    b, sb = md.likelihood_batch(X, max_batch=2, return_status=True)
    assert np.array_equal(sa, sb) and np.all(sa == 0)
    np.testing.assert_allclose(b, a, rtol=1e-13)
    rows = np.stack([_rows(4, x) for x in X[:3]])
    Ga = one.fisher_gram_batch(rows, 0.5)
    Gb, st = md.fisher_gram_batch(rows, 0.5, return_status=True)
    assert np.all(st == 0)
    assert np.abs(Gb - Ga).max() <= 1e-12 * np.abs(Ga).max()
