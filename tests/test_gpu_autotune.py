"""The autotuner of the waveform stage's launch shape (aak_ctx_autotune):
every candidate gives the same waveforms, the fastest is kept, and the
tuning-cache file is written and read back."""
import os

import numpy as np
import pytest

from conftest import golden_mapped, golden_names, load_golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _batch():
    gs = [load_golden(n) for n in golden_names()]
    wb = E.WaveBatch(0)
    wb.plan([g["pars"] for g in gs], nmodes=[int(g["nmodes"]) for g in gs], mapped=[golden_mapped(g) for g in gs])
    wb.upload()
    return wb


@pytest.mark.parametrize("precision", [0, 1])
def test_every_launch_shape_gives_the_same_waveforms(precision):
    wb = _batch()
    N = wb.total_samples
    ref = None
    for v in range(6):
        a = torch.zeros(N, dtype=torch.float64, device="cuda")
        b = torch.zeros_like(a)
        wb.set_variant(precision, v)
        wb.run(a.data_ptr(), b.data_ptr(), precision=precision)
        torch.cuda.synchronize()
        x = np.concatenate([a.cpu().numpy(), b.cpu().numpy()])
        if ref is None:
            ref = x
        else:
            # the same algorithm and tables in every shape; the instantiations
            # may contract multiply-adds differently, so they agree to the
            # rounding of their arithmetic: FP64, or the FP32 harmonic sums
            tol = 1e-10 if precision == 0 else 1e-5
            assert np.abs(x - ref).max() <= tol * np.abs(ref).max(), (v, np.abs(x - ref).max() / np.abs(ref).max())
    assert wb.device_status() == 0


def test_autotune_keeps_the_fastest_and_uses_its_cache(tmp_path):
    wb = _batch()
    N = wb.total_samples
    a = torch.zeros(N, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    cache = str(tmp_path / "tune.txt")
    v, ms = wb.autotune(a.data_ptr(), b.data_ptr(), precision=1, cache_path=cache)
    assert all(m > 0 for m in ms) and ms[v] == min(ms)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and int(lines[0].split()[1]) == v
    v2, ms2 = wb.autotune(a.data_ptr(), b.data_ptr(), precision=1, cache_path=cache)
    assert v2 == v and all(m == -1.0 for m in ms2)  # read from the cache, nothing timed
    assert len(open(cache).read().splitlines()) == 1
    assert os.path.getsize(cache) > 0


def test_template_batches_take_every_launch_shape():
    """GPUAAK.set_variant / autotune (aak_gpu_set_variant): likelihood batches
    give the same inner products with every launch shape of the template
    waveform stage (FP64 to 1e-9, split with the FP32 transform to 1e-5 of
    <h|h>), and autotune keeps the fastest candidate."""
    from emri_kludge_suite_b200.gpuAAK import GPUAAK
    from test_gpu_likelihood import DT, INJ, LENGTH, _oracle_wave, _weights

    w1, w2 = _weights()
    dI, dII = _oracle_wave(INJ)  # data: the injection's oracle waveform, no noise
    g = GPUAAK(1.0, 100, LENGTH, 100.0, DT, True, False)
    g.input_data(np.fft.rfft(dI) * w1, np.fft.rfft(dII) * w2, w1, w2)
    rng = np.random.default_rng(3)
    X = np.tile(INJ, (6, 1))
    X[:, 2] *= 1 + 1e-4 * rng.standard_normal(6)
    X[:, 6:11] += 1e-2 * rng.standard_normal((6, 5))
    for precision, tol in ((0, 1e-9), (2, 1e-5)):
        g.set_precision(precision)
        kp = 0 if precision == 0 else 1
        ref = None
        for v in range(GPUAAK.NUM_VARIANTS):
            g.set_variant(kp, v)
            out = g.likelihood_batch(X, max_batch=4)
            if ref is None:
                ref = out
            assert np.abs(out - ref).max() <= tol * ref[:, 1].max(), (precision, v)
        best, ms = g.autotune(X, max_batch=4)
        assert len(ms) == GPUAAK.NUM_VARIANTS and 0 <= best < GPUAAK.NUM_VARIANTS
        assert ms[best] == min(ms)
        assert np.abs(g.likelihood_batch(X, max_batch=4) - ref).max() <= tol * ref[:, 1].max()
    g.set_precision(0)
