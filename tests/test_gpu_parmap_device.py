"""The batched device solve of the Kerr->AK map (aak_ctx_set_parmap_device):
plans, waveforms and likelihoods equal the host-solved ones bit for bit, with
the plain guess and with a warm start (an untrained network, so that many
points take the fallback to the plain guess).  Calls go through the C ABI."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200 import parmap_mlp as P  # noqa: E402
from emri_kludge_suite_b200.gpuAAK import GPUAAK  # noqa: E402
from emri_kludge_suite_b200.workloads import config1  # noqa: E402

FID = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.8, 2.0, 1.0])


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _sources(n=24):
    src, _ = config1(11, 64)
    out = []
    for p in src[:n]:
        q = dict(p)
        q["length"] = min(int(p["length"]), 200000)
        out.append(q)
    out[5] = dict(out[5], e=-0.2)  # invalid: the same status either way
    return out


def _run(params, device_map, model=None):
    wb = E.WaveBatch(0)
    if model is not None:
        wb.set_parmap_model(model)
    wb.set_parmap_device(device_map)
    wb.plan(params, nmodes=12)
    N = wb.total_samples
    hI = torch.zeros(N, dtype=torch.float64, device="cuda")
    hII = torch.zeros_like(hI)
    wb.upload()
    wb.run(hI.data_ptr(), hII.data_ptr())
    torch.cuda.synchronize()
    return wb, hI.cpu().numpy(), hII.cpu().numpy()


def _untrained_model():
    d = P.make_dataset(1 << 12, 5)
    m = P.ParMapMLP(0, seed=3)
    m.fit_norm(d["x"][d["valid"]], d["y"][d["valid"]])
    return m


@pytest.mark.parametrize("warm", [False, True])
def test_device_map_equals_host_map(warm):
    params = _sources()
    model = _untrained_model() if warm else None
    a, aI, aII = _run(params, False, model)
    b, bI, bII = _run(params, True, model)
    assert np.array_equal(a.status, b.status) and a.status[5] != 0
    assert np.array_equal(a.offsets, b.offsets) and np.array_equal(a.i_plunge, b.i_plunge)
    assert a.newton_stats() == b.newton_stats()
    if warm:
        assert b.newton_stats()["fallbacks"] > 0
    assert np.array_equal(aI, bI) and np.array_equal(aII, bII)


def test_likelihood_batch_with_device_map_is_unchanged():
    rng = np.random.default_rng(2)
    X = np.tile(FID, (40, 1))
    X[:, 2] *= 1 + 1e-3 * rng.standard_normal(40)
    X[:, 6:11] += 1e-1 * rng.standard_normal((40, 5))
    n = 40000
    w = np.ones(n // 2 + 1)
    d = np.zeros(n // 2 + 1, dtype=np.complex128) + 1e-22
    outs = []
    for dev in (False, True):
        g = GPUAAK(1.0, 100, n, 100.0, 10.0, True, False)
        g.input_data(d, d, w, w)
        g.set_parmap_device(dev)
        outs.append(g.likelihood_batch(X, max_batch=16))
    assert np.array_equal(outs[0], outs[1])
