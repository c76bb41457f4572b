"""Learned ParMap warm start on the GPU: the tcgen05 forward and backward
kernels against the CPU oracle (BF16 rounding emulated there), the Adam
update, what a trained network gains over the plain initial guess, and that
the warm-started batch planner yields the same waveforms."""
import numpy as np
import pytest

from conftest import mismatch

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
from oracle import mlp_oracle as O  # noqa: E402

import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200 import parmap_mlp as P  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _model(seed, n):
    d = P.make_dataset(n, seed)
    x, y = d["x"][d["valid"]], d["y"][d["valid"]]
    m = P.ParMapMLP(0, seed=seed)
    m.fit_norm(x, y)
    return m, x, y


def _norm64(m):
    return {k: np.asarray(v, dtype=np.float64) for k, v in m.norm.items()}


def _f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def test_forward_matches_oracle():
    m, x, _ = _model(21, 3000)  # 2,9xx rows: a ragged last tile
    got = m.predict(x)
    ref = O.predict(m.params().astype(np.float64), _f32(x), _norm64(m))
    err = np.abs(got - ref) / m.norm["out_scale"]  # normalised output units
    print(f"forward vs oracle: median {np.median(err):.2e}, max {err.max():.2e}")
    assert np.median(err) < 1e-4
    assert err.max() < 5e-3
    exact = O.predict(m.params().astype(np.float64), _f32(x), _norm64(m), quantize=False)
    assert np.max(np.abs(got - exact) / m.norm["out_scale"]) < 0.1  # BF16 network ~ FP64 network


@pytest.mark.parametrize("n", [512, 1000])
def test_gradients_match_oracle(n):
    m, x, y = _model(22, 1200)
    x, y = x[:n], y[:n]
    xd = torch.tensor(x.astype(np.float32), device="cuda")
    yd = torch.tensor(y.astype(np.float32), device="cuda")
    grad = torch.zeros(P.n_params(), dtype=torch.float32, device="cuda")
    loss = m.gradients_device(xd.data_ptr(), yd.data_ptr(), n, grad.data_ptr())
    g = grad.cpu().numpy().astype(np.float64)
    lref, gref = O.loss_and_grad(m.params().astype(np.float64), _f32(x), _f32(y), _norm64(m))
    assert abs(loss - lref) <= 1e-4 * lref
    worst = 0.0
    for k, (o, s) in O.OFFSETS.items():
        sz = int(np.prod(s))
        rel = np.linalg.norm(g[o:o + sz] - gref[o:o + sz]) / np.linalg.norm(gref[o:o + sz])
        worst = max(worst, rel)
        assert rel < 2e-2, (k, rel)
    print(f"n={n}: loss {loss:.6e} vs {lref:.6e}; worst per-tensor relative gradient error {worst:.2e}")
    assert np.linalg.norm(g - gref) < 5e-3 * np.linalg.norm(gref)


def test_permuted_rows_and_adam_step():
    m, x, y = _model(23, 1500)
    rng = np.random.default_rng(0)
    n = 700
    perm = rng.permutation(x.shape[0])[:n].astype(np.int32)
    xd = torch.tensor(x.astype(np.float32), device="cuda")
    yd = torch.tensor(y.astype(np.float32), device="cuda")
    pd = torch.tensor(perm, device="cuda")
    grad = torch.zeros(P.n_params(), dtype=torch.float32, device="cuda")
    m.gradients_device(xd.data_ptr(), yd.data_ptr(), n, grad.data_ptr(), perm_ptr=pd.data_ptr())
    g = grad.cpu().numpy().astype(np.float64)
    _, gref = O.loss_and_grad(m.params().astype(np.float64), _f32(x[perm]), _f32(y[perm]), _norm64(m))
    assert np.linalg.norm(g - gref) < 5e-3 * np.linalg.norm(gref)
    p0 = m.params().astype(np.float64)
    m.train_step_device(xd.data_ptr(), yd.data_ptr(), n, 1e-3, perm_ptr=pd.data_ptr())
    p1 = m.params().astype(np.float64)
    expect, _, _ = O.adam_step(p0, g, np.zeros_like(g), np.zeros_like(g), 1, 1e-3)
    assert np.max(np.abs(p1 - expect)) < 1e-6


def test_trained_warm_start_saves_newton_iterations():
    train = P.make_dataset(1 << 17, seed=31)
    held = P.make_dataset(1 << 12, seed=32)
    m = P.ParMapMLP(0, seed=1)
    hist = m.train(train["x"][train["valid"]], train["y"][train["valid"]], epochs=40, batch=8192, lr=1e-2)
    assert hist["loss"][-1] < 0.05 * hist["loss"][0]
    ev = P.evaluate(m, held)
    print({k: ev[k] for k in ("iters_cold", "iters_warm", "iters_to_tol_cold", "iters_to_tol_warm", "fallback_rate",
                              "warm_vs_cold_solution_max_rel")})
    # iterations to the reference's stopping test |f|_1 < 1e-6, and in total
    # (the solve then polishes for about two more iterations either way)
    assert ev["iters_to_tol_warm"]["mean"] < 0.75 * ev["iters_to_tol_cold"]["mean"]
    assert ev["iters_warm"]["mean"] < 0.9 * ev["iters_cold"]["mean"]
    assert ev["fallback_rate"] < 0.01
    assert ev["failed_warm"] == 0
    assert ev["residual_abs_warm_max"] < 1e-6
    # both solves end at the same root, to the conditioning of the map
    assert ev["warm_vs_cold_solution_max_rel"] < 1e-9
    # the warm-started batch planner: same waveforms, fewer iterations
    rng = np.random.default_rng(7)
    YEAR = 31558149.8
    srcs = []
    for _ in range(6):
        M, mu, e0 = 10 ** rng.uniform(5.5, 6.5), rng.uniform(5, 50), rng.uniform(0.1, 0.5)
        n = int(rng.integers(20000, 60000))
        rr = (M * 4.925490947641267e-06) ** 2 / (mu * 4.925490947641267e-06)
        p0 = ((10 + 3 * e0) ** 4 + 102.4 * n * 10.0 / rr) ** 0.25
        srcs.append(dict(backint=False, LISA=True, length=n, dt=10.0, p=p0, T=n * 10.0 / YEAR, f=0.0, T_fit=1.0, mu=mu,
                         M=M, s=rng.uniform(0, 0.9), e=e0, iota=rng.uniform(0.2, 1.3), gamma=1.0, psi=0.5,
                         theta_S=0.7, phi_S=1.1, theta_K=1.9, phi_K=0.4, alpha=0.3, D=1.0))
    out = {}
    for warm in (False, True):
        wb = E.WaveBatch(0)
        if warm:
            wb.set_parmap_model(m)
        wb.plan(srcs, nmodes=[30] * len(srcs))
        assert np.all(wb.status == 0)
        hI = torch.zeros(wb.total_samples, dtype=torch.float64, device="cuda")
        hII = torch.zeros_like(hI)
        wb.upload()
        wb.run(hI.data_ptr(), hII.data_ptr())
        torch.cuda.synchronize()
        out[warm] = (hI.cpu().numpy(), hII.cpu().numpy(), wb.newton_stats())
    o = wb.offsets
    for s in range(len(srcs)):
        sl = slice(o[s], o[s + 1])
        mm = mismatch(out[True][0][sl], out[True][1][sl], out[False][0][sl], out[False][1][sl])
        assert mm < 1e-9, (s, mm)
    cold_it, warm_it = out[False][2]["iterations"], out[True][2]["iterations"]
    print(f"batch planner Newton iterations: plain {cold_it}, warm {warm_it}, fallbacks {out[True][2]['fallbacks']}")
    assert warm_it < cold_it
