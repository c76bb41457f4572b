"""Learned ParMap warm start, host side: the separatrix search, the seeded
point/label generator, the warm-vs-plain solver and the CPU oracle of the
network (pinned against finite differences and BF16 rounding cases)."""
import math

import numpy as np
import pytest

from oracle import mlp_oracle as O  # noqa: E402

from emri_kludge_suite_b200 import parmap_mlp as P  # noqa: E402


def test_separatrix_schwarzschild_is_6_plus_2e():
    # a = 0: p_sep = 6 + 2e for every inclination (Cutler, Kennefick & Poisson 1994)
    for e, iota in ((0.1, 0.3), (0.5, 1.2), (0.69, 2.8)):
        assert abs(P.separatrix(e, iota, 0.0) - (6.0 + 2.0 * e)) < 2e-6


def test_separatrix_equatorial_circular_limit_is_isco():
    # e -> 0, iota = 0: the prograde ISCO (Bardeen, Press & Teukolsky 1972)
    a = 0.7
    z1 = 1 + (1 - a * a) ** (1 / 3) * ((1 + a) ** (1 / 3) + (1 - a) ** (1 / 3))
    z2 = math.sqrt(3 * a * a + z1 * z1)
    isco = 3 + z2 - math.sqrt((3 - z1) * (3 + z1 + 2 * z2))
    assert abs(P.separatrix(1e-4, 0.0, a) - isco) < 2e-3


def test_dataset_is_seeded_and_thread_independent():
    a = P.make_dataset(256, seed=11, nthreads=1)
    b = P.make_dataset(256, seed=11, nthreads=4)
    c = P.make_dataset(128, seed=11, first_index=128, nthreads=3)
    assert np.array_equal(a["x"], b["x"]) and np.array_equal(a["iters"], b["iters"])
    assert np.array_equal(a["x"][128:], c["x"])
    d = P.make_dataset(256, seed=12)
    assert not np.array_equal(a["x"], d["x"])


def test_dataset_distribution_and_labels():
    d = P.make_dataset(2048, seed=5)
    x = d["x"]
    assert np.all((x[:, 1] >= 1e-3) & (x[:, 1] < 0.7))
    assert np.all((x[:, 2] >= 0) & (x[:, 2] <= math.pi))
    assert np.all((x[:, 3] >= 0) & (x[:, 3] < 0.95))
    assert np.all(x[:, 0] <= 20.0)
    for i in range(0, 2048, 97):  # p >= p_sep + 0.1
        assert x[i, 0] >= P.separatrix(x[i, 1], x[i, 2], x[i, 3]) + 0.1 - 1e-6
    v = d["valid"]
    assert v.mean() > 0.95
    # the labels are fixed points of the solver: starting there only polishes
    # at rounding level (the solve iterates until the step stalls)
    s = P.solve_batch(x[v], d["omega"][v], d["y"][v])
    assert np.all(s["fallback"] == 0)
    assert np.median(s["iters"]) <= 1 and np.max(s["iters"]) <= 8
    assert np.max(np.abs(s["y"] - d["y"][v])) < 1e-12
    assert np.max(s["residual"]) < 1e-6


def test_warm_solve_falls_back_from_a_bad_guess():
    d = P.make_dataset(64, seed=9)
    v = d["valid"]
    x, om, y = d["x"][v], d["omega"][v], d["y"][v]
    bad = y + np.array([0.3, 0.5, 0.4])  # far from the root
    s = P.solve_batch(x, om, bad)
    cold = P.solve_batch(x, om, None)
    # where the warm solve is refused it is redone from the plain guess
    fb = s["fallback"] == 1
    assert fb.any()
    assert np.array_equal(s["y"][fb], cold["y"][fb])
    assert np.max(s["residual"]) < 1e-6


def test_bf16_rounding_cases():
    one = 1.0
    ulp = 2.0**-7  # BF16 spacing at 1
    assert O.bf16(one + ulp / 2) == one  # tie -> even
    assert O.bf16(one + 3 * ulp / 2) == one + 2 * ulp  # tie -> even (up)
    assert O.bf16(one + ulp / 2 + 2.0**-20) == one + ulp
    assert O.bf16(-3.0) == -3.0
    assert O.bf16(0.0) == 0.0


def _small_net(seed):
    rng = np.random.default_rng(seed)
    p = P.init_params(seed).astype(np.float64)
    norm = {"in_shift": np.array([0.3, 0.35, 0.0, 0.47]), "in_scale": np.array([8.0, 3.0, 1.4, 3.6]),
            "out_shift": np.array([1.02, 1.05, 0.01]), "out_scale": np.array([0.03, 0.08, 0.04])}
    x = np.stack([rng.uniform(4, 20, 16), rng.uniform(0.01, 0.7, 16), rng.uniform(0, math.pi, 16),
                  rng.uniform(0, 0.95, 16)], axis=1)
    y = np.stack([rng.normal(1.02, 0.03, 16), rng.normal(1.05, 0.08, 16), rng.normal(0.0, 0.04, 16)], axis=1)
    return p, norm, x, y


def test_oracle_gradient_matches_finite_differences():
    p, norm, x, y = _small_net(3)
    loss, g = O.loss_and_grad(p, x, y, norm, quantize=False)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(np.arange(o, o + int(np.prod(s))), min(6, int(np.prod(s))), replace=False)
                          for o, s in O.OFFSETS.values()])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (O.loss_and_grad(pp, x, y, norm, False)[0] - O.loss_and_grad(pm, x, y, norm, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(abs(fd), 1e-3), (i, fd, g[i])


def test_oracle_quantized_is_close_to_exact():
    p, norm, x, y = _small_net(4)
    lq, gq = O.loss_and_grad(p, x, y, norm, quantize=True)
    le, ge = O.loss_and_grad(p, x, y, norm, quantize=False)
    assert abs(lq - le) < 0.05 * le
    assert np.linalg.norm(gq - ge) < 0.1 * np.linalg.norm(ge)
