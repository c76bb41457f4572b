"""Learned warm start of the Kerr -> AK parameter map.

The reference solves, at every coarse inspiral point, a 3 x 3 nonlinear
system for (v_map, M_map, s_map) from the initial guess (1/sqrt(p), M, a)
(ParMap, src/suite/KSParMap.cc:397-440, starting point at :409).  Here a
4 -> 128 -> 128 -> 128 -> 3 SiLU network with BF16 weights and activations and
FP32 accumulation predicts the solution from (p, e, iota, a); the plain
Newton solve then starts from the prediction, stays the judge (|f|_1 < 1e-6)
and is the fallback from the plain guess when a warm solve fails.

* :func:`make_dataset` -- seeded points p ~ U(p_sep + 0.1, 20), e ~ U(0, 0.7),
  iota ~ U(0, pi), a ~ U(0, 0.95) labelled by the plain solve (host threads).
* :class:`ParMapMLP` -- the network on one GPU: tensor-core inference and
  training kernels of libaak_b200.so (forward, backward, Adam).
* :func:`evaluate` -- Newton iterations cold vs warm, residuals, fallbacks.

Outputs are map coordinates y = (v_map sqrt(p), M_map / M, s_map - a).
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from ._lib import check, lib, ptr

LABEL_MASS = 1.0e6


def n_params() -> int:
    return int(lib().aak_mlp_num_params())


def max_train_rows() -> int:
    return int(lib().aak_mlp_max_train_rows())


def separatrix(e: float, iota: float, a: float) -> float:
    """p_sep by bisection on geodesic stability."""
    out = ctypes.c_double()
    check(lib().aak_parmap_separatrix(float(e), float(iota), float(a), ctypes.byref(out)), "aak_parmap_separatrix")
    return out.value


def make_dataset(n: int, seed: int, first_index: int = 0, nthreads: int = 0) -> dict:
    """Points first_index .. first_index + n - 1 of the seeded distribution,
    with Kerr frequencies and plain-solve labels (NaN rows: failed solves)."""
    x = np.zeros((n, 4))
    y = np.zeros((n, 3))
    om = np.zeros((n, 3))
    it = np.zeros(n, dtype=np.int32)
    check(lib().aak_parmap_dataset(int(n), int(seed), int(first_index), int(nthreads), ptr(x), ptr(y), ptr(om),
                                   ptr(it)), "aak_parmap_dataset")
    return {"x": x, "y": y, "omega": om, "iters": it, "valid": label_valid(y, it)}


def label_valid(y: np.ndarray, iters: np.ndarray) -> np.ndarray:
    """Labels usable for training: the plain solve converged to a physical
    root (M_map > 0, v_map sqrt(p) in (0.5, 2), |s_map - a| < 1).  Close to
    the separatrix at high spin the PN frequencies cannot match the Kerr ones
    and the plain solve fails or lands on a spurious root (about 2 % of the
    distribution)."""
    with np.errstate(invalid="ignore"):
        return ((iters >= 0) & np.all(np.isfinite(y), axis=1) & (y[:, 0] > 0.5) & (y[:, 0] < 2.0) & (y[:, 1] > 0.0)
                & (np.abs(y[:, 2]) < 1.0))


def solve_batch(x: np.ndarray, omega: np.ndarray, guess: np.ndarray | None = None, nthreads: int = 0) -> dict:
    """Map solves at M = LABEL_MASS from `guess` (map coordinates) or the plain guess."""
    n = x.shape[0]
    x = np.ascontiguousarray(x, dtype=np.float64)
    omega = np.ascontiguousarray(omega, dtype=np.float64)
    g = None if guess is None else np.ascontiguousarray(guess, dtype=np.float64)
    y = np.zeros((n, 3))
    it = np.zeros(n, dtype=np.int32)
    tol = np.zeros(n, dtype=np.int32)
    res = np.zeros(n)
    gres = np.zeros(n)
    fb = np.zeros(n, dtype=np.int32)
    t0 = time.perf_counter()
    check(lib().aak_parmap_solve_batch(int(n), ptr(x), ptr(omega), ptr(g), int(nthreads), ptr(y), ptr(it), ptr(tol),
                                       ptr(res), ptr(gres) if g is not None else None, ptr(fb)),
          "aak_parmap_solve_batch")
    return {"y": y, "iters": it, "iters_to_tol": tol, "residual": res,
            "guess_residual": gres if g is not None else None, "fallback": fb, "seconds": time.perf_counter() - t0}


def init_params(seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases, seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for fan_in, n_w, n_b in ((4, 128 * 4, 128), (128, 128 * 128, 128), (128, 128 * 128, 128), (128, 3 * 128, 3)):
        b = 1.0 / math.sqrt(fan_in)
        out.append(rng.uniform(-b, b, n_w))
        out.append(rng.uniform(-b, b, n_b))
    p = np.concatenate(out).astype(np.float32)
    assert p.size == n_params()
    return p


def input_features(x: np.ndarray) -> np.ndarray:
    """(1/sqrt(p), e, cos iota, a): the quantities the network is normalised in."""
    return np.stack([1.0 / np.sqrt(x[:, 0]), x[:, 1], np.cos(x[:, 2]), x[:, 3]], axis=1)


class ParMapMLP:
    """The warm-start network on one GPU (handle to ``aak_mlp``)."""

    def __init__(self, device: int = 0, seed: int = 0, params: np.ndarray | None = None):
        self.handle = ctypes.c_void_p()
        check(lib().aak_mlp_create(int(device), ctypes.byref(self.handle)), "aak_mlp_create")
        self.device = device
        self.norm = {"in_shift": np.zeros(4, np.float32), "in_scale": np.ones(4, np.float32),
                     "out_shift": np.zeros(3, np.float32), "out_scale": np.ones(3, np.float32)}
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if self.handle:
            lib().aak_mlp_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters and normalisation
    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != n_params():
            raise ValueError(f"expected {n_params()} parameters, got {p.size}")
        check(lib().aak_mlp_set_params(self.handle, ptr(p)), "aak_mlp_set_params")

    def params(self) -> np.ndarray:
        p = np.zeros(n_params(), dtype=np.float32)
        check(lib().aak_mlp_get_params(self.handle, ptr(p)), "aak_mlp_get_params")
        return p

    def set_norm(self, in_shift, in_scale, out_shift, out_scale):
        n = {"in_shift": np.ascontiguousarray(in_shift, dtype=np.float32),
             "in_scale": np.ascontiguousarray(in_scale, dtype=np.float32),
             "out_shift": np.ascontiguousarray(out_shift, dtype=np.float32),
             "out_scale": np.ascontiguousarray(out_scale, dtype=np.float32)}
        check(lib().aak_mlp_set_norm(self.handle, ptr(n["in_shift"]), ptr(n["in_scale"]), ptr(n["out_shift"]),
                                     ptr(n["out_scale"])), "aak_mlp_set_norm")
        self.norm = n

    def fit_norm(self, x: np.ndarray, y: np.ndarray):
        """Standardise inputs and outputs by the statistics of a training set."""
        g = input_features(x)
        self.set_norm(g.mean(0), 1.0 / np.maximum(g.std(0), 1e-12), y.mean(0), np.maximum(y.std(0), 1e-12))

    def set_adam(self, beta1=0.9, beta2=0.999, eps=1e-8):
        check(lib().aak_mlp_set_adam(self.handle, float(beta1), float(beta2), float(eps)), "aak_mlp_set_adam")

    # ---- inference
    def predict(self, x: np.ndarray) -> np.ndarray:
        """Map coordinates for host points x[n][4] (synchronous)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros((x.shape[0], 3))
        check(lib().aak_mlp_predict_host(self.handle, ptr(x), ptr(y), int(x.shape[0])), "aak_mlp_predict_host")
        return y

    def forward_device(self, x_ptr: int, y_ptr: int, n: int, stream: int = 0):
        check(lib().aak_mlp_forward(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr), int(n),
                                    ctypes.c_void_p(stream)), "aak_mlp_forward")

    # ---- training
    def gradients_device(self, x_ptr: int, y_ptr: int, n: int, grad_ptr: int, perm_ptr: int = 0, stream: int = 0):
        loss = ctypes.c_float()
        check(lib().aak_mlp_gradients(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                      ctypes.c_void_p(perm_ptr or None), int(n), ctypes.c_void_p(grad_ptr),
                                      ctypes.byref(loss), ctypes.c_void_p(stream)), "aak_mlp_gradients")
        return float(loss.value)

    def train_step_device(self, x_ptr: int, y_ptr: int, n: int, lr: float, perm_ptr: int = 0, stream: int = 0,
                          want_loss: bool = False):
        loss = ctypes.c_float()
        check(lib().aak_mlp_train_step(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                       ctypes.c_void_p(perm_ptr or None), int(n), float(lr),
                                       ctypes.byref(loss) if want_loss else None, ctypes.c_void_p(stream)),
              "aak_mlp_train_step")
        return float(loss.value) if want_loss else None

    def train(self, x: np.ndarray, y: np.ndarray, epochs: int = 30, batch: int = 8192, lr: float = 2e-3,
              lr_min: float = 2e-5, seed: int = 0, fit_norm: bool = True) -> dict:
        """Adam on the GPU with a cosine learning-rate schedule; minibatches are
        drawn from a per-epoch permutation held on the device."""
        import torch  # device memory and the permutation only

        keep = np.all(np.isfinite(y), axis=1)
        x, y = x[keep], y[keep]  # callers pass the rows their label_valid mask keeps
        if fit_norm:
            self.fit_norm(x, y)
        batch = min(int(batch), max_train_rows())
        dev = torch.device("cuda", self.device)
        xd = torch.as_tensor(x.astype(np.float32), device=dev).contiguous()
        yd = torch.as_tensor(y.astype(np.float32), device=dev).contiguous()
        n = xd.shape[0]
        gen = torch.Generator(device=dev)
        gen.manual_seed(int(seed))
        steps_per_epoch = (n + batch - 1) // batch
        total = epochs * steps_per_epoch
        hist = []
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        step = 0
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen, device=dev).to(torch.int32)
            for k in range(steps_per_epoch):
                lo = k * batch
                nb = min(batch, n - lo)
                cur = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * step / max(total - 1, 1)))
                last = k == steps_per_epoch - 1
                loss = self.train_step_device(xd.data_ptr(), yd.data_ptr(), nb, cur, perm_ptr=perm.data_ptr() + 4 * lo,
                                              want_loss=last)
                step += 1
            hist.append(loss)
        torch.cuda.synchronize(dev)
        return {"epochs": epochs, "steps": step, "batch": batch, "train_points": int(n), "seconds": time.perf_counter() - t0,
                "loss": hist}

    # ---- persistence
    def save(self, path: str):
        np.savez(path, params=self.params(), **{k: v for k, v in self.norm.items()})

    @classmethod
    def load(cls, path: str, device: int = 0) -> "ParMapMLP":
        d = np.load(path)
        m = cls(device=device, params=d["params"])
        m.set_norm(d["in_shift"], d["in_scale"], d["out_shift"], d["out_scale"])
        return m


def _pct(a: np.ndarray) -> dict:
    a = np.asarray(a, dtype=np.float64)
    return {"mean": float(a.mean()), "p50": float(np.percentile(a, 50)), "p90": float(np.percentile(a, 90)),
            "p99": float(np.percentile(a, 99)), "max": float(a.max())}


def evaluate(model: ParMapMLP, data: dict, nthreads: int = 0) -> dict:
    """Held-out comparison of the plain and warm-started map solves on the
    points whose plain solve reaches a physical root."""
    ok = data["valid"] if "valid" in data else np.all(np.isfinite(data["y"]), axis=1)
    x, om, ytrue = data["x"][ok], data["omega"][ok], data["y"][ok]
    t0 = time.perf_counter()
    pred = model.predict(x)
    t_pred = time.perf_counter() - t0
    cold = solve_batch(x, om, None, nthreads)
    warm = solve_batch(x, om, pred, nthreads)
    scale = LABEL_MASS * np.abs(om).sum(axis=1)  # |Omega|_1 M: residual scale
    sol_diff = np.max(np.abs(warm["y"] - cold["y"]) / np.maximum(np.abs(cold["y"]), 1e-3), axis=1)
    return {
        "points": int(x.shape[0]),
        "iters_cold": _pct(np.abs(cold["iters"])),
        "iters_warm": _pct(np.abs(warm["iters"])),
        "iterations_saved_frac": float(1.0 - np.abs(warm["iters"]).mean() / np.abs(cold["iters"]).mean()),
        "iters_to_tol_cold": _pct(cold["iters_to_tol"]),
        "iters_to_tol_warm": _pct(warm["iters_to_tol"]),
        "iterations_to_tol_saved_frac": float(1.0 - warm["iters_to_tol"].mean() / cold["iters_to_tol"].mean()),
        "fallback_rate": float(warm["fallback"].mean()),
        "failed_cold": int(np.sum(cold["iters"] < 0)),
        "failed_warm": int(np.sum(warm["iters"] < 0)),
        "residual_rel_cold_max": float(np.max(cold["residual"] / scale)),
        "residual_rel_warm_max": float(np.max(warm["residual"] / scale)),
        "residual_abs_warm_max": float(np.max(warm["residual"])),
        "guess_residual_rel": _pct(warm["guess_residual"] / scale),
        "prediction_abs_err": {k: float(v) for k, v in zip(("v_sqrt_p", "M_ratio", "ds"), np.max(np.abs(pred - ytrue), axis=0))},
        "warm_vs_cold_solution_max_rel": float(sol_diff.max()),
        "solve_seconds_cold": cold["seconds"],
        "solve_seconds_warm": warm["seconds"],
        "predict_seconds": t_pred,
    }
