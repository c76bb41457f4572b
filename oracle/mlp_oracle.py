"""CPU oracle of the learned ParMap warm-start network -- TEST INFRASTRUCTURE.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
may import this module; the product path never does.

The network is the 4 -> 128 -> 128 -> 128 -> 3 SiLU multilayer perceptron of
``emri_kludge_suite_b200/csrc/kernels/parmap_mlp.cu``.  This module restates
its forward pass and the back-propagated gradient of its loss in float64.
With ``quantize=True`` it rounds to BF16 (round to nearest, ties to even) at
exactly the points where the tensor-core kernels round:

* every weight matrix (W1 .. W4; biases stay unrounded);
* the activations a1, a2, a3 and the back-propagated gradients dz3, dz2
  (the operands of the 128 x 128 tensor-core products);

so the GPU result differs from it only by FP32-versus-FP64 accumulation and
the rare BF16 rounding decision that this difference flips.  With
``quantize=False`` it is the exact float64 network, whose gradient is pinned
against central finite differences in the CPU tests.

The network has no counterpart in the reference; the map it approximates is
ParMap (src/suite/KSParMap.cc:397-440), whose plain solve labels the data.
"""
from __future__ import annotations

import numpy as np

H = 128
LAYOUT = (("W1", (H, 4)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
          ("W4", (3, H)), ("b4", (3,)))
OFFSETS = {}
_o = 0
for _name, _shape in LAYOUT:
    OFFSETS[_name] = (_o, _shape)
    _o += int(np.prod(_shape))
N_PARAMS = _o  # 34051


def unpack(params: np.ndarray) -> dict:
    p = np.asarray(params, dtype=np.float64)
    return {k: p[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFFSETS.items()}


def pack(d: dict) -> np.ndarray:
    out = np.zeros(N_PARAMS)
    for k, (o, s) in OFFSETS.items():
        out[o:o + int(np.prod(s))] = np.asarray(d[k], dtype=np.float64).ravel()
    return out


def bf16(a) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), via float32."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16) & 0xFFFFFFFF
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def features(x: np.ndarray, in_shift, in_scale) -> np.ndarray:
    x = np.asarray(x, dtype=np.float64)
    g = np.stack([1.0 / np.sqrt(x[:, 0]), x[:, 1], np.cos(x[:, 2]), x[:, 3]], axis=1)
    return (g - np.asarray(in_shift, dtype=np.float64)) * np.asarray(in_scale, dtype=np.float64)


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * _sig(z)


def dsilu(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def forward(params, x, norm, quantize: bool = True):
    """Network output in normalised units and the intermediate values."""
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    P = unpack(params)
    W1, W2, W3, W4 = (q(P[k]) for k in ("W1", "W2", "W3", "W4"))
    f = features(x, norm["in_shift"], norm["in_scale"])
    z1 = f @ W1.T + P["b1"]
    a1 = q(silu(z1))
    z2 = a1 @ W2.T + P["b2"]
    a2 = q(silu(z2))
    z3 = a2 @ W3.T + P["b3"]
    a3 = q(silu(z3))
    y = a3 @ W4.T + P["b4"]
    cache = dict(f=f, z1=z1, a1=a1, z2=z2, a2=a2, z3=z3, a3=a3, W1=W1, W2=W2, W3=W3, W4=W4)
    return y, cache


def predict(params, x, norm, quantize: bool = True) -> np.ndarray:
    """Map coordinates (v_map sqrt(p), M_map / M, s_map - a)."""
    y, _ = forward(params, x, norm, quantize)
    return y * np.asarray(norm["out_scale"]) + np.asarray(norm["out_shift"])


def loss_and_grad(params, x, y_true, norm, quantize: bool = True):
    """Mean squared error over rows and the 3 outputs, in normalised output
    units, and its gradient with respect to the flat parameter vector."""
    q = bf16 if quantize else (lambda v: np.asarray(v, dtype=np.float64))
    y, c = forward(params, x, norm, quantize)
    B = y.shape[0]
    t = (np.asarray(y_true, dtype=np.float64) - np.asarray(norm["out_shift"])) / np.asarray(norm["out_scale"])
    d = y - t
    loss = float(np.sum(d * d) / (3.0 * B))
    dy = 2.0 * d / (3.0 * B)
    g = {"W4": dy.T @ c["a3"], "b4": dy.sum(0)}
    dz3 = q((dy @ c["W4"]) * dsilu(c["z3"]))
    g["W3"], g["b3"] = dz3.T @ c["a2"], dz3.sum(0)
    dz2 = q((dz3 @ c["W3"]) * dsilu(c["z2"]))
    g["W2"], g["b2"] = dz2.T @ c["a1"], dz2.sum(0)
    dz1 = (dz2 @ c["W2"]) * dsilu(c["z1"])
    g["W1"], g["b1"] = dz1.T @ c["f"], dz1.sum(0)
    return loss, pack(g)


def adam_step(params, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam update (Kingma & Ba 2015, bias-corrected) in float64."""
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    mh = m / (1 - beta1**step)
    vh = v / (1 - beta2**step)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
