"""Shared fixtures.  GPU tests carry the ``gpu`` marker; everything else runs on CPU."""
from __future__ import annotations

import glob
import json
import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    lib = os.path.join(REPO, "emri_kludge_suite_b200", "libaak_b200.so")
    if not os.path.exists(lib):
        from emri_kludge_suite_b200 import build

        build.build()
    if not os.path.exists(os.path.join(REPO, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "oracle"], check=True)


_ensure_built()


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    d = {k: z[k] for k in z.files}
    d["pars"] = json.loads(str(d["pars"]))
    return d


def golden_mapped(g):
    from emri_kludge_suite_b200.aak import Mapped

    n = int(g["steps"])
    return Mapped(n, g["e_traj"], g["v_map"], g["M_map"], g["s_map"], g["dt_map"], float(g["Phi0"]), 2, 0)


def mismatch(a1, a2, b1, b2):
    """1 - <a|b>/sqrt(<a|a><b|b>) with a flat noise spectrum over both channels."""
    a = np.concatenate([a1, a2])
    b = np.concatenate([b1, b2])
    na, nb = np.dot(a, a), np.dot(b, b)
    if na == 0.0 and nb == 0.0:
        return 0.0
    return 1.0 - np.dot(a, b) / np.sqrt(na * nb)


def psd_mismatch(a1, a2, b1, b2, dt, dur=1):
    """1 - <a|b>/sqrt(<a|a><b|b>) with the noise-weighted inner product
    4 Re sum_k a~_k conj(b~_k) / S_n(f_k) over both channels (k >= 1; the PSD
    is the oracle's LISA_Noise restatement, pinned to the reference's)."""
    from oracle import oracle as O

    n = len(a1)
    f = np.fft.rfftfreq(n, dt)[1:]
    w = 1.0 / O.lisa_noise(f, dur=dur)
    ab = aa = bb = 0.0
    for x, y in ((a1, b1), (a2, b2)):
        X, Y = np.fft.rfft(x)[1:], np.fft.rfft(y)[1:]
        ab += float(np.sum(w * (X * np.conj(Y)).real))
        aa += float(np.sum(w * np.abs(X) ** 2))
        bb += float(np.sum(w * np.abs(Y) ** 2))
    if aa == 0.0 and bb == 0.0:
        return 0.0
    return 1.0 - ab / np.sqrt(aa * bb)


def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref_available():
    from oracle import oracle as O

    return O.ref_available()
