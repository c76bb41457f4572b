"""Generate tests/golden/psd/lisa_noise.npz from the reference's own noise
model, pygpuAAK/LISAnoise.py, imported from the reference checkout
($AAK_REFERENCE_SRC, else the build container's read-only checkout).

It stores LISA_Noise(f, L, f_star, dur) on a log-spaced grid 1e-5 .. 1 Hz for
dur in (0, 0.5, 1, 2, 4) and for a second (L, f_star), the frequencies of
generate_noise_frequencies for the configuration-4 span (length and a
subset), and the standard
deviation of generate_noise_single_channel's draw (the reference draws from
numpy's global generator, so only its scale is reproducible).

    python tests/golden/psd/make_lisa_noise.py
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_module():
    for root in (os.environ.get("AAK_REFERENCE_SRC"), "/root/reference"):
        path = os.path.join(root, "pygpuAAK", "LISAnoise.py") if root else None
        if path and os.path.exists(path):
            spec = importlib.util.spec_from_file_location("ref_LISAnoise", path)
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            return mod
    raise FileNotFoundError("the reference's pygpuAAK/LISAnoise.py was not found")


def main():
    R = reference_module()
    f = np.logspace(-5, 0, 2001)
    out = {"f": f}
    for dur in (0, 0.5, 1, 2, 4):
        out[f"S_dur{dur}"] = R.LISA_Noise(f, dur=dur)
    out["S_L2e9_fstar0.025_dur1"] = R.LISA_Noise(f, L=2.0e9, f_star=0.025, dur=1)
    fq = R.generate_noise_frequencies(3_200_000 * 10.0, 0.1)
    pick = np.unique(np.concatenate([np.arange(16), np.arange(len(fq) - 16, len(fq)), np.arange(0, len(fq), 9973)]))
    out["freqs_cfg4_len"] = np.array([len(fq)])
    out["freqs_cfg4_idx"] = pick
    out["freqs_cfg4_at"] = fq[pick]
    fr = np.linspace(1e-4, 1e-2, 200_000)
    np.random.seed(20261203)
    n = R.generate_noise_single_channel(R.LISA_Noise, [], {"dur": 1}, 1e-7, fr)
    out["noise_abs2_over_S"] = np.array([np.mean(np.abs(n) ** 2 / R.LISA_Noise(fr, dur=1))])
    path = os.path.join(HERE, "lisa_noise.npz")
    np.savez_compressed(path, **out)
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as fh:
        json.dump({"lisa_noise": hashlib.sha256(open(path, "rb").read()).hexdigest()}, fh, indent=1)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
