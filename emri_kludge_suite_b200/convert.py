"""Sampler-to-physical parameter conversion with the reference call shape
(``pygpuAAK/convert.py``): keys prefixed ``ln_``, ``cos_``, ``sin_`` are
mapped through exp / arccos / arcsin, and the angles phi_S, phi_K, gamma,
psi, alpha are wrapped into [0, 2 pi).  Distances stay in Gpc (the unit the
waveform takes)."""
from __future__ import annotations

import numpy as np

_WRAP_2PI = {"S", "K", "gamma", "psi", "alpha", "phiRef"}


class Converter:
    def __init__(self, source_type, key_order, **kwargs):
        if source_type != "emri":
            raise ValueError("only source_type 'emri' is supported")
        self.key_order = list(key_order)
        self.conversions = []
        self.recycles = []
        for i, key in enumerate(self.key_order):
            head = key.split("_")[0]
            if head in ("ln", "cos", "sin"):
                self.conversions.append((head, i))
            if key in ("phi_S", "phi_K", "gamma", "psi", "alpha", "phiRef"):
                self.recycles.append(i)

    def convert(self, x):
        for head, i in self.conversions:
            x[i] = {"ln": np.exp, "cos": np.arccos, "sin": np.arcsin}[head](x[i])
        return x

    def recycle(self, x):
        for i in self.recycles:
            x[i] = x[i] % (2 * np.pi)
        return x
