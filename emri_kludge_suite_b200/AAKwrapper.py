"""Module with the reference ``AAKwrapper`` call shape (AAKwrapper/AAKwrapper.pyx:50-88).

``wave(pars) -> (t, hI, hII, timing)``; the waveform is computed on the GPU.
"""
from .aak import wave  # noqa: F401

__all__ = ["wave"]
