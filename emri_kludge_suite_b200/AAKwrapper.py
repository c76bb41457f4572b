"""Module with the reference ``AAKwrapper`` call shapes (AAKwrapper/AAKwrapper.pyx:50-177).

``wave(pars) -> (t, hI, hII, timing)``, ``phase(pars) -> (t, phase_r,
phase_theta, phase_phi, omega_r, omega_theta, omega_phi, eccentricity,
timing)`` and ``tdi(pars) -> (f, Xf_r, Xf_im, Yf_r, Yf_im, Zf_r, Zf_im,
timing)``; all are computed on the GPU.
"""
from .aak import phase, tdi, wave  # noqa: F401

__all__ = ["wave", "phase", "tdi"]
