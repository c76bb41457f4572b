"""Module with the reference ``AAKwrapper`` call shapes (AAKwrapper/AAKwrapper.pyx:50-133).

``wave(pars) -> (t, hI, hII, timing)`` and ``phase(pars) -> (t, phase_r,
phase_theta, phase_phi, omega_r, omega_theta, omega_phi, eccentricity,
timing)``; both are computed on the GPU.
"""
from .aak import phase, wave  # noqa: F401

__all__ = ["wave", "phase"]
