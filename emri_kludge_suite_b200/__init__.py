"""B200-native AAK EMRI waveform and LISA likelihood (sm_100a).

Drop-in for the waveform hot path of alvincjk/EMRI_Kludge_Suite:
``AAKwrapper.wave`` / ``phase`` / ``tdi`` (CPU AAK call shapes) and ``GPUAAK`` / ``pyGPUAAK``
(GPU likelihood call shapes), backed by libaak_b200.so (include/aak.h).
"""
from . import AAKwrapper  # noqa: F401
from .aak import PHASE_ROWS, TDI_ROWS, AAKValueError, Mapped, WaveBatch, front_end, genwave, phase, tdi, wave  # noqa: F401

__version__ = "0.1.0"
