"""Python surface of the B200 AAK library.

* :func:`wave` -- the call shape of the reference ``AAKwrapper.wave(pars)``
  (AAKwrapper/AAKwrapper.pyx:50-88): returns ``(t, hI, hII, timing)``.
* :func:`tdi` -- ``AAKwrapper.tdi(pars)`` (AAKwrapper/AAKwrapper.pyx:135-177):
  returns ``(f, Xf_r, Xf_im, Yf_r, Yf_im, Zf_r, Zf_im, timing)``.
* :func:`phase` -- ``AAKwrapper.phase(pars)`` (AAKwrapper/AAKwrapper.pyx:90-133):
  returns ``(t, phase_r, phase_theta, phase_phi, omega_r, omega_theta,
  omega_phi, eccentricity, timing)``.
* :func:`front_end` / :func:`genwave` -- the two halves of ``AAKwave``
  (src/suite/AAKpy.cc:16-51): mapped trajectory, then GenWave/waveform.
* :class:`WaveBatch` -- many sources in one launch, outputs in device memory.

Failures raise :class:`AAKValueError` (a ``ValueError``) where the reference
would terminate the process.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import AAKMapped, AAKValueError, check, lib, make_params, params_array, ptr

__all__ = ["wave", "phase", "tdi", "PHASE_ROWS", "TDI_ROWS", "front_end", "genwave", "Mapped", "WaveBatch", "AAKValueError"]


@dataclass
class Mapped:
    """Mapped trajectory handed to GenWave (src/suite/AAKpy.cc:29-44)."""

    steps: int
    e_traj: np.ndarray
    v_map: np.ndarray
    M_map: np.ndarray
    s_map: np.ndarray
    dt_map: np.ndarray
    Phi0: float
    inspiral_flag: int
    newton_iterations: int

    def to_struct(self) -> AAKMapped:
        m = AAKMapped()
        m.steps = self.steps
        m.inspiral_flag = self.inspiral_flag
        m.newton_iterations = self.newton_iterations
        m.Phi0 = self.Phi0
        for name in ("e_traj", "v_map", "M_map", "s_map", "dt_map"):
            arr = getattr(m, name)
            src = getattr(self, name)
            for i in range(self.steps):
                arr[i] = float(src[i])
        return m

    @staticmethod
    def from_struct(m: AAKMapped) -> "Mapped":
        n = m.steps
        return Mapped(
            n,
            *[np.array(getattr(m, k)[:n], dtype=np.float64) for k in ("e_traj", "v_map", "M_map", "s_map", "dt_map")],
            float(m.Phi0),
            int(m.inspiral_flag),
            int(m.newton_iterations),
        )


def front_end(pars: dict, warm_start: np.ndarray | None = None) -> Mapped:
    """Coarse Kerr inspiral, Kerr frequencies and the Kerr->AK map (host)."""
    m = AAKMapped()
    ws = None
    if warm_start is not None:
        ws = np.ascontiguousarray(warm_start, dtype=np.float64)
    check(lib().aak_front_end(ctypes.byref(make_params(pars)), ptr(ws), ctypes.byref(m)), "aak_front_end")
    return Mapped.from_struct(m)


def wave(pars: dict):
    """AAKwrapper.wave: ``(t, hI, hII, timing)`` for the dict of SetPar fields."""
    n = int(pars["length"])
    t = np.zeros(n)
    hI = np.zeros(n)
    hII = np.zeros(n)
    secs = ctypes.c_double(0.0)
    check(lib().aak_wave(ctypes.byref(make_params(pars)), ptr(t), ptr(hI), ptr(hII), ctypes.byref(secs)), "aak_wave")
    return t, hI, hII, secs.value


#: rows of the phase product, in the order of AAKwrapper.phase
PHASE_ROWS = ("t", "phase_r", "phase_theta", "phase_phi", "omega_r", "omega_theta", "omega_phi", "eccentricity")


def phase(pars: dict):
    """AAKwrapper.phase: ``(t, phase_r, phase_theta, phase_phi, omega_r,
    omega_theta, omega_phi, eccentricity, timing)`` for the dict of SetPar fields
    (GenPhase, src/suite/AAKPhase.cc:315-374, on the GPU in FP64)."""
    n = int(pars["length"])
    rows = [np.zeros(n) for _ in PHASE_ROWS]
    secs = ctypes.c_double(0.0)
    check(lib().aak_phase(ctypes.byref(make_params(pars)), *[ptr(a) for a in rows], ctypes.byref(secs)), "aak_phase")
    return (*rows, secs.value)


#: rows of the frequency-domain TDI, in the order of AAKwrapper.tdi (after f)
TDI_ROWS = ("Xf_r", "Xf_im", "Yf_r", "Yf_im", "Zf_r", "Zf_im")


def tdi(pars: dict):
    """AAKwrapper.tdi: ``(f, Xf_r, Xf_im, Yf_r, Yf_im, Zf_r, Zf_im, timing)`` on the
    (length + 1) // 2 bins f = i / ((length - 1) dt) (GenTDI,
    src/suite/AAKTDI.cc:799-829, on the GPU in FP64)."""
    n = (int(pars["length"]) + 1) // 2
    f = np.zeros(n)
    rows = [np.zeros(n) for _ in TDI_ROWS]
    secs = ctypes.c_double(0.0)
    check(lib().aak_tdi(ctypes.byref(make_params(pars)), ptr(f), *[ptr(a) for a in rows], ctypes.byref(secs)),
          "aak_tdi")
    return (f, *rows, secs.value)


def genwave(pars: dict, mapped: Mapped, nmodes: int = 0):
    """GenWave -> waveform on a mapped trajectory (src/suite/AAK.cc:565-591).

    ``nmodes <= 0`` keeps the reference harmonic rule.  Returns (t, hI, hII).
    """
    n = int(pars["length"])
    t, hI, hII = np.zeros(n), np.zeros(n), np.zeros(n)
    arrs = [np.ascontiguousarray(getattr(mapped, k), dtype=np.float64) for k in ("e_traj", "v_map", "M_map", "s_map", "dt_map")]
    e, v, Mm, sm, dtm = arrs
    check(
        lib().aak_genwave(
            ptr(t), ptr(hI), ptr(hII), float(pars["dt"]), n, ptr(e), ptr(v), float(pars["M"]), ptr(Mm),
            float(pars["mu"]), float(pars["s"]), ptr(sm), float(pars["D"]), float(pars["iota"]), float(pars["gamma"]),
            float(mapped.Phi0), float(pars["theta_S"]), float(pars["phi_S"]), float(pars["alpha"]),
            float(pars["theta_K"]), float(pars["phi_K"]), ptr(dtm), int(mapped.steps), int(bool(pars["backint"])),
            int(bool(pars["LISA"])), int(nmodes),
        ),
        "aak_genwave",
    )
    return t, hI, hII


class WaveBatch:
    """A batch of sources planned on host threads and generated on one GPU.

    Outputs live in caller-provided device memory (``torch.cuda`` tensors or
    raw pointers) laid out by :attr:`offsets`.
    """

    def __init__(self, device: int = 0):
        self._ctx = ctypes.c_void_p()
        check(lib().aak_ctx_create(int(device), ctypes.byref(self._ctx)), "aak_ctx_create")
        self.device = device
        self.nsrc = 0
        self.offsets = np.zeros(1, dtype=np.int64)
        self.status = np.zeros(0, dtype=np.int32)
        self.i_plunge = np.zeros(0, dtype=np.int32)
        self.i_buffer = np.zeros(0, dtype=np.int32)
        self.total_samples = 0

    def close(self):
        if self._ctx:
            lib().aak_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _info(self):
        n = self.nsrc
        self.offsets = np.zeros(n + 1, dtype=np.int64)
        self.status = np.zeros(n, dtype=np.int32)
        self.i_plunge = np.zeros(n, dtype=np.int32)
        self.i_buffer = np.zeros(n, dtype=np.int32)
        tot = ctypes.c_int64()
        check(
            lib().aak_batch_info(self._ctx, ctypes.byref(tot), ptr(self.offsets), ptr(self.status), ptr(self.i_plunge),
                                 ptr(self.i_buffer)),
            "aak_batch_info",
        )
        self.total_samples = int(tot.value)

    def set_parmap_model(self, model=None):
        """Warm-start the Kerr->AK map of every coarse point with a trained
        :class:`~emri_kludge_suite_b200.parmap_mlp.ParMapMLP` (None: plain guess).
        The model must stay alive while this batch plans with it."""
        self._model = model
        check(lib().aak_ctx_set_parmap_model(self._ctx, model.handle if model is not None else None),
              "aak_ctx_set_parmap_model")

    def set_parmap_device(self, on: bool = True):
        """Solve the Kerr->AK map of all coarse points of a batch on the GPU (one
        launch) instead of on the planning threads; results are bit-identical."""
        check(lib().aak_ctx_set_parmap_device(self._ctx, int(bool(on))), "aak_ctx_set_parmap_device")

    def set_evolve_device(self, on: bool = True):
        """Run every source's coarse AK recurrence on the GPU (one thread per
        source) between two host planning passes, instead of on the planning
        threads; knots agree with the host's to about 1e-15 relative."""
        check(lib().aak_ctx_set_evolve_device(self._ctx, int(bool(on))), "aak_ctx_set_evolve_device")

    def plan_ms(self) -> dict:
        """Wall times (ms) of the last plan's passes with the device evolution."""
        ms = np.zeros(4)
        check(lib().aak_batch_plan_ms(self._ctx, ptr(ms)), "aak_batch_plan_ms")
        return dict(zip(("host_before", "device_evolution", "host_after", "total"), ms.tolist()))

    def newton_stats(self) -> dict:
        """Map statistics of the last plan: points, Newton iterations, fallbacks."""
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().aak_batch_newton_stats(self._ctx, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
              "aak_batch_newton_stats")
        return {"points": a.value, "iterations": b.value, "fallbacks": c.value}

    def plan(self, params, nmodes=None, nthreads: int = 0, mapped=None):
        """Host planning; ``params`` is a list of pars dicts (or aak_params)."""
        self.nsrc = len(params)
        P = params_array(params)
        nm = None
        if nmodes is not None:
            nm = np.ascontiguousarray(np.broadcast_to(np.asarray(nmodes, dtype=np.int32), (self.nsrc,)))
        if mapped is not None:
            M = (AAKMapped * self.nsrc)()
            for i, m in enumerate(mapped):
                M[i] = m.to_struct() if isinstance(m, Mapped) else m
            check(lib().aak_batch_plan_mapped(self._ctx, P, M, self.nsrc, ptr(nm), int(nthreads)), "aak_batch_plan_mapped")
        else:
            check(lib().aak_batch_plan(self._ctx, P, self.nsrc, ptr(nm), int(nthreads)), "aak_batch_plan")
        self._info()
        return self

    def plan_bytes(self) -> int:
        b = ctypes.c_int64()
        check(lib().aak_batch_plan_bytes(self._ctx, ctypes.byref(b)), "aak_batch_plan_bytes")
        return int(b.value)

    def upload(self, stream: int = 0):
        check(lib().aak_batch_upload(self._ctx, ctypes.c_void_p(stream)), "aak_batch_upload")

    def run(self, hI_ptr: int, hII_ptr: int, t_ptr: int = 0, traj_ptr: int = 0, traj_stride: int = 0,
            precision: int = 0, stream: int = 0):
        check(
            lib().aak_batch_run(self._ctx, ctypes.c_void_p(hI_ptr), ctypes.c_void_p(hII_ptr), ctypes.c_void_p(t_ptr),
                                ctypes.c_void_p(traj_ptr), int(traj_stride), int(precision), ctypes.c_void_p(stream)),
            "aak_batch_run",
        )

    def run_phase(self, out_ptr: int, stride: int, stream: int = 0):
        """The AAK phase product of every source into device memory: 8 rows
        (:data:`PHASE_ROWS`) of ``stride`` doubles indexed by :attr:`offsets`."""
        check(lib().aak_batch_run_phase(self._ctx, ctypes.c_void_p(out_ptr), int(stride), ctypes.c_void_p(stream)),
              "aak_batch_run_phase")

    def phase_host(self, params, nthreads: int = 0):
        """Plan + upload + phase product + copy back (host buffers).
        Returns (rows, offsets, status) with rows of shape (8, total samples)."""
        self.nsrc = len(params)
        P = params_array(params)
        total = int(sum(int(p["length"]) if isinstance(p, dict) else int(p.length) for p in params))
        rows = np.zeros((8, total))
        offs = np.zeros(self.nsrc + 1, dtype=np.int64)
        st = np.zeros(self.nsrc, dtype=np.int32)
        check(lib().aak_phase_batch_host(self._ctx, P, self.nsrc, int(nthreads), ptr(rows), ptr(offs), ptr(st)),
              "aak_phase_batch_host")
        self._info()
        return rows, offs, st

    def tdi_host(self, params, nthreads: int = 0):
        """Frequency-domain TDI of every source (as :func:`tdi`) in one batch.
        Returns (rows, bin_offsets, status): rows (6, total bins) in
        :data:`TDI_ROWS` order, source s at bins bin_offsets[s]:bin_offsets[s + 1]."""
        self.nsrc = len(params)
        P = params_array(params)
        nb = int(sum((int(p["length"] if isinstance(p, dict) else p.length) + 1) // 2 for p in params))
        rows = np.zeros((6, nb))
        offs = np.zeros(self.nsrc + 1, dtype=np.int64)
        st = np.zeros(self.nsrc, dtype=np.int32)
        check(lib().aak_tdi_batch_host(self._ctx, P, self.nsrc, int(nthreads), ptr(rows), ptr(offs), ptr(st)),
              "aak_tdi_batch_host")
        return rows, offs, st

    def launches(self) -> int:
        return int(lib().aak_batch_last_launches(self._ctx))

    def device_status(self) -> int:
        """Wait for the device; the aak_status of the batch kernels' bounded
        waits since the last upload or call (0, or AAK_ERR_DEVICE_TIMEOUT)."""
        return int(lib().aak_batch_device_status(self._ctx))

    def run_graph(self, hI_ptr: int, hII_ptr: int, precision: int = 0, stream: int = 0):
        """:meth:`run` as one CUDA graph (captured on first use, replayed after)."""
        check(lib().aak_batch_run_graph(self._ctx, ctypes.c_void_p(hI_ptr), ctypes.c_void_p(hII_ptr), int(precision),
                                        ctypes.c_void_p(stream)), "aak_batch_run_graph")

    def autotune(self, hI_ptr: int, hII_ptr: int, precision: int = 1, cache_path: str | None = None):
        """Time every launch shape of the waveform stage on the uploaded batch
        (outputs into the given device buffers) and keep the fastest for
        ``precision``; with ``cache_path``, reuse or append a tuning-cache
        entry.  Returns (variant, ms per variant; -1 where not timed)."""
        v = ctypes.c_int32()
        ms = (ctypes.c_float * 6)()
        path = cache_path.encode() if cache_path else None
        check(lib().aak_ctx_autotune(self._ctx, ctypes.c_void_p(hI_ptr), ctypes.c_void_p(hII_ptr), int(precision), path,
                                     ctypes.byref(v), ms), "aak_ctx_autotune")
        return int(v.value), [float(x) for x in ms]

    def set_variant(self, precision: int, variant: int):
        """Launch shape of the waveform stage for ``precision`` (0: default)."""
        check(lib().aak_ctx_set_variant(self._ctx, int(precision), int(variant)), "aak_ctx_set_variant")

    def set_precision(self, precision: int):
        """Precision of :meth:`generate_host` (0: FP64, 1: split)."""
        check(lib().aak_ctx_set_precision(self._ctx, int(precision)), "aak_ctx_set_precision")

    def run_plain(self, hI_ptr: int, hII_ptr: int, traj_ptr: int, traj_stride: int, stream: int = 0):
        """The plain FP64 per-source path (baseline): one source at a time, dense
        trajectory in ``traj_ptr`` (9 x traj_stride doubles), five jn() per harmonic."""
        check(lib().aak_batch_run_plain(self._ctx, ctypes.c_void_p(hI_ptr), ctypes.c_void_p(hII_ptr),
                                        ctypes.c_void_p(traj_ptr), int(traj_stride), ctypes.c_void_p(stream)),
              "aak_batch_run_plain")

    def generate_host(self, params, nmodes=None, nthreads: int = 0):
        """Plan + upload + run + copy back (host buffers).  Returns (hI, hII, offsets, status)."""
        self.nsrc = len(params)
        P = params_array(params)
        total = int(sum(int(p["length"]) if isinstance(p, dict) else int(p.length) for p in params))
        hI = np.zeros(total)
        hII = np.zeros(total)
        offs = np.zeros(self.nsrc + 1, dtype=np.int64)
        st = np.zeros(self.nsrc, dtype=np.int32)
        nm = None
        if nmodes is not None:
            nm = np.ascontiguousarray(np.broadcast_to(np.asarray(nmodes, dtype=np.int32), (self.nsrc,)))
        check(
            lib().aak_wave_batch_host(self._ctx, P, self.nsrc, ptr(nm), int(nthreads), ptr(hI), ptr(hII), ptr(offs),
                                      ptr(st)),
            "aak_wave_batch_host",
        )
        self._info()
        return hI, hII, offs, st
