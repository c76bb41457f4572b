"""``GPUAAK`` with the call shape of the reference Cython class
(pygpuAAK/GPUAAK.pyx:50-93, include/AAK_manager.hh:106-153), backed by
``aak_gpu_*`` in libaak_b200.so.

Additions: :meth:`GPUAAK.likelihood_batch` evaluates many templates per call
(one batched generation, one batched FFT, one reduction) instead of one
template per call.  Templates follow the reference CPU AAK conventions.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import AAKError, check, lib, ptr

_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)


def _bind():
    L = lib()
    if getattr(L, "_gpu_bound", False):
        return L
    v = ctypes.c_void_p
    L.aak_gpu_create.argtypes = [ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(v)]
    L.aak_gpu_destroy.argtypes = [v]
    L.aak_gpu_destroy.restype = None
    L.aak_gpu_input_data.argtypes = [v, _dp, _dp, _dp, _dp, ctypes.c_int32]
    L.aak_gpu_gen.argtypes = [v, _dp]
    L.aak_gpu_get_waveform.argtypes = [v, _dp, _dp, _dp]
    L.aak_gpu_likelihood.argtypes = [v, _dp]
    L.aak_gpu_likelihood_batch.argtypes = [v, _dp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _dp, _i32p]
    L.aak_gpu_last_timing.argtypes = [v, _dp]
    L.aak_gpu_set_precision.argtypes = [v, ctypes.c_int32]
    L.aak_gpu_set_variant.argtypes = [v, ctypes.c_int32, ctypes.c_int32]
    L.aak_gpu_fisher.argtypes = [v, _dp, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _dp, _i32p]
    L.aak_gpu_fisher_batch.argtypes = [v, _dp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _dp,
                                       _i32p]
    L._gpu_bound = True
    return L


class GPUAAK:
    def __init__(self, T_fit, init_length, length, init_dt, dt, LISA, backint):
        L = _bind()
        self.length = int(length)
        self._precision = 0
        self.fft_length = self.length // 2 + 1
        self._g = ctypes.c_void_p()
        check(L.aak_gpu_create(float(T_fit), int(init_length), int(length), float(init_dt), float(dt), int(bool(LISA)),
                               int(bool(backint)), ctypes.byref(self._g)), "aak_gpu_create")
        self._w = [np.ones(self.fft_length), np.ones(self.fft_length)]
        self._spectral = False

    def __del__(self):
        try:
            if self._g:
                lib().aak_gpu_destroy(self._g)
                self._g = ctypes.c_void_p()
        except Exception:
            pass

    def input_data(self, hI_f_, hII_f_, channel_ASDinv1_, channel_ASDinv2_):
        h1 = np.ascontiguousarray(hI_f_, dtype=np.complex128)
        h2 = np.ascontiguousarray(hII_f_, dtype=np.complex128)
        w1 = np.ascontiguousarray(channel_ASDinv1_, dtype=np.float64)
        w2 = np.ascontiguousarray(channel_ASDinv2_, dtype=np.float64)
        n = len(h1)
        check(lib().aak_gpu_input_data(self._g, h1.view(np.float64).ctypes.data_as(_dp),
                                       h2.view(np.float64).ctypes.data_as(_dp), ptr(w1), ptr(w2), n),
              "aak_gpu_input_data")
        self._w = [w1.copy(), w2.copy()]

    def gpu_gen_AAK(self, iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D):
        x = np.array([iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D], dtype=np.float64)
        check(lib().aak_gpu_gen(self._g, ptr(x)), "gpu_gen_AAK")
        self._spectral = False

    def GetWaveform(self, is_Fourier=False):
        n = self.length + 2
        t, hI, hII = np.zeros(n), np.zeros(n), np.zeros(n)
        check(lib().aak_gpu_get_waveform(self._g, ptr(t), ptr(hI), ptr(hII)), "GetWaveform")
        if self._spectral:
            # the reference weights the spectra in place during Likelihood()
            m = 2 * self.fft_length
            for arr, w in ((hI, self._w[0]), (hII, self._w[1])):
                arr[:m:2] *= w
                arr[1:m:2] *= w
        return t, hI, hII

    def Likelihood(self):
        out = np.zeros(2)
        check(lib().aak_gpu_likelihood(self._g, ptr(out)), "Likelihood")
        self._spectral = True
        return out

    def WaveformThroughLikelihood(self, iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D,
                                  return_waveform=False):
        self.gpu_gen_AAK(iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D)
        if return_waveform:
            return (0.0, 0.0)
        return self.Likelihood()

    # ------------------------------------------------------------------ batched extension
    def likelihood_batch(self, params, max_batch=256, nthreads=0, return_status=False):
        """params: (nsrc, 14) in gpu_gen_AAK order -> (nsrc, 2) [4<h|d>, 4<h|h>]."""
        x = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        if x.shape[1] != 14:
            raise ValueError("params must have 14 columns (gpu_gen_AAK order)")
        n = x.shape[0]
        out = np.zeros((n, 2))
        st = np.zeros(n, dtype=np.int32)
        check(lib().aak_gpu_likelihood_batch(self._g, ptr(x), n, int(max_batch), int(nthreads), ptr(out), ptr(st)),
              "likelihood_batch")
        self._spectral = False
        return (out, st) if return_status else out

    def fisher_gram(self, params, scale, nthreads=0, return_status=False):
        """Per-channel Gram matrices of finite-difference template spectra.

        params: (2 nd, 14) in gpu_gen_AAK order, rows 2i and 2i+1 the two
        evaluations of derivative i (nd <= 16).  The 2 nd templates are generated
        as one batch, transformed and reduced on the device; returns G of shape
        (2, nd, nd) with G[c, i, j] = 4 Re sum_f conj(D_i) D_j,
        D_i = scale * w_c * (FFT h_{2i+1} - FFT h_{2i}), w_c the input_data weights.
        """
        x = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        if x.shape[1] != 14 or x.shape[0] % 2:
            raise ValueError("params must be (2 nd, 14) in gpu_gen_AAK order")
        nd = x.shape[0] // 2
        G = np.zeros((2, nd, nd))
        st = np.zeros(2 * nd, dtype=np.int32)
        check(lib().aak_gpu_fisher(self._g, ptr(x), nd, float(scale), int(nthreads), ptr(G), ptr(st)), "fisher")
        self._spectral = True
        return (G, st) if return_status else G

    def fisher_gram_batch(self, params, scale, nthreads=0, return_status=False):
        """fisher_gram of several points in one call.

        params: (npts, 2 nd, 14), each block laid out as for fisher_gram;
        returns G of shape (npts, 2, nd, nd), G[k] = fisher_gram(params[k]).
        The next point is planned on host threads while the device generates,
        transforms and reduces the current one.
        """
        x = np.ascontiguousarray(params, dtype=np.float64)
        if x.ndim != 3 or x.shape[2] != 14 or x.shape[1] % 2:
            raise ValueError("params must be (npts, 2 nd, 14) in gpu_gen_AAK order")
        npts, nd = x.shape[0], x.shape[1] // 2
        G = np.zeros((npts, 2, nd, nd))
        st = np.zeros((npts, 2 * nd), dtype=np.int32)
        check(lib().aak_gpu_fisher_batch(self._g, ptr(x), npts, nd, float(scale), int(nthreads), ptr(G), ptr(st)),
              "fisher_batch")
        self._spectral = True
        return (G, st) if return_status else G

    def set_parmap_device(self, on: bool = True):
        """Solve the Kerr->AK map of a template batch's coarse points on the GPU
        (bit-identical to the host solve)."""
        check(lib().aak_gpu_set_parmap_device(self._g, int(bool(on))), "set_parmap_device")

    def set_precision(self, precision: int):
        """0: FP64 throughout (default); 1: split precision; 2: split templates,
        FP32 transform and compensated FP32 products (likelihood batches)."""
        check(lib().aak_gpu_set_precision(self._g, int(precision)), "set_precision")
        self._precision = int(precision)

    NUM_VARIANTS = 6  # AAK_NUM_VARIANTS: launch shapes of the waveform stage

    def set_variant(self, precision: int, variant: int):
        """Launch shape of the template waveform stage for kernel precision 0
        (FP64) or 1 (split, also precision 2)."""
        check(lib().aak_gpu_set_variant(self._g, int(precision), int(variant)), "set_variant")

    def autotune(self, params, max_batch=256, nthreads=0):
        """Pick the waveform stage's launch shape for the current precision on
        a representative sample of templates (params: (n, 14)): each candidate
        runs likelihood_batch(params) once to warm up and once timed (device
        time of the waveform stage); the fastest is kept.  Returns (choice,
        ms per candidate)."""
        kp = 0 if self._precision == 0 else 1
        ms = []
        for v in range(self.NUM_VARIANTS):
            self.set_variant(kp, v)
            self.likelihood_batch(params, max_batch=max_batch, nthreads=nthreads)
            self.likelihood_batch(params, max_batch=max_batch, nthreads=nthreads)
            ms.append(self.last_timing_ms()["waveform"])
        best = int(np.argmin(ms))
        self.set_variant(kp, best)
        return best, ms

    def set_warm_start(self, model=None):
        """Seed every Kerr->AK map solve of the template batches with a trained
        :class:`~emri_kludge_suite_b200.parmap_mlp.ParMapMLP` (None: plain guess)."""
        self._model = model
        check(lib().aak_gpu_set_parmap_model(self._g, model.handle if model is not None else None),
              "set_warm_start")

    def last_timing_ms(self):
        ms = np.zeros(4)
        check(lib().aak_gpu_last_timing(self._g, ptr(ms)), "timing")
        return dict(zip(("host_plan", "waveform", "fft", "reduce"), ms))
