"""``pyGPUAAK`` with the call shape of the reference (pygpuAAK/pygpuAAK.py:20-300):
noise-weighted negative log-likelihood NLL = (d_d + h_h - 2 d_h) / 2 of
templates against LISA-like data, evaluated in batches on the GPU.
"""
from __future__ import annotations

import numpy as np

from .convert import Converter
from .gpuAAK import GPUAAK
from .LISAnoise import LISA_Noise, generate_noise_frequencies, generate_noise_single_channel


class pyGPUAAK:
    def __init__(self, data_info, length, dt, init_dt, key_order, **kwargs):
        prop_defaults = {"T_fit": 1.0, "LISA": True, "backint": True, "eps": 1e-6, "nwalkers": 1, "ndevices": 1,
                         "wd_dur": 1, "add_noise": None, "max_batch": 256, "noise_seed": None}
        self.ndim = len(key_order)
        self.length = length
        self.init_dt = init_dt
        self.dt = dt
        self.converter = Converter("emri", key_order)
        self.key_order = key_order
        self.total_time = self.length * self.dt
        self.init_length = int(np.ceil(self.total_time / self.init_dt))
        for prop, default in prop_defaults.items():
            setattr(self, prop, kwargs.get(prop, default))
            kwargs[prop] = kwargs.get(prop, default)
        if int(self.ndevices) > 1:
            # the reference accepts ndevices but uses one device; here the
            # templates of a batch are split over the devices (LPT)
            from .shard import MultiDeviceGPUAAK

            self.generator = MultiDeviceGPUAAK(range(int(self.ndevices)), self.T_fit, self.init_length, self.length,
                                               self.init_dt, self.dt, self.LISA, self.backint)
        else:
            self.generator = GPUAAK(self.T_fit, self.init_length, self.length, self.init_dt, self.dt, self.LISA,
                                    self.backint)
        self.determine_freqs_noise(**kwargs)
        self.data_info = data_info
        self.create_input_data(**kwargs)

    def determine_freqs_noise(self, **kwargs):
        self.freqs = generate_noise_frequencies(self.length * self.dt, 1 / self.dt)
        self.fft_length = len(self.freqs)
        df = 1.0 / (self.length * self.dt)
        self.freqs[0] = self.freqs[1] / 10.0
        self.added_noise = [0.0, 0.0]
        if self.add_noise is not None:
            rng = np.random.default_rng(self.noise_seed)
            self.added_noise[0] = generate_noise_single_channel(LISA_Noise, [], {"dur": self.wd_dur}, df, self.freqs, rng)
            self.added_noise[1] = generate_noise_single_channel(LISA_Noise, [], {"dur": self.wd_dur}, df, self.freqs, rng)

    def create_input_data(self, **kwargs):
        self.noise_channel1_inv = 1.0 / np.sqrt(LISA_Noise(self.freqs, dur=self.wd_dur)) * np.sqrt(self.dt / self.length)
        self.noise_channel2_inv = 1.0 / np.sqrt(LISA_Noise(self.freqs, dur=self.wd_dur)) * np.sqrt(self.dt / self.length)
        if "channel1" in self.data_info:
            self.injection_channel1 = self.data_info["channel1"].copy()
            self.injection_channel2 = self.data_info["channel2"].copy()
        else:
            self.injection_params = self.data_info["injection_params"]
            zero = np.zeros_like(self.noise_channel1_inv, dtype=np.complex128)
            one = np.ones_like(self.noise_channel1_inv, dtype=np.float64)
            self.generator.input_data(zero, zero, one, one)
            inj = np.tile(np.array([self.injection_params.get(key) for key in self.key_order]), (1, 1))
            hI_f, hII_f = self.getNLL(inj.T, return_TDI=True)
            self.injection_channel1_no_noise = hI_f
            self.injection_channel2_no_noise = hII_f
            self.injection_channel1 = hI_f[0] + self.added_noise[0]
            self.injection_channel2 = hII_f[0] + self.added_noise[1]
        self.data_channel1 = self.noise_channel1_inv * self.injection_channel1
        self.data_channel2 = self.noise_channel2_inv * self.injection_channel2
        self.generator.input_data(self.data_channel1, self.data_channel2, self.noise_channel1_inv,
                                  self.noise_channel2_inv)
        self.d_d = 4 * np.sum([np.abs(self.data_channel1) ** 2, np.abs(self.data_channel2) ** 2])

    def NLL(self, iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D, return_snr=False,
            return_TDI=False, return_waveform=False, **kwargs):
        cols = [np.atleast_1d(np.asarray(v, dtype=np.float64))
                for v in (iota, s, p, e, M, mu, gamma, psi, alph, theta_S, phi_S, theta_K, phi_K, D)]
        n = len(cols[0])
        X = np.stack([np.broadcast_to(c, (n,)) for c in cols], axis=1)
        if return_TDI or return_waveform:
            if return_TDI:
                hI = np.zeros((n, self.fft_length), dtype=np.complex128)
                hII = np.zeros((n, self.fft_length), dtype=np.complex128)
            else:
                hI = np.zeros((n, self.length + 2))
                hII = np.zeros((n, self.length + 2))
            for i in range(n):
                self.generator.WaveformThroughLikelihood(*X[i], return_waveform=return_waveform)
                _, t1, t2 = self.generator.GetWaveform(is_Fourier=return_TDI)
                if return_TDI:
                    hI[i].real, hI[i].imag = t1[0::2][: self.fft_length], t1[1::2][: self.fft_length]
                    hII[i].real, hII[i].imag = t2[0::2][: self.fft_length], t2[1::2][: self.fft_length]
                else:
                    hI[i], hII[i] = t1, t2
            return hI, hII
        like = self.generator.likelihood_batch(X, max_batch=self.max_batch)
        d_h, h_h = like[:, 0], like[:, 1]
        if return_snr:
            return np.sqrt(d_h), np.sqrt(h_h)
        return 1 / 2 * (self.d_d + h_h - 2 * d_h)

    def getNLL(self, x, **kwargs):
        x = self.converter.recycle(x)
        x_in = self.converter.convert(x.copy())
        return self.NLL(*x_in, **kwargs)

    def _physical(self, x):
        """Sampler coordinates (ndim, n) -> (n, 14) gpu_gen_AAK parameters, as getNLL converts them."""
        x = self.converter.recycle(x)
        cols = [np.atleast_1d(np.asarray(v, dtype=np.float64)) for v in self.converter.convert(x.copy())]
        n = max(len(c) for c in cols)
        return np.stack([np.broadcast_to(c, (n,)) for c in cols], axis=1)

    def get_Fisher(self, x, form="reference"):
        """Fisher matrix at x by central differences of step eps in each sampler
        coordinate (pygpuAAK/pygpuAAK.py:269-300).  The 2 ndim templates are
        generated as one batch and their weighted spectra reduced on the device
        (GPUAAK.fisher_gram); only the Gram matrices come back to the host.

        form="reference" reproduces the published formula, which pairs the
        channel-I derivative j with itself: M_ij = 4 Re(<d_j h_I, d_j h_I> +
        <d_i h_II, d_j h_II>) for i <= j, mirrored.  form="full" is the
        two-channel Fisher matrix 4 Re(<d_i h_I, d_j h_I> + <d_i h_II, d_j h_II>).
        """
        if form not in ("reference", "full"):
            raise ValueError("form must be 'reference' or 'full'")
        G = self.generator.fisher_gram(self._fisher_rows(x), 1.0 / (2 * self.eps))
        return self._fisher_matrix(G, form).astype(x.dtype)

    def get_Fisher_batch(self, X, form="reference"):
        """get_Fisher at each row of X (npts, ndim) in one device call
        (GPUAAK.fisher_gram_batch: the next point is planned while the device
        works on the current one); returns (npts, ndim, ndim)."""
        if form not in ("reference", "full"):
            raise ValueError("form must be 'reference' or 'full'")
        X = np.atleast_2d(X)
        rows = np.stack([self._fisher_rows(x) for x in X])
        G = self.generator.fisher_gram_batch(rows, 1.0 / (2 * self.eps))
        return np.stack([self._fisher_matrix(g, form) for g in G]).astype(X.dtype)

    def _fisher_rows(self, x):
        """The 2 ndim central-difference templates of x, (2 ndim, 14) physical."""
        x_in = np.tile(x, (2 * self.ndim, 1))
        for i in range(self.ndim):
            x_in[2 * i, i] += self.eps
            x_in[2 * i + 1, i] -= self.eps
        return self._physical(x_in.T)

    @staticmethod
    def _fisher_matrix(G, form):
        if form == "reference":
            A = G[0].diagonal()[None, :] + G[1]
            return np.triu(A) + np.triu(A, 1).T
        return G[0] + G[1]
