"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It is the checker for the product path and
is never used by the product library (``emri_kludge_suite_b200``).

Two native libraries are wrapped:

* ``liboracle.so`` -- ``aak_oracle.c``, the plain-C restatement of the
  reference's dense AAK path (PNevolution + waveform, src/suite/AAK.cc:27-562).
* ``_ref/libaakref.so`` -- the reference's own unmodified C++ sources compiled
  against the project GSL shim (``make -C oracle ref``), wrapped by
  ``ref_harness.cpp``.  Present only where it was built.

The likelihood oracle (:func:`inner_products`) restates the reference's GPU
likelihood semantics in numpy: rFFT of the template channels, weighting by
``noise_inv = S_n^{-1/2} sqrt(dt/N)`` and the ``4 Re<h|d>`` / ``4 <h|h>`` sums of
src/cuda/AAK_manager.cu:352-446 and pygpuAAK/pygpuAAK.py:86-145, 240.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libaakref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)

MSUN_SEC = 6.67259e-11 * 1.98892e30 / 299792458.0 ** 3
GPC = 3.0856775807e16 * 1.0e9 / 299792458.0
YEAR = 31558149.8


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


_oracle = None
_ref = None


def reference_src() -> str | None:
    """The reference checkout to compile oracle/_ref from: $AAK_REFERENCE_SRC,
    else the build container's read-only checkout when it exists."""
    for cand in (os.environ.get("AAK_REFERENCE_SRC"), "/root/reference"):
        if cand and os.path.exists(os.path.join(cand, "src", "suite", "AAK.cc")):
            return cand
    return None


def build(force: bool = False) -> None:
    """Compile liboracle.so (and the reference build when its sources exist)."""
    import subprocess

    ref = reference_src()
    subprocess.run(["make", "-s", "-C", HERE, "all"] + ([f"REF={ref}"] if ref else []), check=True)


def set_threads(n: int) -> None:
    """Host threads of the oracle's per-sample harmonic sums (default 1)."""
    oracle_lib().oracle_set_threads(int(n))


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_waveform.restype = ctypes.c_int
        L.oracle_genwave.restype = ctypes.c_int
        L.oracle_pnevolution.restype = ctypes.c_int
        for n in ("oracle_dvdt", "oracle_dedt"):
            getattr(L, n).restype = ctypes.c_double
            getattr(L, n).argtypes = [ctypes.c_double] * 6
        for n in ("oracle_dtdm", "oracle_drdm", "oracle_dthetadm", "oracle_dphidm"):
            getattr(L, n).restype = ctypes.c_double
            getattr(L, n).argtypes = [ctypes.c_double] * 4
        L.oracle_omega_phi.restype = ctypes.c_double
        L.oracle_omega_phi.argtypes = [ctypes.c_double] * 5
        _oracle = L
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} not built (make -C oracle ref needs the reference sources)")
        L = ctypes.CDLL(REF_SO)
        L.ref_aakwave.restype = ctypes.c_double
        L.ref_front.restype = ctypes.c_int
        L.ref_elisa_noise.restype = ctypes.c_double
        L.ref_elisa_noise.argtypes = [ctypes.c_double]
        _ref = L
    return _ref


class RefParams(ctypes.Structure):
    """Numeric SetPar fields (reference include/KSTools.h:21-53)."""

    _fields_ = [
        (n, ctypes.c_double)
        for n in "length dt p T f T_fit mu M s e iota gamma psi theta_S phi_S theta_K phi_K alpha D".split()
    ] + [("backint", ctypes.c_int), ("LISA", ctypes.c_int)]


PAR_KEYS = "length dt p T f T_fit mu M s e iota gamma psi theta_S phi_S theta_K phi_K alpha D".split()


def make_ref_params(pars: dict) -> RefParams:
    kw = {k: float(pars[k]) for k in PAR_KEYS}
    return RefParams(**kw, backint=int(bool(pars["backint"])), LISA=int(bool(pars["LISA"])))


@dataclass
class MappedTrajectory:
    """Output of the reference front end (AAKpy.cc:20-44): the arrays GenWave takes."""

    steps: int
    e_traj: np.ndarray
    v_map: np.ndarray
    M_map: np.ndarray
    s_map: np.ndarray
    dt_map: np.ndarray
    Phi0: float
    flag: int
    traj: np.ndarray = field(default=None)


def ref_front(pars: dict) -> MappedTrajectory:
    L = ref_lib()
    p = make_ref_params(pars)
    arrs = [np.zeros(100) for _ in range(5)]
    traj = np.zeros(1000)
    steps = ctypes.c_int()
    phi0 = ctypes.c_double()
    flag = L.ref_front(ctypes.byref(p), ctypes.byref(steps), *[_ptr(a) for a in arrs], ctypes.byref(phi0), _ptr(traj))
    n = steps.value
    return MappedTrajectory(n, *[a[:n].copy() for a in arrs], phi0.value, flag, traj[: 10 * n].reshape(n, 10).copy())


def ref_aakwave(pars: dict):
    L = ref_lib()
    p = make_ref_params(pars)
    n = int(pars["length"])
    t, hI, hII = np.zeros(n), np.zeros(n), np.zeros(n)
    secs = L.ref_aakwave(ctypes.byref(p), _ptr(t), _ptr(hI), _ptr(hII))
    return t, hI, hII, secs


def _genwave_args(pars: dict, mt: MappedTrajectory):
    return [
        ctypes.c_double(pars["dt"]),
        ctypes.c_int(int(pars["length"])),
        _ptr(mt.e_traj),
        _ptr(mt.v_map),
        ctypes.c_double(pars["M"]),
        _ptr(mt.M_map),
        ctypes.c_double(pars["mu"]),
        ctypes.c_double(pars["s"]),
        _ptr(mt.s_map),
        ctypes.c_double(pars["D"]),
        ctypes.c_double(pars["iota"]),
        ctypes.c_double(pars["gamma"]),
        ctypes.c_double(mt.Phi0),
        ctypes.c_double(pars["theta_S"]),
        ctypes.c_double(pars["phi_S"]),
        ctypes.c_double(pars["alpha"]),
        ctypes.c_double(pars["theta_K"]),
        ctypes.c_double(pars["phi_K"]),
        _ptr(mt.dt_map),
        ctypes.c_int(mt.steps),
        ctypes.c_int(int(bool(pars["backint"]))),
        ctypes.c_int(int(bool(pars["LISA"]))),
    ]


def ref_genwave(pars: dict, mt: MappedTrajectory, nmodes: int = 0):
    """Reference waveform() on a mapped trajectory, optional harmonic-count override."""
    L = ref_lib()
    n = int(pars["length"])
    t, hI, hII = np.zeros(n), np.zeros(n), np.zeros(n)
    L.ref_genwave(_ptr(t), _ptr(hI), _ptr(hII), *_genwave_args(pars, mt), ctypes.c_int(nmodes))
    return t, hI, hII


def oracle_genwave(pars: dict, mt: MappedTrajectory, nmodes: int = 0):
    """Oracle restatement of the same call; returns (t, hI, hII, i_plunge, i_buffer)."""
    L = oracle_lib()
    n = int(pars["length"])
    t, hI, hII = np.zeros(n), np.zeros(n), np.zeros(n)
    ip, ib = ctypes.c_int(), ctypes.c_int()
    rc = L.oracle_genwave(
        _ptr(t), _ptr(hI), _ptr(hII), *_genwave_args(pars, mt), ctypes.c_int(nmodes), ctypes.byref(ip), ctypes.byref(ib)
    )
    if rc != 0:
        raise ValueError("oracle: fitting error, t_0 too close to plunge")
    return t, hI, hII, ip.value, ib.value


def oracle_genwave_at(pars: dict, mt: MappedTrajectory, idx: np.ndarray, nmodes: int = 0):
    """oracle_genwave at the sample indices idx only (full PNevolution, harmonic
    sums at those samples); returns (hI[idx], hII[idx])."""
    L = oracle_lib()
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    a, b = np.zeros(len(idx)), np.zeros(len(idx))
    rc = L.oracle_genwave_at(*_genwave_args(pars, mt), ctypes.c_int(nmodes),
                             idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.c_int(len(idx)), _ptr(a), _ptr(b))
    if rc != 0:
        raise ValueError("oracle: fitting error, t_0 too close to plunge")
    return a, b


def _pnevo(L, fn, pars, mt):
    n = int(pars["length"])
    outs = [np.zeros(n + 1) for _ in range(10)]
    ip, ib = ctypes.c_int(), ctypes.c_int()
    return n, outs, ip, ib


def oracle_pnevolution(pars: dict, mt: MappedTrajectory):
    """Dense (t, e, v, M, S, gim, Phi, alp, nu, gimdot) from the oracle, plus i_plunge, i_buffer."""
    L = oracle_lib()
    n = int(pars["length"])
    outs = [np.zeros(n + 1) for _ in range(10)]
    ip, ib = ctypes.c_int(), ctypes.c_int()
    par = np.zeros(12)
    par[0] = pars["mu"] * MSUN_SEC
    par[1] = mt.M_map[0] * MSUN_SEC
    par[2] = mt.s_map[0]
    par[3] = mt.e_traj[0]
    par[4] = pars["iota"]
    par[5] = pars["gamma"]
    par[6] = mt.Phi0
    par[11] = pars["alpha"]
    rc = L.oracle_pnevolution(
        *[_ptr(o) for o in outs],
        ctypes.c_double(pars["dt"]),
        ctypes.c_int(n),
        _ptr(par),
        _ptr(mt.e_traj),
        _ptr(mt.v_map),
        ctypes.c_double(pars["M"]),
        _ptr(mt.M_map),
        ctypes.c_double(pars["s"]),
        _ptr(mt.s_map),
        _ptr(mt.dt_map),
        ctypes.c_int(mt.steps),
        ctypes.byref(ip),
        ctypes.byref(ib),
        ctypes.c_int(int(bool(pars["backint"]))),
    )
    if rc != 0:
        raise ValueError("oracle: fitting error, t_0 too close to plunge")
    return outs, ip.value, ib.value


PHASE_KEYS = ("t", "phase_r", "phase_theta", "phase_phi", "omega_r", "omega_theta", "omega_phi", "eccentricity")


def ref_aakphase(pars: dict):
    """Reference AAKphase (src/suite/AAKpy.cc:53-88): the eight arrays of
    PHASE_KEYS and the timing, as AAKwrapper.phase returns them."""
    L = ref_lib()
    p = make_ref_params(pars)
    n = int(pars["length"])
    outs = [np.zeros(n) for _ in PHASE_KEYS]
    L.ref_aakphase.restype = ctypes.c_double
    secs = L.ref_aakphase(ctypes.byref(p), *[_ptr(o) for o in outs])
    return (*outs, secs)


TDI_KEYS = ("f", "Xf_r", "Xf_im", "Yf_r", "Yf_im", "Zf_r", "Zf_im")


def ref_aaktdi(pars: dict):
    """Reference AAKTDI (src/suite/AAKpy.cc:90-125): the seven arrays of TDI_KEYS
    ((length + 1) // 2 bins each) and the timing, as AAKwrapper.tdi returns them."""
    L = ref_lib()
    p = make_ref_params(pars)
    n = (int(pars["length"]) + 1) // 2
    outs = [np.zeros(n) for _ in TDI_KEYS]
    L.ref_aaktdi.restype = ctypes.c_double
    secs = L.ref_aaktdi(ctypes.byref(p), *[_ptr(o) for o in outs])
    return (*outs, secs)


def ref_gentdi(pars: dict, mt: MappedTrajectory):
    """Reference GenTDI (src/suite/AAKTDI.cc:799-829) on a mapped trajectory."""
    L = ref_lib()
    n = (int(pars["length"]) + 1) // 2
    outs = [np.zeros(n) for _ in TDI_KEYS]
    L.ref_gentdi(
        *[_ptr(o) for o in outs], *_genphase_args(pars, mt), ctypes.c_double(pars["D"]),
        ctypes.c_double(pars["iota"]), ctypes.c_double(pars["gamma"]), ctypes.c_double(mt.Phi0),
        ctypes.c_double(pars["theta_S"]), ctypes.c_double(pars["phi_S"]), ctypes.c_double(pars["alpha"]),
        ctypes.c_double(pars["theta_K"]), ctypes.c_double(pars["phi_K"]), _ptr(mt.dt_map), ctypes.c_int(mt.steps),
        ctypes.c_int(int(bool(pars["backint"]))),
    )
    return tuple(outs)


def oracle_gentdi(pars: dict, mt: MappedTrajectory, nmodes: int = 0):
    """The oracle's GenTDI: (TDI_KEYS arrays..., i_plunge of the phase grid)."""
    L = oracle_lib()
    n = (int(pars["length"]) + 1) // 2
    outs = [np.zeros(n) for _ in TDI_KEYS]
    rows = (_dp * 6)(*[_ptr(o) for o in outs[1:]])
    ip = ctypes.c_int()
    rc = L.oracle_gentdi(
        _ptr(outs[0]), rows, *_genphase_args(pars, mt), ctypes.c_double(pars["D"]), ctypes.c_double(pars["iota"]),
        ctypes.c_double(pars["gamma"]), ctypes.c_double(mt.Phi0), ctypes.c_double(pars["theta_S"]),
        ctypes.c_double(pars["phi_S"]), ctypes.c_double(pars["alpha"]), ctypes.c_double(pars["theta_K"]),
        ctypes.c_double(pars["phi_K"]), _ptr(mt.dt_map), ctypes.c_int(mt.steps),
        ctypes.c_int(int(bool(pars["backint"]))), ctypes.c_int(int(nmodes)), ctypes.byref(ip),
    )
    if rc != 0:
        raise ValueError("oracle: fitting error, t_0 too close to plunge")
    return (*outs, ip.value)


def _genphase_args(pars: dict, mt: MappedTrajectory):
    return [
        ctypes.c_double(pars["dt"]),
        ctypes.c_int(int(pars["length"])),
        _ptr(mt.e_traj),
        _ptr(mt.v_map),
        ctypes.c_double(pars["M"]),
        _ptr(mt.M_map),
        ctypes.c_double(pars["mu"]),
        ctypes.c_double(pars["s"]),
        _ptr(mt.s_map),
    ]


def ref_genphase(pars: dict, mt: MappedTrajectory):
    """Reference GenPhase (src/suite/AAKPhase.cc:315-374) on a mapped trajectory."""
    L = ref_lib()
    n = int(pars["length"])
    outs = [np.zeros(n) for _ in PHASE_KEYS]
    L.ref_genphase(
        *[_ptr(o) for o in outs], *_genphase_args(pars, mt), ctypes.c_double(pars["D"]),
        ctypes.c_double(pars["iota"]), ctypes.c_double(pars["gamma"]), ctypes.c_double(mt.Phi0),
        ctypes.c_double(pars["theta_S"]), ctypes.c_double(pars["phi_S"]), ctypes.c_double(pars["alpha"]),
        ctypes.c_double(pars["theta_K"]), ctypes.c_double(pars["phi_K"]), _ptr(mt.dt_map), ctypes.c_int(mt.steps),
        ctypes.c_int(int(bool(pars["backint"]))),
    )
    return tuple(outs)


def oracle_genphase(pars: dict, mt: MappedTrajectory):
    """The oracle's GenPhase: (PHASE_KEYS arrays..., i_plunge, i_buffer)."""
    L = oracle_lib()
    n = int(pars["length"])
    outs = [np.zeros(n) for _ in PHASE_KEYS]
    ip, ib = ctypes.c_int(), ctypes.c_int()
    rc = L.oracle_genphase(
        *[_ptr(o) for o in outs], *_genphase_args(pars, mt), ctypes.c_double(pars["iota"]),
        ctypes.c_double(pars["gamma"]), ctypes.c_double(mt.Phi0), ctypes.c_double(pars["alpha"]), _ptr(mt.dt_map),
        ctypes.c_int(mt.steps), ctypes.c_int(int(bool(pars["backint"]))), ctypes.byref(ip), ctypes.byref(ib),
    )
    if rc != 0:
        raise ValueError("oracle: fitting error, t_0 too close to plunge")
    return (*outs, ip.value, ib.value)


def ref_pnevolution(pars: dict, mt: MappedTrajectory):
    L = ref_lib()
    n = int(pars["length"])
    outs = [np.zeros(n + 1) for _ in range(10)]
    ip, ib = ctypes.c_int(), ctypes.c_int()
    L.ref_pnevolution(
        ctypes.c_double(pars["dt"]),
        ctypes.c_int(n),
        _ptr(mt.e_traj),
        _ptr(mt.v_map),
        ctypes.c_double(pars["M"]),
        _ptr(mt.M_map),
        ctypes.c_double(pars["mu"]),
        ctypes.c_double(pars["s"]),
        _ptr(mt.s_map),
        ctypes.c_double(pars["iota"]),
        ctypes.c_double(pars["gamma"]),
        ctypes.c_double(mt.Phi0),
        ctypes.c_double(pars["alpha"]),
        _ptr(mt.dt_map),
        ctypes.c_int(mt.steps),
        ctypes.c_int(int(bool(pars["backint"]))),
        *[_ptr(o) for o in outs],
        ctypes.byref(ip),
        ctypes.byref(ib),
    )
    return outs, ip.value, ib.value


def oracle_bessel(nmin: int, nmax: int, x: float) -> np.ndarray:
    out = np.zeros(nmax - nmin + 1)
    oracle_lib().oracle_bessel_jn_array(ctypes.c_int(nmin), ctypes.c_int(nmax), ctypes.c_double(x), _ptr(out))
    return out


def oracle_kerr_constants(p, e, cosi, a) -> np.ndarray:
    out = np.zeros(8)
    oracle_lib().oracle_kerr_constants(*[ctypes.c_double(v) for v in (p, e, cosi, a)], _ptr(out))
    return out


def ref_iekg(p, e, cosi, a) -> np.ndarray:
    out = np.zeros(13)
    ref_lib().ref_iekg(*[ctypes.c_double(v) for v in (p, e, cosi, a)], _ptr(out))
    return out


def ref_gkr(p, e, cosi, a) -> np.ndarray:
    out = np.zeros(6)
    ref_lib().ref_gkr(*[ctypes.c_double(v) for v in (p, e, cosi, a)], _ptr(out))
    return out


def ref_ckg(r, cosi, a) -> np.ndarray:
    out = np.zeros(4)
    ref_lib().ref_ckg(*[ctypes.c_double(v) for v in (r, cosi, a)], _ptr(out))
    return out


def ref_lso_table(cosi, a) -> np.ndarray:
    out = np.zeros(4)
    ref_lib().ref_lso_table(ctypes.c_double(cosi), ctypes.c_double(a), _ptr(out))
    return out


def ref_parmap(Omega, p, M, s, e, iota) -> np.ndarray:
    out = np.zeros(3)
    Om = np.ascontiguousarray(Omega, dtype=np.float64)
    ref_lib().ref_parmap(_ptr(out), _ptr(Om), *[ctypes.c_double(v) for v in (p, M, s, e, iota)])
    return out


def ref_pn_rates(v, e, Y, q, m, M) -> np.ndarray:
    out = np.zeros(6)
    ref_lib().ref_pn_rates(*[ctypes.c_double(x) for x in (v, e, Y, q, m, M)], _ptr(out))
    return out


# ----------------------------------------------------------------- likelihood oracle
def lisa_noise(f, L=2.5e9, f_star=19.09e-3, dur=4):
    """Analytic LISA PSD, pygpuAAK/LISAnoise.py:11-43 (restated)."""
    fit = {
        0.5: (0.133, 243, 482, 917, 2.58e-3),
        1: (0.171, 292, 1020, 1680, 2.15e-3),
        2: (0.165, 299, 611, 1340, 1.73e-3),
        4: (0.138, -221, 521, 1680, 1.13e-3),
    }
    f = np.asarray(f, dtype=np.float64)
    P_oms = (1.5e-11) ** 2 * (1 + (2e-3 / f) ** 4)
    P_acc = (3e-15) ** 2 * (1 + (0.4e-3 / f) ** 2) * (1 + (f / 8e-3) ** 4)
    S = 10.0 / (3.0 * L**2) * (P_oms + 2 * (1 + np.cos(f / f_star) ** 2) * P_acc / (2 * np.pi * f) ** 4) * (
        1 + 6 / 10 * (f / f_star) ** 2
    )
    if dur:
        al, be, ka, ga, fk = fit[dur]
        S = S + 9e-45 * f ** (-7 / 3) * np.exp(-(f**al) + be * f * np.sin(ka * f)) * (1 + np.tanh(ga * (fk - f)))
    return S


def noise_weights(length: int, dt: float, dur=1) -> np.ndarray:
    """noise_inv = S_n(f)^{-1/2} sqrt(dt/N), freqs[0] = freqs[1]/10 (pygpuAAK.py:67-96)."""
    n_samples = int(np.round(length * dt / dt))
    nf = int(np.round(n_samples / 2) + 1)
    freqs = np.linspace(0.0, 0.5 / dt, nf)
    freqs[0] = freqs[1] / 10.0
    return 1.0 / np.sqrt(lisa_noise(freqs, dur=dur)) * np.sqrt(dt / length)


def inner_products(hI, hII, data1, data2, w1, w2):
    """[4 Re<h|d>, 4 <h|h>] with data pre-weighted, template weighted by w (AAK_manager.cu:365-446)."""
    HI = np.fft.rfft(np.asarray(hI, dtype=np.float64)) * w1
    HII = np.fft.rfft(np.asarray(hII, dtype=np.float64)) * w2
    d_h = np.real(np.vdot(HI, data1)) + np.real(np.vdot(HII, data2))
    h_h = np.real(np.vdot(HI, HI)) + np.real(np.vdot(HII, HII))
    return np.array([4.0 * d_h, 4.0 * h_h])


def fisher_gram(hI_rows: np.ndarray, hII_rows: np.ndarray, scale: float) -> np.ndarray:
    """Per-channel Gram matrices of the finite-difference derivatives of
    weighted template spectra, as pyGPUAAK.get_Fisher forms them
    (pygpuAAK/pygpuAAK.py:269-300): rows 2i and 2i+1 are the two evaluations of
    derivative i, D_i = scale (row_{2i+1} - row_{2i}), G[c, i, j] = 4 Re
    sum_f conj(D_i) D_j.  Returns (2, nd, nd)."""
    nd = hI_rows.shape[0] // 2
    G = np.zeros((2, nd, nd))
    for c, H in enumerate((hI_rows, hII_rows)):
        D = (H[1::2] - H[0::2]) * scale
        G[c] = 4.0 * np.real(D.conj() @ D.T)
    return G


def fisher_reference_form(G: np.ndarray) -> np.ndarray:
    """The matrix the reference's get_Fisher returns from those Gram sums
    (pygpuAAK/pygpuAAK.py:286-298): for i <= j, M_ij = 4 Re(<D_j^I, D_j^I> +
    <D_i^II, D_j^II>), mirrored to j < i."""
    nd = G.shape[1]
    M = np.zeros((nd, nd))
    for i in range(nd):
        for j in range(i, nd):
            M[i, j] = M[j, i] = G[0, j, j] + G[1, i, j]
    return M
