"""Phase error of the split path's harmonic rotor, per harmonic up to n = 100.

The split kernel forms the harmonic phases exp(i (n Phi' + D0)) in FP32 by the
recurrence w_n = w_{n-1} z_1 from z_1 = exp(i Phi'), where Phi' (the orbital
phase plus the Doppler term) is reduced to [-pi, pi] in FP64 and rounded to
FP32, and re-anchors the rotor every 8th harmonic at exp(i (n Phi' + D0))
with n Phi' + D0 reduced in FP64 (aak_dense.cu: mode_sums_split, pair_step).
This test emulates that arithmetic in numpy float32 (IEEE rounding of every
product and sum; sin/cos of the FP32 argument rounded once, standing in for
sincosf, plus the documented 2^-21.41 absolute error of __sincosf on the
anchors) against an extended-precision reference, and states the error per
harmonic with and without the anchors."""
import numpy as np

F = np.float32
SINCOSF_FAST_ERR = 2.0 ** -21.41  # __sincosf on [-pi, pi], CUDA's documented bound


def _reduce(x):
    """x mod 2 pi in [-pi, pi] in extended precision (the kernel does it in FP64)."""
    x = np.asarray(x, dtype=np.longdouble)
    tp = 2 * np.pi * np.longdouble(1)
    return x - np.rint(x / tp) * tp


def _errors(nmax, anchor_every, rng, nsamp=4000):
    phi = rng.uniform(0, 2e7, nsamp).astype(np.float64)  # up to 1e7 cycles of accumulated phase
    d0 = rng.uniform(-5e-3, 5e-3, nsamp).astype(np.float64)
    r1 = np.asarray(_reduce(phi), dtype=np.float64)  # FP64 reduction of Phi'
    a1 = r1.astype(F)
    c1, s1 = np.cos(a1.astype(np.float64)).astype(F), np.sin(a1.astype(np.float64)).astype(F)
    zr, zi = np.cos(F(d0).astype(np.float64)).astype(F), np.sin(F(d0).astype(np.float64)).astype(F)
    worst = np.zeros(nmax + 1)
    for n in range(1, nmax + 1):
        if anchor_every and n % anchor_every == 0:
            arg = np.asarray(_reduce(np.longdouble(n) * r1.astype(np.longdouble) + d0), dtype=np.float64).astype(F)
            zr = np.cos(arg.astype(np.float64)).astype(F)
            zi = np.sin(arg.astype(np.float64)).astype(F)
            extra = SINCOSF_FAST_ERR
        else:
            tr = (zr * c1).astype(F) - (zi * s1).astype(F)
            zi = ((zr * s1).astype(F) + (zi * c1).astype(F)).astype(F)
            zr = tr.astype(F)
            extra = 0.0
        exact = _reduce(np.longdouble(n) * phi.astype(np.longdouble) + d0)
        got = np.arctan2(zi.astype(np.float64), zr.astype(np.float64))
        err = np.abs(np.asarray(_reduce(got - exact), dtype=np.float64))
        worst[n] = err.max() + extra
    return worst


def test_rotor_phase_error_per_harmonic():
    rng = np.random.default_rng(3)
    plain = _errors(100, 0, rng)
    anchored = _errors(100, 8, np.random.default_rng(3))
    print("max phase error (rad) at n = 10, 30, 61, 100: recurrence only",
          [float(plain[n]) for n in (10, 30, 61, 100)], "with FP64 anchors every 8",
          [float(anchored[n]) for n in (10, 30, 61, 100)])
    # without anchors the error grows with n (about 1e-5 rad at n = 100)
    assert plain[100] > 4 * plain[8]
    # with them it stays at the level of a few FP32 rounding steps for every n
    assert anchored[1:].max() < 1.5e-6
    assert anchored[100] < plain[100] / 3
