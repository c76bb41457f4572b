"""LISA_Noise, generate_noise_frequencies and generate_noise_single_channel
against the reference's own pygpuAAK/LISAnoise.py (fixture
tests/golden/psd/lisa_noise.npz, made by tests/golden/psd/make_lisa_noise.py).
The oracle's restatement (oracle.lisa_noise) is pinned to the same values."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from emri_kludge_suite_b200 import LISAnoise as LN
from oracle import oracle as O

Z = np.load(os.path.join(GOLDEN, "psd", "lisa_noise.npz"))


@pytest.mark.parametrize("dur", [0, 0.5, 1, 2, 4])
def test_psd_matches_reference(dur):
    f = Z["f"]
    ref = Z[f"S_dur{dur}"]
    np.testing.assert_allclose(LN.LISA_Noise(f, dur=dur), ref, rtol=1e-14, atol=0)
    np.testing.assert_allclose(O.lisa_noise(f, dur=dur), ref, rtol=1e-14, atol=0)


def test_psd_other_arm_and_transfer_frequency():
    f = Z["f"]
    np.testing.assert_allclose(LN.LISA_Noise(f, L=2.0e9, f_star=0.025, dur=1), Z["S_L2e9_fstar0.025_dur1"], rtol=1e-14)
    np.testing.assert_allclose(O.lisa_noise(f, L=2.0e9, f_star=0.025, dur=1), Z["S_L2e9_fstar0.025_dur1"], rtol=1e-14)


def test_noise_frequencies_match_reference():
    fq = LN.generate_noise_frequencies(3_200_000 * 10.0, 0.1)
    assert len(fq) == int(Z["freqs_cfg4_len"][0])
    assert np.array_equal(fq[Z["freqs_cfg4_idx"]], Z["freqs_cfg4_at"])


def test_noise_draw_scale_matches_reference():
    fr = np.linspace(1e-4, 1e-2, 200_000)
    n = LN.generate_noise_single_channel(LN.LISA_Noise, [], {"dur": 1}, 1e-7, fr, np.random.default_rng(7))
    ratio = np.mean(np.abs(n) ** 2 / LN.LISA_Noise(fr, dur=1))
    ref = float(Z["noise_abs2_over_S"][0])
    # E|n|^2 / S = 2 (0.5 / sqrt(df))^2 = 0.5 / df; 200,000 draws: 0.3 % standard error
    assert abs(ratio / ref - 1.0) < 0.02
    assert abs(ratio * 1e-7 / 0.5 - 1.0) < 0.02


def test_bad_duration_raises():
    with pytest.raises(ValueError):
        LN.S_c(np.array([1e-3]), dur=3)
