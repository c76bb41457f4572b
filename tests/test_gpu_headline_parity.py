"""Full-length benchmark sources through the batched FP64 and split-precision
paths, against the FP64 oracle and the reference.

The sources are tests/golden/headline/*.npz (configuration 1: the longest,
3.15e6 samples; the largest M; the smallest mu; the highest spin; the most
retrograde; one with backint; configuration 2: the most harmonics, 61; the
longest), with the reference's mapped trajectories.  For each source, both
paths run in one batch through the C ABI and are compared with the oracle's
FP64 waveform over every sample: overlap mismatch flat and LISA-noise weighted,
and max|dh|/max|h|.  End to end, the product's own front end feeds the
batched paths for two sources, against the oracle on the reference's mapped
trajectory.  Set AAK_PARITY_REPORT=<file> to write the per-source figures."""
import json
import os

import numpy as np
import pytest

from conftest import mismatch, psd_mismatch
from test_oracle_headline_pin import HEADLINE, load_headline

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
import emri_kludge_suite_b200 as E  # noqa: E402
from emri_kludge_suite_b200.aak import Mapped  # noqa: E402
from oracle import oracle as O  # noqa: E402

# bars: the north-star mismatch bar for both paths; max|dh|/max|h| of the FP64
# path at the level of its Bessel evaluation, of the split path at its FP32
# harmonic sums
MM_BAR = 1e-6
FP64_MM, FP64_REL = 1e-10, 1e-7
SPLIT_REL = 1e-3
REPORT = {}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    O.set_threads(os.cpu_count() or 1)
    yield
    O.set_threads(1)
    path = os.environ.get("AAK_PARITY_REPORT")
    if path:
        with open(path, "w") as f:
            json.dump(REPORT, f, indent=1, sort_keys=True)


def _mapped(mt):
    return Mapped(mt.steps, mt.e_traj, mt.v_map, mt.M_map, mt.s_map, mt.dt_map, mt.Phi0, 2, 0)


def _run(wb, precision):
    N = wb.total_samples
    hI = torch.zeros(N, dtype=torch.float64, device="cuda")
    hII = torch.zeros_like(hI)
    wb.run(hI.data_ptr(), hII.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    assert wb.device_status() == 0
    return hI.cpu().numpy(), hII.cpu().numpy()


def _metrics(x1, x2, o1, o2, dt):
    scale = max(np.abs(o1).max(), np.abs(o2).max())
    return {"mismatch_flat": float(mismatch(x1, x2, o1, o2)), "mismatch_psd": float(psd_mismatch(x1, x2, o1, o2, dt)),
            "max_rel_dh": float(max(np.abs(x1 - o1).max(), np.abs(x2 - o2).max()) / scale)}


def test_full_length_batched_paths_against_oracle():
    ds = [load_headline(p) for p in HEADLINE]
    assert len(ds) == 8
    wb = E.WaveBatch(0)
    wb.plan([d["pars"] for d in ds], nmodes=[int(d["nmodes"]) for d in ds], mapped=[_mapped(d["mapped"]) for d in ds])
    assert np.all(wb.status == 0)
    wb.upload()
    f64, f32 = _run(wb, 0), _run(wb, 1)
    o = wb.offsets
    bad = []
    for k, (path, d) in enumerate(zip(HEADLINE, ds)):
        name = os.path.basename(path)[:-4]
        t, oI, oII, ip, ib = O.oracle_genwave(d["pars"], d["mapped"], int(d["nmodes"]))
        assert wb.i_plunge[k] == ip
        sl = slice(o[k], o[k + 1])
        m64 = _metrics(f64[0][sl], f64[1][sl], oI, oII, d["pars"]["dt"])
        m32 = _metrics(f32[0][sl], f32[1][sl], oI, oII, d["pars"]["dt"])
        REPORT[name] = {"samples": len(t), "nmodes": int(d["nmodes"]), "fp64": m64, "split": m32}
        print(name, len(t), int(d["nmodes"]), m64, m32)
        if not (m64["mismatch_flat"] <= FP64_MM and m64["mismatch_psd"] <= FP64_MM and m64["max_rel_dh"] <= FP64_REL):
            bad.append((name, "fp64", m64))
        if not (m32["mismatch_flat"] <= MM_BAR and m32["mismatch_psd"] <= MM_BAR and m32["max_rel_dh"] <= SPLIT_REL):
            bad.append((name, "split", m32))
        # and the reference's own samples
        idx = d["idx"]
        scale = max(np.abs(d["ref_hI"]).max(), np.abs(d["ref_hII"]).max())
        assert np.abs(f64[0][sl][idx] - d["ref_hI"]).max() <= FP64_REL * scale, name
        assert np.abs(f64[1][sl][idx] - d["ref_hII"]).max() <= FP64_REL * scale, name
    assert not bad, bad


@pytest.mark.parametrize("name", ["c1_longest", "c1_retrograde"])
def test_end_to_end_own_front_end_against_oracle_on_reference_map(name):
    path = [p for p in HEADLINE if os.path.basename(p)[:-4] == name][0]
    d = load_headline(path)
    wb = E.WaveBatch(0)
    wb.plan([d["pars"]], nmodes=int(d["nmodes"]))  # the product's own front end
    assert wb.status[0] == 0
    wb.upload()
    t, oI, oII, ip, ib = O.oracle_genwave(d["pars"], d["mapped"], int(d["nmodes"]))
    for prec in (0, 1):
        hI, hII = _run(wb, prec)
        m = _metrics(hI, hII, oI, oII, d["pars"]["dt"])
        REPORT[f"{name}_end_to_end_{'split' if prec else 'fp64'}"] = m
        print(name, "end to end", prec, m)
        assert m["mismatch_flat"] <= MM_BAR and m["mismatch_psd"] <= MM_BAR, m
