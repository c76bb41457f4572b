"""Generate tests/golden/*.npz from the reference itself.

Runs the reference AAK code compiled from its own sources (oracle/_ref/
libaakref.so, ``make -C oracle ref``) on a few small parameter sets and
stores its outputs: the mapped trajectory of the front end
(src/suite/AAKpy.cc:20-44), the waveform of AAKwave with the reference
harmonic rule, the waveform of waveform() with a harmonic-count override, the
seven phase arrays of AAKphase (src/suite/AAKpy.cc:53-88, whose time array is
the AAKwave one), the six frequency-domain TDI arrays of AAKTDI
(src/suite/AAKpy.cc:90-125, on f = i / ((length - 1) dt)), and for some cases
the dense PNevolution arrays (src/suite/AAK.cc:27-318).

    python tests/golden/make_golden.py

The fixtures are inputs/outputs of the reference; nothing in them is
produced by the product library.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import oracle as O  # noqa: E402

BASE = dict(backint=False, LISA=True, dt=10.0, p=8.0, T=0.25, f=2e-3, T_fit=1.0, mu=10.0, M=1e6, s=0.5, e=0.2,
            iota=0.785, gamma=0.0, psi=0.0, theta_S=0.5, phi_S=1.0, theta_K=0.8, phi_K=2.0, alpha=0.0, D=1.0)

CASES = {
    # configuration-0 source, short span
    "cfg0_short": dict(length=8000, nmodes=30, dense=True),
    # plunges inside the span: exercises the plunge search, the 10-orbit buffer and the Planck taper
    "plunge": dict(p=6.0, mu=100.0, e=0.2, dt=100.0, length=4000, nmodes=10, gamma=0.3, psi=0.2, alpha=0.4, dense=True),
    # same with backward integration from the plunge (backint)
    "plunge_backint": dict(p=6.0, mu=100.0, e=0.2, dt=100.0, length=4000, nmodes=10, gamma=0.3, psi=0.2, alpha=0.4,
                           backint=True, dense=True),
    # retrograde, detector-frame response (LISA off), different masses and spacing
    "retro_nolisa": dict(p=10.5, mu=30.0, M=3e5, e=0.4, s=0.7, iota=2.0, LISA=False, dt=15.0, length=6000, nmodes=20,
                         theta_S=1.9, phi_S=4.0, theta_K=0.3, phi_K=5.5, gamma=1.1, psi=2.0, alpha=0.7, D=2.0),
    # high eccentricity, many harmonics, high spin
    "high_e": dict(p=20.0, e=0.7, s=0.9, iota=0.3, length=5000, nmodes=61, psi=1.0),
}


def run_case(name, spec):
    pars = dict(BASE)
    spec = dict(spec)
    nmodes = spec.pop("nmodes")
    dense = spec.pop("dense", False)
    pars.update(spec)
    pars["T"] = pars["length"] * pars["dt"] / O.YEAR
    mt = O.ref_front(pars)
    t_w, hI_w, hII_w, _ = O.ref_aakwave(pars)
    t_g, hI_g, hII_g = O.ref_genwave(pars, mt, nmodes)
    phase = O.ref_aakphase(pars)
    assert np.array_equal(phase[0], t_w)
    tdi = O.ref_aaktdi(pars)
    out = dict(
        pars=json.dumps(pars),
        nmodes=np.int32(nmodes),
        steps=np.int32(mt.steps),
        e_traj=mt.e_traj,
        v_map=mt.v_map,
        M_map=mt.M_map,
        s_map=mt.s_map,
        dt_map=mt.dt_map,
        Phi0=np.float64(mt.Phi0),
        traj=mt.traj,
        aakwave_t=t_w,
        aakwave_hI=hI_w,
        aakwave_hII=hII_w,
        genwave_t=t_g,
        genwave_hI=hI_g,
        genwave_hII=hII_g,
    )
    for k, a in zip(O.PHASE_KEYS[1:], phase[1:8]):
        out["aakphase_" + k] = a
    for k, a in zip(O.TDI_KEYS[1:], tdi[1:7]):
        out["aaktdi_" + k] = a
    if dense:
        arrs, ip, ib = O.ref_pnevolution(pars, mt)
        for k, a in zip("t e v M S gim Phi alp nu gimdot".split(), arrs):
            out["dense_" + k] = a
        out["i_plunge"] = np.int32(ip)
        out["i_buffer"] = np.int32(ib)
    return out


def main():
    manifest = {}
    for name, spec in CASES.items():
        out = run_case(name, spec)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        manifest[name] = hashlib.sha256(open(path, "rb").read()).hexdigest()
        print(name, os.path.getsize(path), manifest[name][:16])
    with open(os.path.join(HERE, "MANIFEST.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
