"""The C ABI: the library loads, exports every entry point include/aak.h declares,
and fails with a status code (never a process exit) without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO, cuda_available
from emri_kludge_suite_b200 import _lib


def declared_functions():
    src = open(os.path.join(REPO, "include", "aak.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aak_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_status_strings():
    L = _lib.lib()
    for s in range(0, 10):
        assert L.aak_status_string(s) != b"unknown status"


@pytest.mark.skipif(cuda_available(), reason="checks the no-GPU error path")
def test_gpu_entry_points_fail_loudly_without_gpu():
    import emri_kludge_suite_b200 as E

    pars = dict(backint=False, LISA=True, length=100, dt=10.0, p=8.0, T=0.25, f=2e-3, T_fit=1.0, mu=10.0, M=1e6, s=0.5,
                e=0.2, iota=0.785, gamma=0.0, psi=0.0, theta_S=0.5, phi_S=1.0, theta_K=0.8, phi_K=2.0, alpha=0.0, D=1.0)
    with pytest.raises(_lib.AAKError) as ex:
        E.wave(pars)
    assert ex.value.status == 5
    with pytest.raises(_lib.AAKError):
        E.WaveBatch(0)
    from emri_kludge_suite_b200.parmap_mlp import ParMapMLP

    with pytest.raises(_lib.AAKError) as ex:
        ParMapMLP(0)
    assert ex.value.status == 5


def test_host_only_context_plans_without_gpu():
    import emri_kludge_suite_b200 as E

    pars = dict(backint=False, LISA=True, length=20000, dt=10.0, p=8.0, T=0.25, f=2e-3, T_fit=1.0, mu=10.0, M=1e6,
                s=0.5, e=0.2, iota=0.785, gamma=0.0, psi=0.0, theta_S=0.5, phi_S=1.0, theta_K=0.8, phi_K=2.0, alpha=0.0,
                D=1.0)
    wb = E.WaveBatch(-1)
    wb.plan([pars, dict(pars, e=0.3, length=30000)], nmodes=[30, 30], nthreads=2)
    assert list(wb.status) == [0, 0]
    assert wb.total_samples == 50000
    st = wb.newton_stats()
    assert st["points"] > 0 and st["iterations"] >= st["points"] and st["fallbacks"] == 0
    with pytest.raises(_lib.AAKError) as ex:
        wb.upload()
    assert ex.value.status == 1


def test_null_arguments_are_rejected():
    L = _lib.lib()
    assert L.aak_front_end(None, None, None) == 1
    assert L.aak_wave(None, None, None, None, None) == 1
    assert L.aak_batch_plan(None, None, 0, None, 0) == 1
