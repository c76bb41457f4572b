"""Batch planning runs the coarse AK evolutions of four sources at once (the
lanes of one AVX2 vector where the CPU has them, performing each source's
scalar operations in the same order).  A batch plan must therefore equal the
plans of the same sources planned one per batch (where each source's
evolution runs alone): status, offsets, plunge index and buffer length, on a
host-only context (no GPU)."""
import numpy as np

import emri_kludge_suite_b200 as E
from emri_kludge_suite_b200.workloads import config1


def _sources(n):
    src, _ = config1(29, 64)
    out = []
    for p in src[:n]:
        q = dict(p)
        q["length"] = min(int(p["length"]), 300000)
        out.append(q)
    out[3] = dict(out[3], e=-0.2)  # invalid: its group-mates must be unaffected
    return out


def _fields(wb):
    return wb.status.copy(), np.diff(wb.offsets), wb.i_plunge.copy(), wb.i_buffer.copy()


def test_grouped_batch_plan_equals_single_plans():
    params = _sources(22)  # five groups of four and a remainder of two
    wb = E.WaveBatch(-1)
    wb.plan(params, nmodes=30, nthreads=3)
    batch = _fields(wb)
    single = [[] for _ in range(4)]
    for p in params:
        w1 = E.WaveBatch(-1)
        w1.plan([p], nmodes=30, nthreads=1)
        for k, f in enumerate(_fields(w1)):
            single[k].append(f[0])
    assert batch[0][3] != 0
    for k in range(4):
        assert np.array_equal(batch[k], np.array(single[k])), k
