"""One batch over several GPUs: split by greedy LPT, no data-path exchange.

The reference's ``pyGPUAAK`` accepts ``ndevices`` but evaluates every template
on one device in a serial loop (pygpuAAK/pygpuAAK.py:31, 204-232).  Here a
caller's batch of sources (cost = samples x harmonics) or likelihood templates
(equal costs) is divided over devices with :func:`lpt_partition`
(``aak_lpt_partition``); every device plans and generates its own units, and
only per-unit results come back (waveform rows, or the (4<h|d>, 4<h|h>) pair
of a template), reassembled in the caller's order.

* :class:`MultiDeviceWaveBatch` and :class:`MultiDeviceGPUAAK`: one process
  driving several devices (one host thread per device; the C ABI releases the
  GIL during its calls).
* :func:`rank_indices` and :func:`gather_rows`: one process per GPU under
  ``torch.distributed`` -- every rank computes the same split from the same
  list, works on its own part, and the per-unit rows are gathered with one
  all-gather (NCCL over NVLink on GPUs, gloo on the CPU).
"""
from __future__ import annotations

import ctypes
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from ._lib import check, lib, params_array, ptr  # noqa: F401


def _bind():
    return lib()


def source_costs(params, nmodes=None) -> np.ndarray:
    """Device cost of each source: its samples x harmonics (the reference
    harmonic rule int(30 e), at least 4, where nmodes is not given)."""
    n = len(params)
    if nmodes is None:
        nm = np.array([4 if p["e"] < 0.135 else max(int(30 * p["e"]), 1) for p in params], dtype=np.float64)
    else:
        nm = np.broadcast_to(np.asarray(nmodes, dtype=np.float64), (n,))
    return np.array([float(p["length"]) for p in params]) * nm


def lpt_partition(costs, parts: int):
    """assign[i] in [0, parts) for each unit and the summed cost per part."""
    c = np.ascontiguousarray(costs, dtype=np.float64)
    assign = np.zeros(len(c), dtype=np.int32)
    load = np.zeros(int(parts), dtype=np.float64)
    check(_bind().aak_lpt_partition(ptr(c) if len(c) else None, len(c), int(parts), ptr(assign), ptr(load)),
          "aak_lpt_partition")
    return assign, load


def rank_indices(costs, rank: int, world: int) -> np.ndarray:
    """The units of `rank` in the LPT split of the whole list over `world` ranks
    (every rank computes the same split), in the caller's order."""
    assign, _ = lpt_partition(costs, world)
    return np.flatnonzero(assign == rank)


def gather_rows(rows, idx, n: int, group=None):
    """Reassemble per-unit rows from all ranks: rank r holds rows[k] of unit
    idx[k].  Returns the (n, ...) array in the caller's order on every rank.
    One all-gather of a fixed-size buffer (n rows, zero where the rank has no
    unit) -- the only collective of the split."""
    import torch
    import torch.distributed as dist

    rows = np.asarray(rows, dtype=np.float64)
    shape = (n,) + rows.shape[1:]
    buf = np.zeros(shape)
    own = np.zeros(n)
    if len(idx):
        buf[np.asarray(idx)] = rows
        own[np.asarray(idx)] = 1.0
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.from_numpy(np.concatenate([buf.reshape(n, -1), own[:, None]], axis=1)).to(dev)
    world = dist.get_world_size(group)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    full = sum(o.cpu().numpy() for o in out)
    if not np.all(full[:, -1] == 1.0):
        raise RuntimeError("gather_rows: every unit must belong to exactly one rank")
    return full[:, :-1].reshape(shape)


class MultiDeviceWaveBatch:
    """generate_host over several devices: LPT split by samples x harmonics,
    one WaveBatch (and host thread) per device, outputs in the caller's order."""

    def __init__(self, devices):
        from .aak import WaveBatch

        self.devices = list(devices)
        self.batches = [WaveBatch(d) for d in self.devices]

    def set_precision(self, precision: int):
        for b in self.batches:
            b.set_precision(precision)

    def close(self):
        for b in self.batches:
            b.close()

    def generate_host(self, params, nmodes=None, nthreads: int = 0):
        """Returns (hI, hII, offsets, status) laid out as WaveBatch.generate_host
        would for the whole list on one device."""
        n = len(params)
        nm = None if nmodes is None else np.broadcast_to(np.asarray(nmodes, dtype=np.int32), (n,))
        assign, _ = lpt_partition(source_costs(params, nm), len(self.devices))
        parts = [np.flatnonzero(assign == k) for k in range(len(self.devices))]
        per = max(1, int(nthreads) // len(self.devices)) if nthreads else 0

        def work(k):
            idx = parts[k]
            if len(idx) == 0:
                return None
            return self.batches[k].generate_host([params[i] for i in idx], None if nm is None else nm[idx], per)

        with ThreadPoolExecutor(len(self.devices)) as ex:
            res = list(ex.map(work, range(len(self.devices))))
        lengths = np.array([int(p["length"]) for p in params], dtype=np.int64)
        offs = np.zeros(n + 1, dtype=np.int64)
        offs[1:] = np.cumsum(lengths)
        hI, hII = np.zeros(int(offs[-1])), np.zeros(int(offs[-1]))
        st = np.zeros(n, dtype=np.int32)
        for k, r in enumerate(res):
            if r is None:
                continue
            aI, aII, ao, ast = r
            for j, i in enumerate(parts[k]):
                hI[offs[i]:offs[i + 1]] = aI[ao[j]:ao[j + 1]]
                hII[offs[i]:offs[i + 1]] = aII[ao[j]:ao[j + 1]]
                st[i] = ast[j]
        return hI, hII, offs, st


class MultiDeviceGPUAAK:
    """GPUAAK.likelihood_batch over several devices: the data and weights are
    replicated on every device, templates are split by LPT (equal costs: a
    balanced split of the counts) and generated, transformed and reduced on
    their own devices at once; the (4<h|d>, 4<h|h>) rows are reassembled in the
    caller's order."""

    def __init__(self, devices, T_fit, init_length, length, init_dt, dt, LISA, backint):
        import torch

        from .gpuAAK import GPUAAK

        self.devices = list(devices)
        self.gens = []
        for d in self.devices:
            torch.cuda.set_device(d)
            self.gens.append(GPUAAK(T_fit, init_length, length, init_dt, dt, LISA, backint))
        torch.cuda.set_device(self.devices[0])

    def input_data(self, hI_f, hII_f, w1, w2):
        for g in self.gens:
            g.input_data(hI_f, hII_f, w1, w2)

    def set_precision(self, precision: int):
        for g in self.gens:
            g.set_precision(precision)

    def __getattr__(self, name):
        # single-template calls (gpu_gen_AAK, Likelihood, GetWaveform, fisher_gram, ...) run on the first device
        return getattr(self.__dict__["gens"][0], name)

    def likelihood_batch(self, params, max_batch=256, nthreads=0, return_status=False):
        x = np.ascontiguousarray(np.atleast_2d(params), dtype=np.float64)
        n = x.shape[0]
        assign, _ = lpt_partition(np.ones(n), len(self.gens))
        parts = [np.flatnonzero(assign == k) for k in range(len(self.gens))]
        per = max(1, int(nthreads) // len(self.gens)) if nthreads else 0

        def work(k):
            if len(parts[k]) == 0:
                return None
            return self.gens[k].likelihood_batch(x[parts[k]], max_batch=max_batch, nthreads=per, return_status=True)

        with ThreadPoolExecutor(len(self.gens)) as ex:
            res = list(ex.map(work, range(len(self.gens))))
        out = np.zeros((n, 2))
        st = np.zeros(n, dtype=np.int32)
        for k, r in enumerate(res):
            if r is not None:
                out[parts[k]], st[parts[k]] = r
        return (out, st) if return_status else out

    def fisher_gram_batch(self, params, scale, nthreads=0, return_status=False):
        """GPUAAK.fisher_gram_batch with the points split over the devices
        (equal costs: a balanced split of the counts); the Gram matrices are
        reassembled in the caller's order."""
        x = np.ascontiguousarray(params, dtype=np.float64)
        if x.ndim != 3 or x.shape[2] != 14 or x.shape[1] % 2:
            raise ValueError("params must be (npts, 2 nd, 14) in gpu_gen_AAK order")
        n, nd = x.shape[0], x.shape[1] // 2
        assign, _ = lpt_partition(np.ones(n), len(self.gens))
        parts = [np.flatnonzero(assign == k) for k in range(len(self.gens))]
        per = max(1, int(nthreads) // len(self.gens)) if nthreads else 0

        def work(k):
            if len(parts[k]) == 0:
                return None
            return self.gens[k].fisher_gram_batch(x[parts[k]], scale, nthreads=per, return_status=True)

        with ThreadPoolExecutor(len(self.gens)) as ex:
            res = list(ex.map(work, range(len(self.gens))))
        G = np.zeros((n, 2, nd, nd))
        st = np.zeros((n, 2 * nd), dtype=np.int32)
        for k, r in enumerate(res):
            if r is not None:
                G[parts[k]], st[parts[k]] = r
        return (G, st) if return_status else G
