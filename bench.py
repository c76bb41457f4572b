#!/usr/bin/env python
"""AAK waveform throughput on B200 (one JSON line on rank 0).

Workload (configuration 1 of the AAK benchmark): 512 sources drawn from a
fixed seed -- log10 M ~ U(5,7) Msun, mu ~ U(1,100) Msun, a ~ U(0,0.95),
e0 ~ U(0.05,0.5), cos(iota) ~ U(-1,1), isotropic sky and spin directions,
phases ~ U(0,2pi), D = 1 Gpc, T ~ U(0.1,1) yr, dt = 10 s, harmonics n = 1..30,
LISA response, FP64 throughout; p0 chosen so that the source does not plunge
within T (checked on the planned trajectory, redrawn otherwise).

A step is one pass of the dense AAK path over the whole batch.
  value : samples/s of the GPU kernels with the planned batch resident in HBM
  e2e   : samples/s through the C ABI (aak_wave_batch_host) with host
          parameters in and pinned host waveforms out: host front end and
          coarse evolution on all host threads, H2D, kernels, D2H
  --impl reference : the reference's own CPU AAK (oracle/_ref, compiled from
          its sources) on all host cores, same workload, bounded sample.

Multi-GPU (torchrun, one rank per GPU): one caller batch of 512 x N sources
(and 4096 x N likelihood templates) is split over the ranks by greedy LPT on
samples x harmonics; no collective on the data path, one all-gather of the
per-template (4<h|d>, 4<h|h>) rows; value is the total over ranks divided by
the max-over-ranks device time ("weak" scaling: 512 sources per GPU).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import resource
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

from emri_kludge_suite_b200.workloads import DT, MSUN_SEC, NMODES, SEED, YEAR, config1, config2, draw_source  # noqa: E402


# ----------------------------------------------------------------------------- workload
# Algorithmic work of the harmonic sum, in the convention of the FP32/FP64 FMA
# probes (every multiply and every add one flop, an FMA two): per harmonic the
# reference's algebra of src/suite/AAK.cc:484-526 (Doppler phase, the a, b, c
# combinations, A+, Ax, the NK-frame rotation and the two responses: 24
# FMA-equivalents = 48 flops) and three Bessel recurrence steps (2 flops each);
# 60 flops per sample outside the harmonic loop.  Transcendentals (sin/cos of
# n Phi, the Bessel seeds) are SFU work and not counted.
FLOPS_PER_SAMPLE_BASE = 60.0
FLOPS_PER_HARMONIC = 48.0 + 6.0


def flops_per_sample(nmodes: float) -> float:
    return FLOPS_PER_SAMPLE_BASE + FLOPS_PER_HARMONIC * nmodes


def bench_config(nsrc: int, world: int) -> dict:
    """The workload description both arms print (same keys and values)."""
    return {"workload": f"config1: {nsrc} AAK sources/GPU, T~U(0.1,1) yr, dt=10 s, n=1..30, LISA response",
            "nsrc_per_gpu": nsrc, "nmodes": NMODES, "seed": SEED, "dt_s": DT,
            "l2": "outputs 16 B/sample x ~8.7e8 samples per GPU exceed the 126 MB L2",
            "parallelism": f"sources sharded, {world} rank(s)"}


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax.append(float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ----------------------------------------------------------------------------- CPU reference
def _ref_worker(args):
    """Run the reference AAK (front end + waveform with n = 1..30) until the time budget is used."""
    tasks, budget = args
    sys.path.insert(0, REPO)
    from oracle import oracle as O

    samples, busy, done = 0, 0.0, 0
    t_start = time.perf_counter()
    for pars in tasks:
        if time.perf_counter() - t_start > budget:
            break
        t0 = time.perf_counter()
        mt = O.ref_front(pars)
        if mt.steps < 3:
            continue
        O.ref_genwave(pars, mt, NMODES)
        busy += time.perf_counter() - t0
        samples += int(pars["length"])
        done += 1
    return samples, busy, done


def cpu_reference(sources, budget_s: float = 15.0, sample_len: int = 20000, procs: int = 0,
                  untruncated: bool = False) -> dict:
    """Reference CPU AAK throughput on the host cores (spawn pool; the reference is not thread-safe).

    The bounded sample truncates the configuration-1 sources to sample_len
    samples, which spreads each source's fixed front-end cost (LSO search,
    Kerr constants, the map solve) over fewer samples than at full length.
    untruncated=True also times the procs shortest sources at their full
    length (one per process) as a check on that bias."""
    import multiprocessing as mp

    from oracle import oracle as O

    if not O.ref_available():
        raise RuntimeError("oracle/_ref/libaakref.so is not built")
    procs = procs or (os.cpu_count() or 1)
    # bounded sample: the config-1 sources truncated to sample_len samples each
    tasks = []
    for p in sources:
        q = dict(p)
        q["length"] = min(int(p["length"]), sample_len)
        q["T"] = q["length"] * q["dt"] / YEAR
        tasks.append(q)
    per = [tasks[i::procs] for i in range(procs)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [(t, budget_s) for t in per])
        full = None
        if untruncated:
            short = sorted(sources, key=lambda p: int(p["length"]))[:procs]
            rf = pool.map(_ref_worker, [([p], 1e9) for p in short])
            fs, fb = sum(r[0] for r in rf), max(r[1] for r in rf)
            full = {"value": fs / fb if fb > 0 else 0.0, "unit": "samples/s", "sources": sum(r[2] for r in rf),
                    "samples": fs, "sample": f"the {procs} shortest config-1 sources at full length "
                                              f"({min(int(p['length']) for p in short)}-"
                                              f"{max(int(p['length']) for p in short)} samples), one per process"}
    wall = time.perf_counter() - t0
    samples = sum(r[0] for r in res)
    busy = max(r[1] for r in res)
    done = sum(r[2] for r in res)
    out = {"value": samples / busy if busy > 0 else 0.0, "unit": "samples/s", "cores": procs, "kind": "reference",
           "sample": f"{done} config-1 sources truncated to {sample_len} samples, front end + waveform() with "
                     f"n=1..{NMODES} (reference AAK, GSL shim with Jn_array as a downward recurrence), "
                     f"{procs} processes, {budget_s:.0f} s budget each",
           "wall_s": wall}
    if full is not None:
        out["untruncated"] = full
    return out


def _ref_like_worker(args):
    """One process: the reference AAKwave on the configuration-4 fiducial source
    truncated to sample_len samples, then one full-length FP64 rFFT inner
    product of both channels with the data (pyGPUAAK.NLL's host work per
    template, pygpuAAK.py:204-232)."""
    sample_len, length = args
    sys.path.insert(0, REPO)
    from oracle import oracle as O

    iota, s_, p, e, M, mu, gamma, psi, alph, thS, phS, thK, phK, D = FIDUCIAL
    pars = dict(backint=False, LISA=True, length=sample_len, dt=DT, p=p, T=sample_len * DT / YEAR, f=0.0, T_fit=1.0,
                mu=mu, M=M, s=s_, e=e, iota=iota, gamma=gamma, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK,
                phi_K=phK, alpha=alph, D=D)
    O.ref_aakwave(pars)  # warm-up
    t0 = time.perf_counter()
    O.ref_aakwave(pars)
    rate = sample_len / (time.perf_counter() - t0)
    rng = np.random.default_rng(1)
    hI, hII = rng.standard_normal(length), rng.standard_normal(length)
    nb = length // 2 + 1
    dI, dII = rng.standard_normal(nb) + 1j * rng.standard_normal(nb), rng.standard_normal(nb) + 1j * rng.standard_normal(nb)
    w = rng.random(nb)
    t0 = time.perf_counter()
    fI, fII = np.fft.rfft(hI) * w, np.fft.rfft(hII) * w
    d_h = 4.0 * float(np.real(np.vdot(fI, dI) + np.vdot(fII, dII)))
    h_h = 4.0 * float(np.real(np.vdot(fI, fI) + np.vdot(fII, fII)))
    t_ip = time.perf_counter() - t0
    assert np.isfinite(d_h + h_h)
    return rate, t_ip


def cpu_likelihood_reference(procs: int = 0, sample_len: int = 200000) -> dict:
    """likelihoods/s of the reference's CPU path on the host cores: per
    template its own AAKwave (timed on a sample_len-sample truncation of the
    fiducial source, scaled to LIKE_LENGTH samples) plus a full-length numpy
    rFFT inner product, one template at a time per process."""
    import multiprocessing as mp

    from oracle import oracle as O

    if not O.ref_available():
        return {"value": None, "unit": "likelihoods/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libaakref.so is not built"}
    procs = procs or (os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_ref_like_worker, [(sample_len, LIKE_LENGTH)] * procs)
    per_template = [LIKE_LENGTH / r + t for r, t in res]
    value = sum(1.0 / x for x in per_template)
    return {"value": value, "unit": "likelihoods/s", "cores": procs, "kind": "reference",
            "seconds_per_likelihood": float(np.mean(per_template)),
            "waveform_samples_per_s_per_core": float(np.mean([r for r, _ in res])),
            "fft_inner_product_s": float(np.mean([t for _, t in res])),
            "sample": f"reference AAKwave on the fiducial config-4 source truncated to {sample_len} samples (scaled to "
                      f"{LIKE_LENGTH}), plus a {LIKE_LENGTH}-sample numpy rFFT inner product of both channels; "
                      f"{procs} processes, one template each"}


# ----------------------------------------------------------------------------- likelihood (config 4)
FIDUCIAL = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.8, 2.0, 1.0])  # gpu_gen_AAK order
# DRAM bytes (read + write) per sample of the split waveform kernel, from an ncu
# capture of that kernel on all 512 sources of the configuration-1 draw cut to
# an eighth of their length (bench.py --profile waveform512)
TRAFFIC_BYTES_PER_SAMPLE = (923.200768e6 + 1849.097e6) / 108_999_922
LIKE_LENGTH = 3_200_000  # 1 yr at dt = 10 s rounded up to the 5-smooth FFT length 2^10 * 5^5


def config4_templates(n: int, seed: int = SEED + 4):
    """Fiducial (configuration 0 source, T ~ 1 yr) perturbed by 1e-5 relative in M, mu, p0 and 1e-3 rad in angles."""
    rng = np.random.default_rng(seed)
    X = np.tile(FIDUCIAL, (n, 1))
    for j in (2, 4, 5):
        X[:, j] *= 1.0 + 1e-5 * rng.standard_normal(n)
    for j in (0, 6, 7, 8, 9, 10, 11, 12):
        X[:, j] += 1e-3 * rng.standard_normal(n)
    return X


def run_parmap_warm_start(n_train: int, local_rank: int):
    """Configuration 3: train the warm-start network on n_train seeded points
    (labels from the plain map solve), evaluate it on 2^16 held-out points and
    time its tensor-core inference kernel.  Returns (report, model)."""
    import torch

    from emri_kludge_suite_b200 import parmap_mlp as PM

    t0 = time.perf_counter()
    train = PM.make_dataset(n_train, SEED + 3)
    held = PM.make_dataset(1 << 16, SEED + 33)
    t_data = time.perf_counter() - t0
    m = PM.ParMapMLP(local_rank, seed=SEED)
    v = train["valid"]
    hist = m.train(train["x"][v], train["y"][v], epochs=60, batch=8192, lr=1e-2, seed=SEED)
    ev = PM.evaluate(m, held)
    # inference kernel throughput: n_train points resident on the device
    xd = torch.tensor(train["x"].astype(np.float32), device="cuda")
    yd = torch.empty((n_train, 3), dtype=torch.float32, device="cuda")
    for _ in range(3):
        m.forward_device(xd.data_ptr(), yd.data_ptr(), n_train)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 20
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        m.forward_device(xd.data_ptr(), yd.data_ptr(), n_train)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    tc_flops = 2.0 * 2 * 128 * 128  # the two 128 x 128 tensor-core layers, per point
    all_flops = 2.0 * (4 * 128 + 2 * 128 * 128 + 3 * 128)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "MEASURED_PEAKS.json")))
    except Exception:
        pass
    bf16_peak = peaks.get("bf16_tflops") or 1590.0
    tflops = tc_flops * n_train / (ms * 1e-3) / 1e12
    rep = {
        "workload": "config3: MLP 4->128->128->128->3 SiLU, BF16 weights/activations, FP32 accumulate; "
                    f"{n_train} training points p~U(p_sep+0.1,20), e~U(0,0.7), iota~U(0,pi), a~U(0,0.95); "
                    "2^16 held out; labels = plain map solve",
        "train_points": int(v.sum()), "label_failures": int((~v).sum()), "heldout_points": ev["points"],
        "dataset_seconds": t_data, "epochs": hist["epochs"], "batch": hist["batch"], "train_steps": hist["steps"],
        "train_seconds": hist["seconds"], "train_rows_per_s": hist["epochs"] * int(v.sum()) / hist["seconds"],
        "loss_first_epoch": hist["loss"][0], "loss_final": hist["loss"][-1],
        "newton": {k: ev[k] for k in ("iters_cold", "iters_warm", "iterations_saved_frac", "iters_to_tol_cold",
                                       "iters_to_tol_warm", "iterations_to_tol_saved_frac", "fallback_rate",
                                       "failed_cold", "failed_warm")},
        "residual": {"rel_cold_max": ev["residual_rel_cold_max"], "rel_warm_max": ev["residual_rel_warm_max"],
                     "abs_warm_max": ev["residual_abs_warm_max"], "guess_rel": ev["guess_residual_rel"]},
        "prediction_abs_err_max": ev["prediction_abs_err"],
        "warm_vs_cold_solution_max_rel": ev["warm_vs_cold_solution_max_rel"],
        "solve_seconds": {"cold": ev["solve_seconds_cold"], "warm": ev["solve_seconds_warm"],
                          "predict": ev["predict_seconds"]},
        "inference": {"points_per_s": n_train / (ms * 1e-3), "ms_per_launch": ms, "points": n_train,
                      "flops_per_point": all_flops, "tensor_tflops": tflops, "bf16_peak_tflops": bf16_peak,
                      "frac_of_measured_bf16": tflops / bf16_peak},
    }
    return rep, m


def run_fisher(g, n_points: int) -> dict:
    """Fisher matrices (14 x 14, 28 templates each) at config-4 points: host
    planning + waveforms + FFT + device Gram, all points in one pipelined call
    (the next point planned while the device works on the current one), and one
    call per point beside it."""
    P = config4_templates(n_points, seed=SEED + 41)
    step = 1e-6 * np.maximum(np.abs(FIDUCIAL), 1.0)
    rows = []
    for x in P:
        X = np.tile(x, (28, 1))
        for i in range(14):
            X[2 * i, i] += step[i]
            X[2 * i + 1, i] -= step[i]
        rows.append(X)
    g.fisher_gram(rows[0], 1.0)  # warm-up (rows, FFT plan, scratch)
    t0 = time.perf_counter()
    for X in rows:
        _, st = g.fisher_gram(X, 1.0, return_status=True)
        if np.any(st != 0):
            raise RuntimeError("a Fisher template failed")
    wall_single = time.perf_counter() - t0
    rows = np.stack(rows)
    g.fisher_gram_batch(rows[:2], 1.0)  # warm-up of the second planning context
    t0 = time.perf_counter()
    _, st = g.fisher_gram_batch(rows, 1.0, return_status=True)
    wall = time.perf_counter() - t0
    if np.any(st != 0):
        raise RuntimeError("a Fisher template failed")
    m = g.last_timing_ms()
    ms = np.array([m["host_plan"], m["waveform"], m["fft"], m["reduce"]]) / n_points
    nbins = LIKE_LENGTH // 2 + 1
    gram_bytes = 2 * 28 * nbins * 16.0  # each template spectrum read once, both channels
    gbs = gram_bytes / (ms[3] * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs") or 6650.0
    return {"workload": "config4 points, 14 parameters, central differences (28 templates of 3.2e6 samples per "
                        "matrix), reference harmonic rule, FP64",
            "points": n_points, "fisher_per_s": n_points / wall, "fisher_per_s_gpu": 1e3 / float(ms[1:].sum()),
            "fisher_per_s_one_call_per_point": n_points / wall_single,
            "ms_per_matrix": dict(zip(("host_plan", "waveform", "fft", "gram"), ms.tolist())),
            "gram_roofline": {"kernel": "k_fisher_partial + k_fisher_final", "bound": "hbm", "achieved": gbs,
                              "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                              "bytes": gram_bytes, "peak_source": "measured copy bandwidth (MEASURED_PEAKS.json)"
                              if peaks.get("hbm_gbs") else "fallback"},
            "gpu_launches_per_matrix": 6,  # spline solve, tile pre-pass (2), k_waveform, Fisher Gram (2) (+ cuFFT)
            "cpu_baseline": ref_fisher_seconds()}


def ref_fisher_seconds(sample_len: int = 200000) -> dict:
    """The reference's CPU cost of one such Fisher matrix: its own AAKwave on the
    fiducial config-4 source truncated to sample_len samples (one process),
    scaled to 28 templates of 3.2e6 samples.  The reference's get_Fisher adds an
    FFT and host dot products per template on top."""
    from oracle import oracle as O

    if not O.ref_available():
        return {"value": None, "sample": "unavailable: oracle/_ref/libaakref.so is not built"}
    iota, s_, p, e, M, mu, gamma, psi, alph, thS, phS, thK, phK, D = FIDUCIAL
    pars = dict(backint=False, LISA=True, length=sample_len, dt=DT, p=p, T=sample_len * DT / YEAR, f=0.0, T_fit=1.0,
                mu=mu, M=M, s=s_, e=e, iota=iota, gamma=gamma, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK,
                phi_K=phK, alpha=alph, D=D)
    t0 = time.perf_counter()
    O.ref_aakwave(pars)
    rate = sample_len / (time.perf_counter() - t0)
    return {"value": 28 * LIKE_LENGTH / rate, "unit": "s per Fisher matrix (waveforms only)", "cores": 1,
            "kind": "reference", "sample": f"reference AAKwave, fiducial config-4 source, {sample_len} samples, "
                                          f"{rate:.3g} samples/s, scaled to 28 x {LIKE_LENGTH} samples"}


def template_pars(x) -> dict:
    """gpu_gen_AAK-order parameters -> an AAKwrapper pars dict over the configuration-4 span."""
    iota, s_, p, e, M, mu, gamma, psi, alph, thS, phS, thK, phK, D = x
    return dict(backint=False, LISA=True, length=LIKE_LENGTH, dt=DT, p=p, T=LIKE_LENGTH * DT / YEAR, f=0.0, T_fit=1.0,
                mu=mu, M=M, s=s_, e=e, iota=iota, gamma=gamma, psi=psi, theta_S=thS, phi_S=phS, theta_K=thK, phi_K=phK,
                alpha=alph, D=D)


def run_evolve_compare(sources, local_rank: int, nthreads: int, n_templates: int = 4096) -> dict:
    """Batch planning with the coarse AK recurrences on the host threads (AVX2
    lane groups, the default) against one GPU thread per source
    (aak_ctx_set_evolve_device), on the configuration-1 sources and on
    configuration-4 likelihood templates: wall time of one plan each way."""
    import emri_kludge_suite_b200 as E

    out = {}
    for name, plist, nm in (("config1_512_sources", sources, NMODES),
                            (f"config4_{n_templates}_templates", [template_pars(x) for x in config4_templates(n_templates)],
                             None)):
        res = {}
        for mode in ("host", "device"):
            wb = E.WaveBatch(local_rank)
            wb.set_evolve_device(mode == "device")
            wb.plan(plist, nmodes=nm, nthreads=nthreads)  # warm-up: page-locks the knot arrays at full size
            t0 = time.perf_counter()
            wb.plan(plist, nmodes=nm, nthreads=nthreads)
            res[mode] = {"plan_s": time.perf_counter() - t0, "failed": int(np.sum(wb.status != 0))}
            if mode == "device":
                res[mode]["passes_ms"] = wb.plan_ms()
            wb.close()
        res["device_over_host"] = res["device"]["plan_s"] / res["host"]["plan_s"]
        out[name] = res
    out["host_threads"] = nthreads
    return out


def run_likelihood(n_templates: int, local_rank: int, model=None, n_fisher: int = 0, with_cpu: bool = False,
                   rank: int = 0, world: int = 1) -> dict:
    """likelihoods/s of the batched path: host planning + waveforms + FFT + reduction, end to end per call."""
    from emri_kludge_suite_b200.gpuAAK import GPUAAK
    from emri_kludge_suite_b200.LISAnoise import LISA_Noise, generate_noise_frequencies, generate_noise_single_channel

    g = GPUAAK(1.0, 100, LIKE_LENGTH, 100.0, DT, True, False)
    freqs = generate_noise_frequencies(LIKE_LENGTH * DT, 1 / DT)
    freqs[0] = freqs[1] / 10.0
    w = 1.0 / np.sqrt(LISA_Noise(freqs, dur=1)) * np.sqrt(DT / LIKE_LENGTH)
    # data: fiducial waveform + seeded LISA-coloured noise, pre-weighted
    ones = np.ones_like(w)
    zero = np.zeros(len(w), dtype=np.complex128)
    g.input_data(zero, zero, ones, ones)
    g.gpu_gen_AAK(*FIDUCIAL)
    g.Likelihood()
    _, sI, sII = g.GetWaveform(is_Fourier=True)
    nb = len(w)
    hI_f = sI[0:2 * nb:2] + 1j * sI[1:2 * nb:2]
    hII_f = sII[0:2 * nb:2] + 1j * sII[1:2 * nb:2]
    rng = np.random.default_rng(SEED + 40)
    df = 1.0 / (LIKE_LENGTH * DT)
    n1 = generate_noise_single_channel(LISA_Noise, [], {"dur": 1}, df, freqs, rng)
    n2 = generate_noise_single_channel(LISA_Noise, [], {"dur": 1}, df, freqs, rng)
    dI, dII = w * (hI_f + n1), w * (hII_f + n2)
    g.input_data(dI, dII, w, w)
    # one caller batch of n_templates x world templates, split over the ranks
    # (equal costs: LPT balances the counts); per-template (4<h|d>, 4<h|h>)
    # rows are gathered back with one all-gather
    X_all = config4_templates(n_templates * world)
    mine = np.arange(len(X_all))
    if world > 1:
        from emri_kludge_suite_b200.shard import rank_indices

        mine = rank_indices(np.ones(len(X_all)), rank, world)
    X = X_all[mine]
    n_templates = len(X)
    d_d = 4.0 * float(np.sum(np.abs(dI) ** 2) + np.sum(np.abs(dII) ** 2))  # pygpuAAK.py:67

    def timed():
        g.likelihood_batch(X[: min(256, n_templates)])  # warm-up at the batch size (rows, FFT plan, tables)
        t0 = time.perf_counter()
        o, st = g.likelihood_batch(X, return_status=True)
        wall = time.perf_counter() - t0
        ms = g.last_timing_ms()
        gpu_s = (ms["waveform"] + ms["fft"] + ms["reduce"]) * 1e-3
        return o, st, {"likelihoods_per_s": n_templates / wall, "likelihoods_per_s_gpu": n_templates / gpu_s,
                       "failed": int(np.sum(st != 0)), "ms": ms}

    out64, st64, plain = timed()
    if world > 1:
        from emri_kludge_suite_b200.shard import gather_rows

        t0 = time.perf_counter()
        gathered = gather_rows(out64, mine, len(X_all))
        plain["gather"] = {"templates": len(X_all), "seconds": time.perf_counter() - t0,
                           "finite": bool(np.all(np.isfinite(gathered)))}
    res = {"workload": "config4: fiducial config-0 source, 3.2e6 samples (1.014 yr, dt=10 s), LISA-coloured noise, "
                       "templates perturbed 1e-5 rel (M, mu, p0) / 1e-3 rad (angles), reference harmonic rule",
           "templates": n_templates, "samples_per_template": LIKE_LENGTH, "fp64_plain": plain}
    if n_fisher > 0:
        res["fisher"] = run_fisher(g, n_fisher)
    res.update({k: plain[k] for k in ("likelihoods_per_s", "likelihoods_per_s_gpu", "failed", "ms")})
    # split precision + learned warm start vs the plain FP64 path
    g.set_precision(1)
    g.set_warm_start(model)
    outs, sts, fast = timed()
    g.set_precision(0)
    g.set_warm_start(None)
    ok = (st64 == 0) & (sts == 0)
    logl64 = -0.5 * (d_d + out64[:, 1] - 2.0 * out64[:, 0])
    logls = -0.5 * (d_d + outs[:, 1] - 2.0 * outs[:, 0])
    fast["max_abs_dlogL_vs_fp64"] = float(np.max(np.abs(logls - logl64)[ok])) if ok.any() else None
    fast["max_abs_logL"] = float(np.max(np.abs(logl64[ok]))) if ok.any() else None
    fast["warm_start"] = model is not None
    res["split_warm"] = fast
    # split templates with the FP32 transform and compensated FP32 inner products
    g.set_precision(2)
    g.set_warm_start(model)
    out32, st32, f32 = timed()
    g.set_precision(0)
    g.set_warm_start(None)
    ok32 = (st64 == 0) & (st32 == 0)
    logl32 = -0.5 * (d_d + out32[:, 1] - 2.0 * out32[:, 0])
    f32["max_abs_dlogL_vs_fp64"] = float(np.max(np.abs(logl32 - logl64)[ok32])) if ok32.any() else None
    f32["median_abs_dlogL_vs_fp64"] = float(np.median(np.abs(logl32 - logl64)[ok32])) if ok32.any() else None
    res["split_fp32_fft"] = f32
    # the same without the warm start: the start's tensor-core inference waits
    # for the persistent waveform kernel of the previous batch, which holds
    # every SM, so the warm start lengthens the pipelined host planning
    g.set_precision(2)
    o32n, s32n, f32n = timed()
    g.set_precision(0)
    okn = (st64 == 0) & (s32n == 0)
    f32n["max_abs_dlogL_vs_fp64"] = float(np.max(np.abs(-0.5 * (d_d + o32n[:, 1] - 2.0 * o32n[:, 0]) - logl64)[okn])) \
        if okn.any() else None
    res["split_fp32_fft_no_warm_start"] = f32n
    # HBM roofline of the inner-product kernel.  Each template's spectra of
    # both channels stream from HBM once; the data and weights (77 MB in FP64,
    # 38 MB in FP32) stay in the 126 MB L2 across the templates of a batch, so
    # the HBM-bound bytes per template are the spectra.  The byte count of the
    # formula with the data and weights is reported beside it.
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs") or 6650.0
    nb = LIKE_LENGTH // 2 + 1
    for key, run_, stream_bin, formula_bin, kern in (("fp64_plain", plain, 2 * 16, 2 * (16 + 16) + 8, "k_inner_partial"),
                                                     ("split_fp32_fft", f32, 2 * 8, 2 * (8 + 8) + 4, "k_inner_partial_f32")):
        ms_red = run_["ms"]["reduce"]
        gbs = stream_bin * nb * n_templates / (ms_red * 1e-3) / 1e9 if ms_red > 0 else None
        res[key]["reduce_roofline"] = {
            "kernel": kern + " + k_inner_final", "bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
            "frac": gbs / hbm if gbs else None, "bytes_per_template": stream_bin * nb,
            "bytes_rule": "template spectra of both channels (HBM); data and weights are L2-resident",
            "formula_bytes_per_template": formula_bin * nb,
            "formula_gbs": formula_bin * nb * n_templates / (ms_red * 1e-3) / 1e9 if ms_red > 0 else None,
            "peak_source": "measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peaks.get("hbm_gbs") else "fallback"}
    if with_cpu:
        res["cpu_baseline"] = cpu_likelihood_reference()
    return res


# ----------------------------------------------------------------------------- GPU arm
def ref_phase_rate(sources, n_src: int = 16, sample_len: int = 200000) -> dict:
    """The reference's own AAKphase (front end + GenPhase), one process, on a
    bounded sample of the configuration-1 sources."""
    from oracle import oracle as O

    if not O.ref_available():
        return {"value": None, "unit": "samples/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libaakref.so is not built"}
    tot, t0 = 0, time.perf_counter()
    for p in sources[:n_src]:
        q = dict(p)
        q["length"] = min(int(p["length"]), sample_len)
        q["T"] = q["length"] * q["dt"] / YEAR
        O.ref_aakphase(q)
        tot += q["length"]
    dt = time.perf_counter() - t0
    return {"value": tot / dt, "unit": "samples/s", "cores": 1, "kind": "reference",
            "sample": f"{n_src} config-1 sources truncated to {sample_len} samples, reference AAKphase "
                      "(front end + GenPhase), one process"}


def run_tdi(sources, local_rank: int, nthreads: int, n_ref: int = 4) -> dict:
    """Frequency-domain AAK TDI (AAKwrapper.tdi) of 16 configuration-1 sources in
    one batch, end to end through aak_tdi_batch_host (host front end and grid
    planning, the phase-grid and stationary-phase kernels, copies back); the
    reference's own AAKTDI timed on the first n_ref of them, one process."""
    import emri_kludge_suite_b200 as E
    from oracle import oracle as O

    sub = sources[:: max(1, len(sources) // 16)][:16]
    wb = E.WaveBatch(local_rank)
    wb.tdi_host(sub[:2], nthreads=nthreads)  # warm-up (context, buffers)
    times = []
    for _ in range(2):
        t0 = time.perf_counter()
        rows, offs, st = wb.tdi_host(sub, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
    wall = float(np.mean(times))
    bins = int(offs[-1])
    wb.close()
    res = {"workload": "frequency-domain AAK TDI (X, Y, Z on f = i / T) of 16 configuration-1 sources (every 32nd), "
                       "reference harmonic rule, FP64",
           "sources": len(sub), "failed": int(np.sum(st != 0)), "bins": bins, "seconds_per_batch": wall,
           "sources_per_s": len(sub) / wall, "bins_per_s": bins / wall, "gpu_launches_per_batch": 4,
           "e2e": {"value": len(sub) / wall, "unit": "TDI waveforms/s", "h2d_bytes_per_step": None,
                   "d2h_bytes_per_step": 48 * bins}}
    if O.ref_available():
        # the reference keeps 30 complex transfer-function rows per harmonic on its phase grid
        # (0.01 M^2 / mu spacing): time it on sources whose grid stays below 2e5 points
        def grid_points(p):
            return (int(p["length"]) - 1) * p["dt"] / (0.01 * p["M"] ** 2 / p["mu"] * MSUN_SEC)

        ref_src = [p for p in sub if grid_points(p) < 2e5][:n_ref]
        t0 = time.perf_counter()
        nb = 0
        for p in ref_src:
            O.ref_aaktdi(p)
            nb += (int(p["length"]) + 1) // 2
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": len(ref_src) / dt, "unit": "TDI waveforms/s", "cores": 1,
                               "kind": "reference", "bins_per_s": nb / dt,
                               "sample": f"reference AAKTDI (front end + GenTDI) on {len(ref_src)} of the same sources "
                                         "(phase grids below 2e5 points), one process"}
    return res


def run_phases(args, wb, sources, sptr, stream, N, N_all, reduce_max, local_rank, nthreads):
    """AAK phase product (GenPhase: t, 3 phases, 3 rates, e per sample, FP64) of
    the uploaded configuration-1 batch: device-resident kernel time, roofline,
    and end to end through aak_phase_batch_host on a subset."""
    import ctypes

    import torch

    import emri_kludge_suite_b200 as E
    from emri_kludge_suite_b200 import _lib

    L = _lib.lib()
    out = torch.empty(8 * N, dtype=torch.float64, device="cuda")  # 64 B/sample (> L2)
    for _ in range(args.warmup):
        wb.run_phase(out.data_ptr(), N, stream=sptr)
    torch.cuda.synchronize()
    assert wb.device_status() == 0
    ms3 = (ctypes.c_float * 3)()
    L.aak_batch_set_profiling(wb._ctx, 1)
    kern = np.zeros(3)
    for _ in range(2):
        wb.run_phase(out.data_ptr(), N, stream=sptr)
        _lib.check(L.aak_batch_kernel_ms(wb._ctx, ms3), "kernel timing")
        kern += np.array(ms3[:])
    kern /= 2
    L.aak_batch_set_profiling(wb._ctx, 0)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        wb.run_phase(out.data_ptr(), N, stream=sptr)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = reduce_max(ev0.elapsed_time(ev1)) / args.steps
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs")
    hbm_src = "measured copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if hbm else "fallback 6650 GB/s"
    hbm = hbm or 6650.0
    bytes_per_sample = 64.0  # the eight output rows; knot windows add < 1 B/sample
    gbs = bytes_per_sample * N / (kern[2] * 1e-3) / 1e9
    del out
    torch.cuda.empty_cache()
    # end to end on the sources of the plain-path subset, pinned host rows
    sub = sources[:: max(1, len(sources) // 16)][:16]
    wp = E.WaveBatch(local_rank)
    Np = int(sum(int(p["length"]) for p in sub))
    host = torch.empty(8 * Np, dtype=torch.float64, pin_memory=True)
    P = _lib.params_array(sub)
    offs = np.zeros(len(sub) + 1, dtype=np.int64)
    st = np.zeros(len(sub), dtype=np.int32)
    times = []
    for k in range(3):  # the first call warms the context's buffers
        t0 = time.perf_counter()
        _lib.check(L.aak_phase_batch_host(wp._ctx, P, len(sub), nthreads,
                                          ctypes.cast(host.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                          _lib.ptr(offs), _lib.ptr(st)), "aak_phase_batch_host")
        if k > 0:
            times.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(times))
    h2d = int(wp.plan_bytes())
    wp.close()
    return {
        "workload": "AAK phase product (GenPhase rows t, phase_r/theta/phi, omega_r/theta/phi, e; FP64) "
                    "of the configuration-1 batch",
        "value": N_all / (ms * 1e-3), "unit": "samples/s", "ms_per_step": ms,
        "kernel_ms": {"clears": kern[0], "phase_and_freeze": kern[2]},
        "roofline": {"kernel": "k_tile_params + k_waveform<fp64, phase> + k_phase_freeze", "bound": "hbm", "achieved": gbs,
                     "peak": hbm, "unit": "GB/s", "frac": gbs / hbm, "peak_source": hbm_src,
                     "bytes_per_sample": bytes_per_sample},
        "e2e": {"value": Np / e2e_s, "unit": "samples/s", "seconds_per_step": e2e_s, "sources": len(sub),
                "samples": Np, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 64 * Np, "host_threads": nthreads},
        "gpu_launches_per_step": 3,  # k_tile_params, k_waveform<fp64, phase>, k_phase_freeze
    }


def _mem_available_gb():
    """MemAvailable of the host (Linux), in GB; None elsewhere."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return round(int(line.split()[1]) / 1e6, 1)
    except OSError:
        pass
    return None


def run_gpu(args, rank, world, local_rank):
    import torch

    import emri_kludge_suite_b200 as E
    from emri_kludge_suite_b200 import _lib

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

    # one caller batch of nsrc x world sources, split over the ranks by LPT on
    # samples x harmonics (world = 1: the seeded 512-source draw itself)
    from emri_kludge_suite_b200.shard import rank_indices, source_costs

    all_sources, rng = config1(SEED, args.nsrc * world)
    mine = rank_indices(source_costs(all_sources, NMODES), rank, world) if world > 1 else np.arange(len(all_sources))
    sources = [all_sources[i] for i in mine]
    if world > 1:
        rng = np.random.default_rng([SEED, rank])  # redraws (rare) stay on their rank
    wb = E.WaveBatch(local_rank)
    # the host cores are shared by the ranks of one node
    nthreads = max(1, (os.cpu_count() or 1) // world)
    t_plan0 = time.perf_counter()
    for _ in range(8):  # redraw sources that fail or plunge inside T
        wb.plan(sources, nmodes=NMODES, nthreads=nthreads)
        bad = [i for i in range(len(sources))
               if wb.status[i] != 0 or wb.i_plunge[i] != int(sources[i]["length"]) - 1]
        if not bad:
            break
        for i in bad:
            sources[i] = draw_source(rng)
    t_plan = time.perf_counter() - t_plan0
    N = wb.total_samples
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    wb.upload(sptr)
    hI = torch.empty(N, dtype=torch.float64, device="cuda")
    hII = torch.empty(N, dtype=torch.float64, device="cuda")
    L = _lib.lib()
    import ctypes

    tfl = ctypes.c_double(0.0)
    _lib.check(L.aak_probe_fp64_tflops(local_rank, ctypes.byref(tfl)), "fp64 probe")
    fp64_peak = tfl.value
    _lib.check(L.aak_probe_fp32_tflops(local_rank, ctypes.byref(tfl)), "fp32 probe")
    fp32_peak = tfl.value
    ms3 = (ctypes.c_float * 3)()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)

    def reduce_max(x):
        if not dist:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if dist:
        tot = torch.tensor([float(N)], device="cuda", dtype=torch.float64)
        dist.all_reduce(tot)
        N_all = float(tot.item())
    else:
        N_all = float(N)

    # ---- autotuner: every launch shape of the waveform stage timed on this
    #      batch, the fastest kept per precision (no cache file: all timed)
    tune = {}
    for prec, name in ((0, "fp64"), (1, "split")):
        v, ms_v = wb.autotune(hI.data_ptr(), hII.data_ptr(), precision=prec)
        tune[name] = {"choice": v, "ms_per_variant": ms_v}
    tune["variants"] = ["pre-pass, joint 1, 3 CTAs/SM", "tables inside the tiles, 2 CTAs/SM",
                        "pre-pass, joint 1 (split) / 2 (FP64), 2 CTAs/SM", "pre-pass, joint 4, 2 CTAs/SM",
                        "pre-pass, joint 2 / 1, 3 CTAs/SM (split) / 2 CTAs/SM (FP64)",
                        "pre-pass, joint 2, 2 CTAs/SM (split) / 3 CTAs/SM (FP64)"]

    # ---- plain FP64 batched path (precision 0): per-kernel times
    for _ in range(args.warmup):
        wb.run(hI.data_ptr(), hII.data_ptr(), stream=sptr)
    torch.cuda.synchronize()
    L.aak_batch_set_profiling(wb._ctx, 1)
    kern = np.zeros(3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        wb.run(hI.data_ptr(), hII.data_ptr(), stream=sptr)
        _lib.check(L.aak_batch_kernel_ms(wb._ctx, ms3), "kernel timing")
        kern += np.array(ms3[:])
    ev1.record(stream)
    torch.cuda.synchronize()
    L.aak_batch_set_profiling(wb._ctx, 0)
    ms64 = reduce_max(ev0.elapsed_time(ev1))
    kern /= args.steps
    value64 = N_all * args.steps / (ms64 * 1e-3)

    # ---- split precision (the headline path): per-kernel times first
    hI2 = torch.empty_like(hI)
    hII2 = torch.empty_like(hII)
    for _ in range(args.warmup):
        wb.run(hI2.data_ptr(), hII2.data_ptr(), precision=1, stream=sptr)
    L.aak_batch_set_profiling(wb._ctx, 1)
    kern_s = np.zeros(3)
    for _ in range(2):
        wb.run(hI2.data_ptr(), hII2.data_ptr(), precision=1, stream=sptr)
        _lib.check(L.aak_batch_kernel_ms(wb._ctx, ms3), "kernel timing")
        kern_s += np.array(ms3[:])
    kern_s /= 2
    L.aak_batch_set_profiling(wb._ctx, 0)
    # then the timed steps: one graph replay (two clears and the waveform kernel) per step
    for _ in range(args.warmup):
        wb.run_graph(hI2.data_ptr(), hII2.data_ptr(), precision=1, stream=sptr)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        wb.run_graph(hI2.data_ptr(), hII2.data_ptr(), precision=1, stream=sptr)
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = reduce_max(ev0.elapsed_time(ev1))
    # k_spline_coeffs, the tile pre-pass (two kernels, when the tuned shape uses
    # it) and k_waveform<split> per replay; the clears are memset nodes
    launches = wb.launches() * args.steps
    value = N_all * args.steps / (ms * 1e-3)
    # accuracy of every source against the FP64 outputs of the same batch
    worst_mm, worst_rel, mms = 0.0, 0.0, []
    o = wb.offsets
    for s in range(len(sources)):
        a1, a2 = hI[o[s]:o[s + 1]], hII[o[s]:o[s + 1]]
        b1, b2 = hI2[o[s]:o[s + 1]], hII2[o[s]:o[s + 1]]
        aa = float(a1.dot(a1) + a2.dot(a2))
        bb = float(b1.dot(b1) + b2.dot(b2))
        ab = float(a1.dot(b1) + a2.dot(b2))
        mm = 1.0 - ab / math.sqrt(aa * bb) if aa > 0 and bb > 0 else 0.0
        rel = float(torch.maximum((a1 - b1).abs().max(), (a2 - b2).abs().max()) /
                    torch.maximum(a1.abs().max(), a2.abs().max()))
        mms.append(mm)
        worst_mm, worst_rel = max(worst_mm, mm), max(worst_rel, rel)
    accuracy = {"max_mismatch": worst_mm, "median_mismatch": float(np.median(mms)), "max_rel_dh": worst_rel,
                "sources": len(sources), "bar": 1e-6}
    fps = flops_per_sample(NMODES)
    ach64 = fps * N / ((kern[1] + kern[2]) * 1e-3) / 1e12
    fp64 = {"value": value64, "unit": "samples/s", "ms_per_step": ms64 / args.steps,
            "kernel_ms": {"clears": kern[0], "tile_prepass": kern[1], "waveform_fp64": kern[2]},
            "roofline": {"kernel": "k_tile_params + k_tile_table + k_waveform<fp64>", "bound": "fp64",
                         "achieved": ach64, "peak": fp64_peak,
                         "unit": "TFLOP/s", "frac": ach64 / fp64_peak if fp64_peak > 0 else None,
                         "peak_source": "measured FP64 FMA rate on this GPU (aak_probe_fp64_tflops)"},
            "split_speedup": ms64 / ms}
    del hI2, hII2
    split = {"value": value, "kernel_ms": {"clears": kern_s[0], "tile_prepass": kern_s[1], "waveform_split": kern_s[2]}}

    # ---- frequency-domain TDI of a subset of the batch
    tdi = run_tdi(sources, local_rank, nthreads) if args.tdi and rank == 0 else None

    # ---- AAK phase product of the same batch
    phases = None
    if args.phases:
        phases = run_phases(args, wb, sources, sptr, stream, N, N_all, reduce_max, local_rank, nthreads)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            phases["cpu_baseline"] = ref_phase_rate(sources)

    # ---- plain FP64 per-source path on a subset of the same sources (the baseline)
    plain = None
    if args.plain_sources > 0:
        sub = sources[:: max(1, len(sources) // args.plain_sources)][: args.plain_sources]
        wp = E.WaveBatch(local_rank)
        wp.plan(sub, nmodes=NMODES, nthreads=nthreads)
        wp.upload(sptr)
        Np = wp.total_samples
        pI = torch.empty(Np, dtype=torch.float64, device="cuda")
        pII = torch.empty_like(pI)
        traj = torch.empty(9 * Np, dtype=torch.float64, device="cuda")
        wp.run_plain(pI.data_ptr(), pII.data_ptr(), traj.data_ptr(), Np, stream=sptr)  # warm-up
        torch.cuda.synchronize()
        ev0.record(stream)
        wp.run_plain(pI.data_ptr(), pII.data_ptr(), traj.data_ptr(), Np, stream=sptr)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms_plain = ev0.elapsed_time(ev1)
        sps = Np / (ms_plain * 1e-3)
        plain = {"samples_per_s": sps, "sources": len(sub), "samples": int(Np), "ms": ms_plain,
                 "launches": wp.launches(),
                 "method": "per source: phase kernels on a one-source view writing the dense FP64 trajectory "
                           "(72 B/sample), then one thread per sample with 5 jn() + cos/sin + rotation per harmonic",
                 "speedup_batched_fp64": value64 / sps,
                 "speedup_batched_split": value / sps}
        del pI, pII, traj
        wp.close()
        torch.cuda.empty_cache()  # the plain path's 77 GB of buffers go back before configuration 2

    # ---- configuration 2: split precision vs FP64 per source at high eccentricity,
    #      mismatch flat and weighted by the LISA noise PSD
    cfg2 = None
    if args.config2_sources > 0:
        from emri_kludge_suite_b200.LISAnoise import LISA_Noise

        src2, nm2 = config2(SEED + 2 + rank, args.config2_sources)
        w2 = E.WaveBatch(local_rank)
        w2.plan(src2, nmodes=nm2, nthreads=nthreads)
        w2.upload(sptr)
        N2 = w2.total_samples
        a64 = torch.empty(2 * N2, dtype=torch.float64, device="cuda")
        a32 = torch.empty_like(a64)
        w2.run(a64.data_ptr(), a64.data_ptr() + 8 * N2, precision=0, stream=sptr)
        w2.run(a32.data_ptr(), a32.data_ptr() + 8 * N2, precision=1, stream=sptr)
        torch.cuda.synchronize()
        ev0.record(stream)
        w2.run(a32.data_ptr(), a32.data_ptr() + 8 * N2, precision=1, stream=sptr)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms2 = ev0.elapsed_time(ev1)
        # the PSD (dur = 1 yr) on a log grid of 2e5 points, interpolated in log f on the device
        lf0, lf1, ng = math.log(1e-9), math.log(0.06), 200_000
        logS = torch.tensor(np.log(LISA_Noise(np.exp(np.linspace(lf0, lf1, ng)), dur=1)), device="cuda")

        def inv_psd(n, dt):
            f = torch.fft.rfftfreq(n, dt, dtype=torch.float64, device="cuda")[1:]
            x = (torch.log(f) - lf0) / (lf1 - lf0) * (ng - 1)
            k = x.floor().clamp(0, ng - 2).long()
            fr = x - k
            return torch.exp(-(logS[k] * (1 - fr) + logS[k + 1] * fr))

        o2 = w2.offsets
        mm2, rel2, psd2 = [], [], []
        for s_ in range(len(src2)):
            if w2.status[s_] != 0:
                continue
            x1, x2 = a64[o2[s_]:o2[s_ + 1]], a64[N2 + o2[s_]:N2 + o2[s_ + 1]]
            y1, y2 = a32[o2[s_]:o2[s_ + 1]], a32[N2 + o2[s_]:N2 + o2[s_ + 1]]
            aa, bb, ab = float(x1.dot(x1) + x2.dot(x2)), float(y1.dot(y1) + y2.dot(y2)), float(x1.dot(y1) + x2.dot(y2))
            mm2.append(1.0 - ab / math.sqrt(aa * bb) if aa > 0 and bb > 0 else 0.0)
            rel2.append(float(torch.maximum((x1 - y1).abs().max(), (x2 - y2).abs().max()) /
                              torch.maximum(x1.abs().max(), x2.abs().max())))
            w = inv_psd(len(x1), DT)
            paa = pbb = pab = 0.0
            for u, v in ((x1, y1), (x2, y2)):
                U, V = torch.fft.rfft(u)[1:], torch.fft.rfft(v)[1:]
                pab += float((w * (U * V.conj()).real).sum())
                paa += float((w * U.abs() ** 2).sum())
                pbb += float((w * V.abs() ** 2).sum())
            psd2.append(1.0 - pab / math.sqrt(paa * pbb) if paa > 0 and pbb > 0 else 0.0)
        cfg2 = {"workload": "config2: e0~U(0.05,0.7), n_max=min(100,ceil(10/(1-e0)^1.5)), otherwise config1",
                "sources": len(src2), "ok_sources": int(np.sum(w2.status == 0)), "samples": int(N2),
                "nmodes_min_max": [int(min(nm2)), int(max(nm2))], "split_samples_per_s": N2 / (ms2 * 1e-3),
                "max_mismatch": float(max(mm2)), "median_mismatch": float(np.median(mm2)),
                "max_mismatch_psd": float(max(psd2)), "median_mismatch_psd": float(np.median(psd2)),
                "psd": "LISA_Noise(dur=1), f > 0, interpolated from a 2e5-point log grid",
                "max_rel_dh": float(max(rel2)), "median_rel_dh": float(np.median(rel2)), "bar": 1e-6,
                "reference": "the FP64 path of the same batch (each source is pinned to the FP64 oracle in the tests)"}
        del a64, a32, logS
        w2.close()
        torch.cuda.empty_cache()

    # ---- batch planning: host recurrences against the device evolution
    evolve_cmp = run_evolve_compare(sources, local_rank, nthreads) if args.evolve_compare and rank == 0 else None

    # ---- end to end through the C ABI with pinned host buffers
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    hIh = torch.empty(N, dtype=torch.float64, pin_memory=True)
    hIIh = torch.empty(N, dtype=torch.float64, pin_memory=True)
    P = _lib.params_array(sources)
    offs = np.zeros(len(sources) + 1, dtype=np.int64)
    st = np.zeros(len(sources), dtype=np.int32)
    nm = np.full(len(sources), NMODES, dtype=np.int32)
    h2d = 0
    e2e_times, e2e_faults = [], []
    wb.set_precision(1)  # the headline path, through the host-buffer entry point
    for k in range(e2e_steps + 1):  # first call warms the host buffers
        if dist:
            dist.barrier()
        f0 = resource.getrusage(resource.RUSAGE_SELF).ru_minflt
        t0 = time.perf_counter()
        _lib.check(L.aak_wave_batch_host(wb._ctx, P, len(sources), _lib.ptr(nm), nthreads,
                                         ctypes.cast(hIh.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                         ctypes.cast(hIIh.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                         _lib.ptr(offs), _lib.ptr(st)), "aak_wave_batch_host")
        dt_e2e = time.perf_counter() - t0
        if k > 0:
            e2e_times.append(dt_e2e)
            e2e_faults.append(resource.getrusage(resource.RUSAGE_SELF).ru_minflt - f0)
    e2e_s = float(np.mean(e2e_times))
    if dist:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    # plan bytes copied to the device per call (descriptors, knots, Bessel table)
    h2d = int(wb.plan_bytes())
    e2e = {"value": N_all / e2e_s, "unit": "samples/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": int(16 * N), "seconds_per_step": e2e_s, "host_threads": nthreads,
           "seconds_each": [round(x, 4) for x in e2e_times], "host_mem_available_gb": _mem_available_gb(),
           "minor_page_faults_each": e2e_faults}

    # ---- roofline of the dominant kernel (split harmonic sum: FP32 mode sums, FP64 phases)
    wave_ms = kern_s[1] + kern_s[2]  # the harmonic sums' Bessel tables are built in the pre-pass
    achieved = fps * N / (wave_ms * 1e-3) / 1e12
    roofline = {"kernel": "k_waveform<split> (with its tile pre-pass k_tile_params + k_tile_table)", "bound": "fp32",
                "achieved": achieved, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": achieved / fp32_peak if fp32_peak > 0 else None,
                "traffic": TRAFFIC_BYTES_PER_SAMPLE * N,
                "traffic_source": "dram read+write per sample of one ncu capture of the same kernel on the 512 "
                                  "sources of this draw cut to an eighth of their length (108,999,922 samples), "
                                  "scaled to this launch",
                "peak_source": "measured FP32 FMA rate on this GPU (aak_probe_fp32_tflops)",
                "flops_per_sample": fps, "flop_convention": "multiplies and adds one flop each (an FMA two), as the "
                "FMA-rate probe; per sample 60 + 54 n: 24 FMA-equivalents (48 flops) of the reference's per-harmonic "
                "algebra and 3 Bessel recurrence steps of 2 flops per harmonic; SFU work not counted",
                "kernel_ms": wave_ms}
    out = {
        "metric": "AAK samples/s & likelihoods/s on 1 B200 at mismatch<=1e-6 vs plain FP64 path",
        "value": value,
        "unit": "samples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64+f32 (FP64 phases and reductions, FP32 harmonic sums)",
        "data": "synthetic (seeded configuration-1 draw)",
        "config": bench_config(len(sources), world),
        "samples_per_gpu": int(N),
        "launch": "one CUDA graph replay per step: the spline solve, two clears and the split waveform kernel",
        "autotune": tune,
        "accuracy_vs_fp64": accuracy,
        "config2_split_vs_fp64": cfg2,
        "kernel_ms": split["kernel_ms"],
        "fp64_path": fp64,
        "plain_fp64_per_source": plain,
        "phase_product": phases,
        "tdi": tdi,
        "front_end_device_evolution": evolve_cmp,
        "roofline": roofline,
        "clocks": clk,
        "e2e": e2e,
        "gpu_launches": launches,
        "host_plan_seconds": t_plan,
    }
    model = None
    if args.parmap_points > 0 and rank == 0:
        out["parmap_warm_start"], model = run_parmap_warm_start(args.parmap_points, local_rank)
    if args.likelihood > 0:
        del hI, hII, hIh, hIIh
        wb.close()
        torch.cuda.empty_cache()
        free_b, total_b = torch.cuda.mem_get_info()
        try:
            out["likelihood"] = run_likelihood(args.likelihood, local_rank, model, args.fisher,
                                               with_cpu=rank == 0 and world == 1 and not args.no_cpu_baseline,
                                               rank=rank, world=world)
        except Exception as ex:  # one rank alone: report the failure, keep the waveform line
            if world > 1:
                raise
            from emri_kludge_suite_b200 import _lib

            out["likelihood"] = {"error": f"{type(ex).__name__}: {ex}",
                                 "detail": (_lib.lib().aak_last_error_detail() or b"").decode(errors="replace")}
        out["likelihood"]["device_free_gb_before"] = free_b / 1e9
    return out


# ----------------------------------------------------------------------------- profiling workloads
# Small cases of the same kernels for ncu captures (one GPU):
#   python bench.py --profile waveform   # 16 of the 512 sources, FP64 and split, default and tuned shapes
#   python bench.py --profile waveform512  # all 512 sources at an eighth of their length, split default shape, twice
#   python bench.py --profile phase      # the phase product of the same 16 sources, twice
#   python bench.py --profile fisher     # two 14-parameter Fisher matrices, 28 x 3.2e6-sample templates
#   python bench.py --profile tdi        # frequency-domain TDI of the waveform workload's 16 sources, twice
#   python bench.py --profile mlp        # warm-start network: forward on 2^20 points, a training step
#   python bench.py --profile likelihood # 32 config-4 templates, FP64 and FP32 transform + products
def profile_waveform():
    """16 of the 512 configuration-1 sources (every 32nd; 28,332,971 samples,
    n = 1..30): per precision the earlier default launch shape (FP64: 2
    CTAs/SM; split: 2 samples per thread, 2 CTAs/SM) and the autotuner's
    choice on the full batch (pre-pass, 1 sample per thread, 3 CTAs/SM: shape
    0, the default now), twice each, in the order FP64 v4, FP64 v0, split v5,
    split v0 (16 B/sample of outputs: 453 MB, above the 126 MB L2)."""
    import torch

    from emri_kludge_suite_b200.aak import WaveBatch

    src, _ = config1(SEED, 512)
    wb = WaveBatch(0)
    wb.plan(src[::32][:16], nmodes=NMODES)
    wb.upload()
    n = wb.total_samples
    hI = torch.empty(n, dtype=torch.float64, device="cuda")
    hII = torch.empty_like(hI)
    for precision, variant in ((0, 4), (0, 0), (1, 5), (1, 0)):
        wb.set_variant(precision, variant)
        for _ in range(2):
            wb.run(hI.data_ptr(), hII.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    assert wb.device_status() == 0
    print("waveform workload:", n, "samples")


def profile_waveform512():
    """All 512 configuration-1 sources with their observation times cut to an
    eighth (about 1.1e8 samples, 1.7 GB of FP64 outputs: above the 126 MB L2),
    so that, as on the full batch, a tile's phase-chain predecessor is a whole
    batch row earlier in the work queue; the split default launch shape, twice."""
    import torch

    from emri_kludge_suite_b200.aak import WaveBatch

    src, _ = config1(SEED, 512)
    for p in src:
        p["T"] = p["T"] / 8.0
        p["length"] = p["length"] // 8
    wb = WaveBatch(0)
    wb.plan(src, nmodes=NMODES)
    wb.upload()
    n = wb.total_samples
    hI = torch.empty(n, dtype=torch.float64, device="cuda")
    hII = torch.empty_like(hI)
    wb.set_variant(1, 0)
    for _ in range(2):
        wb.run(hI.data_ptr(), hII.data_ptr(), precision=1)
    torch.cuda.synchronize()
    assert wb.device_status() == 0
    print("waveform512 workload:", n, "samples")


def profile_phase():
    """The phase product of the same 16 sources as the waveform workload, twice
    (64 B/sample of outputs: 1.8 GB, above the 126 MB L2)."""
    import torch

    from emri_kludge_suite_b200.aak import WaveBatch

    src, _ = config1(SEED, 512)
    wb = WaveBatch(0)
    wb.plan(src[::32][:16], nmodes=NMODES)
    wb.upload()
    n = wb.total_samples
    out = torch.empty(8 * n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        wb.run_phase(out.data_ptr(), n)
    torch.cuda.synchronize()
    assert wb.device_status() == 0
    print("phase workload:", n, "samples")


def profile_fisher():
    """Two Fisher-matrix calls at the configuration-4 fiducial point: 28
    templates of 3.2e6 samples (1.43 GB of spectra, above the 126 MB L2)."""
    from emri_kludge_suite_b200.gpuAAK import GPUAAK

    length, dt = 3_200_000, 10.0
    x0 = np.array([0.785, 0.5, 8.0, 0.2, 1e6, 10.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.8, 2.0, 1.0])
    g = GPUAAK(1.0, 100, length, 100.0, dt, True, False)
    X = np.tile(x0, (28, 1))
    for i in range(14):
        X[2 * i, i] += 1e-6 * max(abs(x0[i]), 1.0)
        X[2 * i + 1, i] -= 1e-6 * max(abs(x0[i]), 1.0)
    for _ in range(2):
        G, st = g.fisher_gram(X, 1.0, return_status=True)
        assert np.all(st == 0) and np.all(np.isfinite(G))
    print("fisher workload: 28 x", length, "samples")


def profile_tdi():
    """The frequency-domain TDI of the same 16 sources as the waveform workload, twice."""
    from emri_kludge_suite_b200.aak import WaveBatch

    src, _ = config1(SEED, 512)
    wb = WaveBatch(0)
    for _ in range(2):
        rows, offs, st = wb.tdi_host(src[::32][:16])
    assert np.all(st == 0) and np.all(np.isfinite(rows))
    print("tdi workload:", int(offs[-1]), "bins")


def profile_mlp():
    import torch

    from emri_kludge_suite_b200 import parmap_mlp as P

    d = P.make_dataset(1 << 16, 5)
    m = P.ParMapMLP(0, seed=1)
    m.fit_norm(d["x"][d["valid"]], d["y"][d["valid"]])
    n = 1 << 20
    x = torch.tensor(np.tile(d["x"], (16, 1)).astype(np.float32), device="cuda")
    y = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    yt = torch.tensor(np.tile(np.nan_to_num(d["y"]), (16, 1)).astype(np.float32), device="cuda")
    for _ in range(2):
        m.forward_device(x.data_ptr(), y.data_ptr(), n)
        m.train_step_device(x.data_ptr(), yt.data_ptr(), 16384, 1e-3)
    torch.cuda.synchronize()
    print("mlp workload done")


def profile_likelihood():
    """32 configuration-4 templates (3.2e6 samples each) through the batched
    likelihood, FP64 then FP32 transform + compensated FP32 products (one batch
    of 32 each; 0.8 GB of FP64 spectra, above the 126 MB L2)."""
    from emri_kludge_suite_b200.gpuAAK import GPUAAK

    g = GPUAAK(1.0, 100, LIKE_LENGTH, 100.0, DT, True, False)
    nb = LIKE_LENGTH // 2 + 1
    rng = np.random.default_rng(3)
    d = rng.standard_normal(nb) + 1j * rng.standard_normal(nb)
    g.input_data(d, d, np.ones(nb), np.ones(nb))
    X = config4_templates(32)
    for prec in (0, 2):
        g.set_precision(prec)
        out, st = g.likelihood_batch(X, max_batch=32, return_status=True)
        assert np.all(st == 0) and np.all(np.isfinite(out))
    print("likelihood workload: 32 x", LIKE_LENGTH, "samples, FP64 and FP32 transforms")


PROFILES = {"waveform": profile_waveform, "waveform512": profile_waveform512, "phase": profile_phase, "fisher": profile_fisher,
            "tdi": profile_tdi, "mlp": profile_mlp, "likelihood": profile_likelihood}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--nsrc", type=int, default=512)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--likelihood", type=int, default=4096, help="config-4 templates to time (0: skip)")
    ap.add_argument("--config2-sources", type=int, default=512,
                    help="sources of the configuration-2 accuracy check (0: skip)")
    ap.add_argument("--plain-sources", type=int, default=512,
                    help="sources of the plain FP64 per-source baseline (0: skip; default: the whole batch)")
    ap.add_argument("--fisher", type=int, default=8, help="Fisher matrices to time at config-4 points (0: skip)")
    ap.add_argument("--tdi", type=int, default=1, help="time the frequency-domain TDI of 16 sources (0: skip)")
    ap.add_argument("--phases", type=int, default=1, help="time the AAK phase product of the batch (0: skip)")
    ap.add_argument("--evolve-compare", type=int, default=1,
                    help="time batch planning with the host and the device AK evolution (0: skip)")
    ap.add_argument("--parmap-points", type=int, default=1 << 20,
                    help="config-3 training points of the warm-start network (0: skip)")
    ap.add_argument("--profile", default=None, choices=sorted(PROFILES),
                    help="run one small profiling workload instead of the benchmark")
    args = ap.parse_args()
    if args.profile:
        PROFILES[args.profile]()
        return 0
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        # several ranks share one node's host cores: the multi-GPU line keeps the
        # headline, the end-to-end step and the likelihoods; the single-GPU
        # extras (plain path, configuration 2, phase product, TDI, Fisher,
        # planning comparison) run at N = 1
        args.plain_sources = args.config2_sources = args.fisher = args.tdi = args.phases = 0
        args.evolve_compare = 0

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        sources, _ = config1(SEED, args.nsrc)
        samples_per_step = []
        t_all = time.perf_counter()
        res = None
        for k in range(args.warmup + args.steps):
            res = cpu_reference(sources, budget_s=args.cpu_budget / max(1, args.steps))
            samples_per_step.append(res["value"])
        full = cpu_reference(sources, budget_s=1.0, untruncated=True).get("untruncated")
        vals = samples_per_step[args.warmup:] or samples_per_step
        v = float(np.mean(vals))
        line = {"metric": "AAK samples/s & likelihoods/s on 1 B200 at mismatch<=1e-6 vs plain FP64 path", "value": v,
                "unit": "samples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": (time.perf_counter() - t_all) * 1e3 / (args.warmup + args.steps),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded configuration-1 draw)", "impl": "reference",
                "config": bench_config(len(sources), world),
                "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "untruncated_check": full}
        print(json.dumps(line), flush=True)
        return 0

    if world > 1:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # before any CUDA call: the pool is spawned from a process without a CUDA context
        try:
            sources, _ = config1(SEED, args.nsrc)
            cpu = cpu_reference(sources, budget_s=args.cpu_budget, untruncated=True)
        except Exception as ex:  # reported, never fatal for the GPU arm
            cpu = {"value": None, "unit": "samples/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {ex}"}
    out = run_gpu(args, rank, world, local_rank)
    if rank == 0:
        if cpu is not None:
            out["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample") if k in cpu}
            if cpu.get("untruncated"):
                out["cpu_baseline"]["untruncated_check"] = cpu["untruncated"]
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
