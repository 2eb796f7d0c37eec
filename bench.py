#!/usr/bin/env python
"""Benchmark: survey xi_ell / P_ell jobs per second at 512^3 on one B200.

Workload (the precision-form configuration): a survey sector (RA, Dec in
[-30, 30] deg about +x, r in [500, 1500] Mpc/h, observer at the origin),
20M clustered data points (1e4 Gaussian clumps, sigma 5 Mpc/h) and 100M
uniform randoms, weights U[0.5, 1.5], TSC mass assignment on a 512^3 grid,
ell = 0, 2, 4, xi_ell with rmax 200 / dr 5 and P_ell with kmax 0.3 / dk 0.005.

One step = one survey job: assign D and R' = -alpha R (alpha = sum wD / sum wR)
into two device grids, form NN = D + R' on the device, run the Y_lm
correlator on NN and on RR = R', fetch both histogram tables and solve the
SE15 boundary correction (compute_xi) on the host.  `value` is jobs/s of the
FP32-mixed form with the catalogs already resident in HBM; `e2e` is the same
job through the C ABI from pinned host buffers (host->device copies and the
result readback inside the timed region); `fp64_gpu` is the plain FP64 GPU
form on the same inputs.  Inputs are GBs, far larger than the 126 MB L2, so
no explicit L2 flush is needed between steps.

`cpu_baseline` and `--impl reference` time the reference's own C++ classes
(compiled from its sources with the project FFT shim, OpenMP, all host
threads) on whole jobs of the same workload and the same catalogs; the
reference's FP64 tables from the baseline job are what `vs_reference_fp64`
measures both GPU forms against.
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "xi_ell/P_ell survey jobs/s at 512^3, ell<=4 (FP32-mixed; FP64 GPU alongside)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ngrid", type=int, default=512)
    ap.add_argument("--nd", type=float, default=20e6)
    ap.add_argument("--nr", type=float, default=100e6)
    ap.add_argument("--maxell", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-boxes", type=int, default=64)
    ap.add_argument("--only-batched", action="store_true")
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--only-served", action="store_true")
    ap.add_argument("--served-jobs", type=int, default=24)
    ap.add_argument("--served-slots", type=int, default=2)
    ap.add_argument("--e2e-slots", type=int, default=2)
    ap.add_argument("--mix-jobs", type=int, default=48)
    ap.add_argument("--mix-rate", type=float, default=6.0)
    ap.add_argument("--reference-budget-s", type=float, default=150.0)
    # Wraps the FP32 form's timed steps in fc_profiler_range, for a launch
    # list taken with `ncu --profile-from-start off`.
    ap.add_argument("--profile-range", action="store_true")
    return ap.parse_args()


# ------------------------------------------------------------ environment

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Dist:
    """Barrier and max-reduction across ranks (gloo; no data-path traffic)."""

    def __init__(self, world):
        self.world = world
        self.pg = None
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during a region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# ------------------------------------------------------------------ job

class Workload:
    def __init__(self, a):
        from fftcorr_b200 import mocks
        self.ngrid = (a.ngrid,) * 3
        self.nd = int(a.nd)
        self.nr = int(a.nr)
        self.maxell = a.maxell
        self.rmax, self.dr = 200.0, 5.0
        self.kmax, self.dk = 0.3, 0.005
        self.sector = mocks.Sector()
        self.posmin, self.cell = mocks.survey_box(self.sector, self.rmax, self.ngrid)

    def describe(self):
        return {"workload": "survey xi_ell+P_ell job: sector r 500-1500 Mpc/h, "
                            "RA/Dec +-30 deg, clustered data + uniform randoms",
                "grid": list(self.ngrid), "n_data": self.nd, "n_randoms": self.nr,
                "scheme": "TSC", "maxell": self.maxell, "rmax": self.rmax,
                "dr": self.dr, "kmax": self.kmax, "dk": self.dk,
                "cell_size": round(self.cell, 6),
                "l2": "inputs and grids are GBs (> 126 MB L2); no flush needed"}

    def catalogs(self, seed_offset=0):
        from fftcorr_b200 import mocks
        D = mocks.sector_clustered(self.nd, 2 + 100 * seed_offset, sector=self.sector)
        R = mocks.sector_randoms(self.nr, 3 + 100 * seed_offset, sector=self.sector)
        R[:, 3] *= -(D[:, 3].sum() / R[:, 3].sum())
        return D, R


class SurveyJob:
    """Device objects for one survey job, reused across steps."""

    def __init__(self, w, precision):
        import fftcorr_b200 as fb
        from fftcorr_b200.correlate import TSC_ALIASED_CORRECTION
        self.fb = fb
        self.w = w
        # Grids of the form's precision: the FP32-mixed form's cells are FP32.
        self.gA = fb.ConfigSpaceGrid.from_geometry(w.ngrid, w.posmin, w.cell,
                                                   precision=precision)
        self.gB = fb.ConfigSpaceGrid.from_geometry(w.ngrid, w.posmin, w.cell,
                                                   precision=precision)
        tsc = fb.DistributionScheme.TRIANGULAR_SHAPED_CLOUD
        self.maA = fb.MassAssignor(self.gA, tsc, False, 0)
        self.maB = fb.MassAssignor(self.gB, tsc, False, 0)
        self.corr = fb.Correlator(w.ngrid, w.cell, w.posmin, TSC_ALIASED_CORRECTION,
                                  w.rmax, w.dr, w.kmax, w.dk, w.maxell,
                                  precision=precision)

    def _reset(self):
        from fftcorr_b200 import _lib
        _lib.call("fc_grid_clear", self.gA.handle)
        _lib.call("fc_grid_clear", self.gB.handle)
        self.maA.clear()
        self.maB.clear()

    def _correlate(self):
        from fftcorr_b200.correlate import compute_xi
        self.corr.autocorrelate(self.gA)
        nn = self.corr.results()
        self.corr.autocorrelate(self.gB)
        rr = self.corr.results()
        xi = compute_xi(nn["rhist"].T, rr["rhist"].T)
        return nn, rr, xi

    def run_device(self, dD, nD, dR, nR):
        self._reset()
        self.maA.add_particles_device(dD, nD)
        self.maB.add_particles_device(dR, nR)
        self.gA.add_grid(self.gB)
        return self._correlate()

    def run_host(self, D, R):
        self._reset()
        self.maA.add_particles(D)
        self.maB.add_particles(R)
        self.gA.add_grid(self.gB)
        return self._correlate()

    def result_bytes(self, nn):
        per = sum(np.asarray(v).nbytes for k, v in nn.items() if k != "zerolag") + 8
        return 2 * per


def device_copy(arr):
    from fftcorr_b200 import _lib
    p = ctypes.c_void_p()
    _lib.call("fc_device_malloc", arr.nbytes, ctypes.byref(p))
    _lib.call("fc_memcpy_htod", p, arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes)
    return p.value


class DeviceTimer:
    def __init__(self):
        from fftcorr_b200 import _lib
        self._lib = _lib
        self.h = ctypes.c_void_p()
        _lib.call("fc_timer_create", ctypes.byref(self.h))

    def start(self):
        self._lib.call("fc_timer_start", self.h)

    def stop(self):
        s = ctypes.c_double()
        self._lib.call("fc_timer_stop", self.h, ctypes.byref(s))
        return s.value


def kernel_profile(job, dD, nD, dR, nR):
    """Per-kernel-family device time of one job with profiling on."""
    from fftcorr_b200 import _lib
    _lib.call("fc_corr_set_profiling", job.corr.handle, 1)
    job.run_device(dD, nD, dR, nR)
    arr = (_lib.KernelTime * 32)()
    n = ctypes.c_int()
    _lib.call("fc_corr_profile", job.corr.handle, arr, 32, ctypes.byref(n))
    _lib.call("fc_corr_set_profiling", job.corr.handle, 0)
    out = {}
    for i in range(n.value):
        out[arr[i].name.decode()] = {"launches": arr[i].launches,
                                     "seconds": arr[i].seconds}
    return out


# DRAM bytes (read + write) per launch of the survey pass kernels at 512^3,
# FP32-mixed, from ncu captures (dram__bytes_read.sum + dram__bytes_write.sum,
# or dram__bytes.sum.per_second x gpu__time_duration.sum) of `python -m
# fftcorr_b200.cases survey --precision fp32`, one kernel per capture, whose
# passes run on the benchmark's grid and work arrays (the summaries are
# kept with the profiles).
TRAFFIC_PER_LAUNCH_512 = {
    "zfwd": 1048.8e6,
    "zfwd2": 1603.7e6,
    "yfwd": 1063.2e6,
    "xcorr": 1375.7e6,
    "xcorr00": 801.0e6,
    "yinv": 144.4e6,
    "zinv": 49.1e6,
}


def subgrid_dims(corr):
    """(r-subgrid edge, k-subgrid shape) of a correlator."""
    from fftcorr_b200 import _lib
    rs = (ctypes.c_int * 3)()
    ks = (ctypes.c_int * 3)()
    _lib.call("fc_corr_dims", corr.handle, None, None, None, rs, ks)
    return rs[0], tuple(ks)


def algorithmic_bytes(family, w, precision, rs, ks):
    """HBM bytes one launch must move at minimum (each operand read once,
    each result written once).  Survey fused passes, N = N0 N1 N2 cells,
    h = N2/2 + 1, Nc = N0 N1 h complex cells of e bytes (8 FP32, 16 FP64):
      zfwd   density in (N * s) + W out (Nc * e)
      zfwd2  the z pass of two terms at once: density in (N * s) + two W
             out (2 Nc e)
      yfwd   W in and out (2 Nc e)
      xcorr  W and G in (2 Nc e) + x-pruned Wr out (rs N1 h e)
             + k-subgrid weight read (s bytes a cell) and FP64
             read-modify-write (K0 K1 K2 * (16 + s))
      xcorr00  the ell = 0 term of an autocorrelation: G in (Nc e) + Wr out
             + k-subgrid as xcorr (its transform is a multiple of G)
      yinv   Wr in (rs N1 h e) + Wry out (rs rs h e)
      zinv   Wry in (rs rs h e) + r-subgrid weight read (s bytes a cell)
             and FP64 read-modify-write (rs^3 * (16 + s))"""
    s = 8 if precision == "fp64" else 4
    e = 2 * s
    n0, n1, n2 = w.ngrid
    n = n0 * n1 * n2
    h = n2 // 2 + 1
    nc = n0 * n1 * h
    kc = ks[0] * ks[1] * ks[2]
    table = {
        "zfwd": n * s + nc * e,
        "zfwd2": n * s + 2 * nc * e,
        "yfwd": 2 * nc * e,
        "xcorr": 2 * nc * e + rs * n1 * h * e + kc * (16 + s),
        "xcorr00": nc * e + rs * n1 * h * e + kc * (16 + s),
        "yinv": rs * n1 * h * e + rs * rs * h * e,
        "zinv": rs * rs * h * e + rs ** 3 * (16 + s),
        "weight": n * 8 + n * s,
        "copy_pad": n * 8 + n * s,
        "conj_mul": 3 * nc * e,
        "r2c": n * s + nc * e,
        "c2r": nc * e + n * s,
    }
    return table.get(family)


# --------------------------------------------------------- batched form

def batched_boxes(nboxes, seed0=4):
    """64 periodic mock boxes: L ~ U[1000, 2000] Mpc/h, N from
    {128, 192, 256, 384}^3, Np log-uniform in [0.5M, 8M], clustered (1e4
    centres, sigma 5 Mpc/h), seed 4 + i; catalogs generated on the device."""
    from fftcorr_b200 import catalog
    boxes, desc = [], []
    for i in range(nboxes):
        rng = np.random.default_rng(seed0 + i)
        L = float(rng.uniform(1000.0, 2000.0))
        n = int(rng.choice([128, 192, 256, 384]))
        npart = int(np.exp(rng.uniform(np.log(0.5e6), np.log(8e6))))
        cat = catalog.clustered_box(npart, L, seed=seed0 + i, ncentres=10000,
                                    sigma=5.0)
        boxes.append(((n, n, n), L / n, cat))
        desc.append((n, npart))
    return boxes, desc


def run_batched(a, timed_fn):
    from fftcorr_b200 import _lib
    from fftcorr_b200.batch import PeriodicBatch
    from fftcorr_b200.correlate import NO_CORRECTION
    from fftcorr_b200.particle_mesh import DistributionScheme
    boxes, desc = batched_boxes(a.batch_boxes)
    out = {}
    for prec in ("fp32", "fp64"):
        if prec == "fp64" and a.no_fp64:
            continue
        t0 = time.perf_counter()
        b = PeriodicBatch(boxes, DistributionScheme.CLOUD_IN_CELL, rmax=200.0,
                          dr=5.0, kmax=0.1, dk=0.005, maxell=2,
                          window_correct=NO_CORRECTION, precision=prec)
        build_s = time.perf_counter() - t0
        for _ in range(max(3, a.warmup)):
            b.run()
        n0 = _lib.launch_count()
        secs = [b.run() for _ in range(a.steps)]
        info = b.info
        t = float(np.sum(secs))
        out[prec] = {
            "value": len(boxes) * a.steps / t, "unit": "boxes/s",
            "ms_per_batch": 1000.0 * t / a.steps,
            "ms_per_batch_min": 1000.0 * min(secs),
            "build_and_tune_s": build_s, "info": info,
            "host_launches_per_replay": (_lib.launch_count() - n0) // max(1, a.steps),
        }
        del b
    npart = sum(d[1] for d in desc)
    cells = sum(d[0] ** 3 for d in desc)
    return {"workload": f"{len(boxes)} periodic boxes, L U[1000,2000], N in "
                        "{128,192,256,384}^3, Np log-uniform [0.5M, 8M] clustered "
                        "(1e4 centres, sigma 5), CIC, ell<=2, rmax 200 dr 5, "
                        "kmax 0.1 dk 0.005; one CUDA graph per replay",
            "particles": npart, "cells": cells, "forms": out}


# ----------------------------------------------------------- served form

def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def survey_job_spec(w, seed, precision, nd=None, nr=None, ngrid=None, maxell=None,
                    want_rr=True):
    """The headline survey job as a served request: clustered data and
    uniform randoms in the sector, generated on the device from seeds."""
    from fftcorr_b200 import mocks
    from fftcorr_b200.correlate import TSC_ALIASED_CORRECTION
    from fftcorr_b200.particle_mesh import DistributionScheme
    from fftcorr_b200.serve import (CAT_SECTOR_CLUSTERED, CAT_SECTOR_UNIFORM,
                                    JobSpec, catalog_spec)
    ngrid = ngrid or w.ngrid
    posmin, cell = mocks.survey_box(w.sector, w.rmax, ngrid)
    data = catalog_spec(CAT_SECTOR_CLUSTERED, n=nd or w.nd, ncentres=10000, sigma=5.0,
                        wmin=0.5, wmax=1.5, seed=seed)
    rand = catalog_spec(CAT_SECTOR_UNIFORM, n=nr or w.nr, wmin=0.5, wmax=1.5,
                        seed=seed + 1)
    return JobSpec("survey", ngrid, cell, data, rand, posmin=posmin,
                   scheme=DistributionScheme.TRIANGULAR_SHAPED_CLOUD,
                   window=TSC_ALIASED_CORRECTION, rmax=w.rmax, dr=w.dr,
                   kmax=w.kmax, dk=w.dk,
                   maxell=w.maxell if maxell is None else maxell,
                   precision=precision, want_rr=want_rr)


def host_job_spec(w, D, R, precision):
    """The headline job as a served request on the pinned host catalogs
    (the randoms already carry -alpha in their weights; the server's own
    alpha is then -1 and NN = D - alpha R as in SurveyJob)."""
    from fftcorr_b200 import mocks
    from fftcorr_b200.correlate import TSC_ALIASED_CORRECTION
    from fftcorr_b200.particle_mesh import DistributionScheme
    from fftcorr_b200.serve import CAT_HOST, JobSpec, catalog_spec
    posmin, cell = mocks.survey_box(w.sector, w.rmax, w.ngrid)
    return JobSpec("survey", w.ngrid, cell, catalog_spec(CAT_HOST, posw=D),
                   catalog_spec(CAT_HOST, posw=R), posmin=posmin,
                   scheme=DistributionScheme.TRIANGULAR_SHAPED_CLOUD,
                   window=TSC_ALIASED_CORRECTION, rmax=w.rmax, dr=w.dr,
                   kmax=w.kmax, dk=w.dk, maxell=w.maxell, precision=precision)


def run_e2e_served(a, w, D, R, timer, slots=2):
    """End to end through the serving API: every job copies its catalogs
    from pinned host memory and reads its tables back; with two slots one
    job's copies overlap the other's kernels."""
    from fftcorr_b200.serve import Server
    srv = Server(served_budget(), slots=slots)
    warm = [srv.submit(host_job_spec(w, D, R, "fp32")) for _ in range(slots)]
    for t in warm:
        srv.wait(t)
    timer.start()
    tickets = [srv.submit(host_job_spec(w, D, R, "fp32")) for _ in range(a.steps)]
    for t in tickets:
        srv.wait(t)
    secs = timer.stop()
    bad = [srv.info(t)["message"] for t in tickets if srv.info(t)["status"] != 0]
    srv.close()
    if bad:
        raise RuntimeError("served end-to-end jobs failed: " + "; ".join(bad))
    return secs


def served_budget():
    """180 GB, or the free device memory less a margin when that is less."""
    from fftcorr_b200 import _lib
    free, total = ctypes.c_size_t(), ctypes.c_size_t()
    _lib.call("fc_device_memory", ctypes.byref(free), ctypes.byref(total))
    return int(min(180 * 10**9, free.value - (6 << 30)))


def run_served_saturated(a, w, precision, timer):
    """All requests queued at once: device-timed throughput of the server."""
    from fftcorr_b200.serve import Server
    srv = Server(served_budget(), slots=a.served_slots)
    # One warm-up job per slot, so every slot's resident objects exist.
    warm = [srv.submit(survey_job_spec(w, 900 + i, precision))
            for i in range(a.served_slots)]
    for t in warm:
        srv.wait(t)
    specs = [survey_job_spec(w, 1000 + 10 * i, precision) for i in range(a.served_jobs)]
    timer.start()
    tickets = [srv.submit(s) for s in specs]
    for t in tickets:
        srv.wait(t)
    secs = timer.stop()
    lat = [srv.info(t)["latency_s"] for t in tickets]
    run = [srv.info(t)["run_s"] for t in tickets]
    bad = [srv.info(t)["message"] for t in tickets if srv.info(t)["status"] != 0]
    st = srv.stats()
    srv.close()
    return {"value": len(specs) / secs, "unit": "jobs/s", "jobs": len(specs),
            "slots": a.served_slots, "device_s": secs,
            "p50_latency_s": _pct(lat, 50), "p99_latency_s": _pct(lat, 99),
            "mean_run_s": float(np.mean(run)), "peak_running": st["peak_running"],
            "peak_bytes": st["peak_bytes"], "errors": bad}


def snap7(n):
    """Nearest even 7-smooth integer (2^a 3^b 5^c 7^d)."""
    best = None
    for m in range(max(2, n - 64), n + 65):
        if m % 2:
            continue
        k = m
        for p in (2, 3, 5, 7):
            while k % p == 0:
                k //= p
        if k == 1 and (best is None or abs(m - n) < abs(best - n)):
            best = m
    return best


def mix_job(w, i, rng):
    from fftcorr_b200.particle_mesh import DistributionScheme
    from fftcorr_b200.serve import CAT_CLUSTERED_BOX, JobSpec, catalog_spec
    n = snap7(int(round(np.exp(rng.uniform(np.log(64), np.log(1024))))))
    maxell = int(rng.choice([0, 2, 4]))
    npart = int(np.exp(rng.uniform(np.log(0.1e6), np.log(50e6))))
    want_rr = bool(rng.random() < 0.5)      # xi job (NN and RR) or P job (NN)
    if rng.random() < 0.5:
        L = float(rng.uniform(1000.0, 2000.0))
        data = catalog_spec(CAT_CLUSTERED_BOX, n=npart, boxsize=L, ncentres=10000,
                            sigma=5.0, seed=5000 + i)
        spec = JobSpec("periodic", (n, n, n), L / n, data,
                       scheme=DistributionScheme.CLOUD_IN_CELL, rmax=200.0, dr=5.0,
                       kmax=0.1, dk=0.005, maxell=maxell, precision="fp32")
        return spec, ("periodic", n, maxell, npart)
    nd = max(1, npart // 5)
    spec = survey_job_spec(w, 5000 + 7 * i, "fp32", nd=nd, nr=npart, ngrid=(n, n, n),
                           maxell=maxell, want_rr=want_rr)
    return spec, ("survey", n, maxell, npart)


def run_served_mix(a, w):
    """Poisson arrivals of mixed periodic / survey, xi / P jobs."""
    from fftcorr_b200.serve import Server
    rng = np.random.default_rng(5)
    jobs = [mix_job(w, i, rng) for i in range(a.mix_jobs)]
    gaps = rng.exponential(1.0 / a.mix_rate, len(jobs))
    srv = Server(served_budget(), slots=a.served_slots)
    t0 = time.perf_counter()
    tickets = []
    due = t0
    for (spec, _), gap in zip(jobs, gaps):
        due += gap
        delay = due - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets.append(srv.submit(spec))
    for t in tickets:
        srv.wait(t)
    wall = time.perf_counter() - t0
    infos = [srv.info(t) for t in tickets]
    st = srv.stats()
    srv.close()
    lat = [i["latency_s"] for i in infos]
    return {"value": len(jobs) / wall, "unit": "jobs/s (host wall clock)",
            "jobs": len(jobs), "arrival_rate_per_s": a.mix_rate,
            "p50_latency_s": _pct(lat, 50), "p99_latency_s": _pct(lat, 99),
            "max_latency_s": max(lat), "slots": a.served_slots,
            "peak_running": st["peak_running"], "peak_bytes": st["peak_bytes"],
            "budget": st["budget"], "evictions": st["evictions"],
            "admitted_out_of_order": st["admitted_out_of_order"],
            "errors": [i["message"] for i in infos if i["status"] != 0],
            "mix": "N^3 log-uniform [64^3, 1024^3] snapped to even 7-smooth, "
                   "ell_max from {0,2,4}, periodic/survey 50/50, Np log-uniform "
                   "[0.1M, 50M], xi (NN+RR) / P (NN) 50/50, FP32-mixed, seed 5"}


def run_served(a, w, timer):
    out = {"workload_512": "served survey xi_ell+P_ell jobs at 512^3, ell<=4, "
                           "20M clustered data + 100M randoms generated on the "
                           "device per job, all queued at once"}
    out["fp32"] = run_served_saturated(a, w, "fp32", timer)
    if not a.no_fp64:
        out["fp64"] = run_served_saturated(a, w, "fp64", timer)
        out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    out["mix"] = run_served_mix(a, w)
    return out


# --------------------------------------------------------- CPU baseline

REFERENCE_LABEL = ("reference C++ (cc/ MassAssignor + Correlator, -O3 OpenMP "
                   "-DFFTSLAB, project FFT shim; FFTW unavailable)")


def reference_job(w, D, R, threads):
    """One whole survey job through the reference's own C++ classes on the
    host cores: MassAssignor (CLI buffer 1e6) on D and on R' into two grids,
    NN = D + R', Correlator autocorrelation of NN and of RR = R' at the
    workload's full size.  Timed by the wall clock around the calls.
    Returns (seconds, nn, rr, phases) or None when oracle/_ref is missing."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import ref_lib
    if not ref_lib.available("omp"):
        return None
    t0 = time.perf_counter()
    nn, rr, phases = ref_lib.survey_job(D, R, w.ngrid, w.posmin, w.cell, 2, w.rmax,
                                        w.dr, w.kmax, w.dk, w.maxell, scheme=1,
                                        build="omp")
    secs = time.perf_counter() - t0
    for key, res in (("nn", nn), ("rr", rr)):
        setup, _, fft, extract, mult, ylm, hist, total = res["timers"]
        phases[key + "_reference_timers"] = {
            "setup": setup, "fft": fft, "extract": extract, "multiply": mult,
            "ylm": ylm, "histogram": hist, "total": total}
    return secs, nn, rr, phases


def reference_sample_desc(w, threads, phases):
    return (f"{REFERENCE_LABEL} on {threads} threads: one whole job on the full "
            f"workload ({w.nd} data + {w.nr} randoms assigned, two "
            f"{w.ngrid[0]}^3 ell<={w.maxell} correlations), wall clock; "
            f"mass assignment {phases['mass_assign_s']:.1f} s, correlations "
            f"{phases['correlate_s']:.1f} s")


def maxdev_over_rms0(got, ref):
    """max |got_l - ref_l| / rms(ref_0) for every multipole row l."""
    got, ref = np.atleast_2d(got), np.atleast_2d(ref)
    rms0 = float(np.sqrt(np.mean(ref[0] ** 2)))
    return [float(np.max(np.abs(got[i] - ref[i]))) / rms0 for i in range(ref.shape[0])]


def deviations(res, ref):
    """Per-multipole deviations of one form's (nn, rr, xi) from another's."""
    (nn, rr, xi), (rnn, rrr, rxi) = res, ref
    return {"xi": maxdev_over_rms0(xi.T, rxi.T),
            "NN": maxdev_over_rms0(nn["rhist"], rnn["rhist"]),
            "RR": maxdev_over_rms0(rr["rhist"], rrr["rhist"]),
            "P": maxdev_over_rms0(nn["khist"], rnn["khist"]),
            "counts_equal": bool(np.array_equal(nn["rcounts"], rnn["rcounts"]) and
                                 np.array_equal(nn["kcounts"], rnn["kcounts"]))}


# ------------------------------------------------------------------ main

def run_reference(a, rank, world):
    """The reference arm: whole jobs through the reference C++ on all host
    threads, as many as fit a bounded run (at least one); rank 0 only."""
    if rank != 0:
        return
    w = Workload(a)
    threads = os.cpu_count() or 1
    D, R = w.catalogs()
    from oracle import ref_lib
    if not ref_lib.available("omp"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libfcref_omp.so not built"}))
        return
    times = []
    phases = None
    budget = a.reference_budget_s
    t_start = time.perf_counter()
    while len(times) < max(1, a.steps):
        out = reference_job(w, D, R, threads)
        times.append(out[0])
        phases = out[3]
        if time.perf_counter() - t_start + out[0] > budget:
            break
    secs = float(np.mean(times))
    value = 1.0 / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "jobs/s",
        "n_gpus": 0, "steps": len(times), "warmup": 0,
        "steps_requested": a.steps, "warmup_requested": a.warmup,
        "ms_per_step": 1000.0 * secs, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded mock survey catalogs, see config)",
        "config": bench_config(w, world),
        "timing": ("every step is one whole job on the full workload, timed by "
                   "the wall clock; as many steps as fit the arm's bounded run "
                   f"({budget:.0f} s), no warm-up jobs (CPU code; each job "
                   "allocates and pages in its own arrays); the host compute_xi "
                   "(about 1 ms) is not included"),
        "job_seconds": times,
        "phases": phases,
        "cpu_baseline": {"value": value, "unit": "jobs/s", "cores": threads,
                         "kind": "reference",
                         "sample": reference_sample_desc(w, threads, phases)},
        "e2e": {"value": value, "unit": "jobs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def bench_config(w, world):
    return dict(w.describe(), parallelism=f"replicas x{world}")


def main():
    a = parse()
    rank, world, local = dist_env()
    if a.impl == "reference":
        run_reference(a, rank, world)
        return
    from fftcorr_b200 import _lib
    _lib.call("fc_set_device", local)
    dist = Dist(world)
    if a.only_batched:
        if rank == 0:
            print(json.dumps({"batched": run_batched(a, None)}))
        dist.close()
        return
    if a.only_served:
        if rank == 0:
            print(json.dumps({"served": run_served(a, Workload(a), DeviceTimer())}))
        dist.close()
        return
    w = Workload(a)
    t_gen = time.perf_counter()
    D, R = w.catalogs(seed_offset=rank)
    t_gen = time.perf_counter() - t_gen
    nD, nR = D.shape[0], R.shape[0]
    for arr in (D, R):
        _lib.call("fc_host_register", arr.ctypes.data_as(ctypes.c_void_p), arr.nbytes)
    dD, dR = device_copy(D), device_copy(R)
    timer = DeviceTimer()

    def timed(fn, steps, warmup, profile=False):
        for _ in range(warmup):
            fn()
        dist.barrier()
        n0 = _lib.launch_count()
        if profile:
            _lib.call("fc_profiler_range", 1)
        timer.start()
        for _ in range(steps):
            out = fn()
        secs = timer.stop()
        if profile:
            _lib.call("fc_profiler_range", 0)
        timed.launches = _lib.launch_count() - n0
        return dist.max(secs), out

    # FP32-mixed form: device-resident inputs, then end to end from host.
    job = SurveyJob(w, "fp32")
    with ClockSampler(local) as clocks:
        t_dev, (nn, rr, xi) = timed(lambda: job.run_device(dD, nD, dR, nR),
                                    a.steps, a.warmup, a.profile_range)
    launches_dev = timed.launches
    rs, ks = subgrid_dims(job.corr)
    t_e2e_sync, _ = timed(lambda: job.run_host(D, R), a.steps, 1)
    prof = kernel_profile(job, dD, nD, dR, nR)
    ma_stats = job.maB._stats()
    res32 = (nn, rr, xi)
    result_bytes = job.result_bytes(nn)
    del job
    t_e2e = dist.max(run_e2e_served(a, w, D, R, timer, slots=a.e2e_slots))

    fp64 = None
    res64 = None
    if not a.no_fp64:
        job64 = SurveyJob(w, "fp64")
        t64, (nn64, rr64, xi64) = timed(lambda: job64.run_device(dD, nD, dR, nR),
                                        a.steps, 1)
        prof64 = kernel_profile(job64, dD, nD, dR, nR)
        res64 = (nn64, rr64, xi64)
        del job64
        fp64 = {
            "value": world * a.steps / t64, "unit": "jobs/s",
            "ms_per_step": 1000.0 * t64 / a.steps,
            "fp32_vs_fp64_gpu_maxdev_over_rms_0": deviations(res32, res64),
            "kernels": prof64,
        }

    value = world * a.steps / t_dev
    e2e_value = world * a.steps / t_e2e
    peak, peak_kind = measured_hbm_peak()
    # Roofline of the dominant hand-written kernel, and every family's
    # fraction beside it.
    roof = None
    fam_roof = {}
    for fam, v in prof.items():
        alg = algorithmic_bytes(fam, w, "fp32", rs, ks)
        if alg and v["launches"]:
            per = v["seconds"] / v["launches"]
            fam_roof[fam] = {"achieved_gbs": alg / per / 1e9,
                             "frac": alg / per / 1e9 / peak,
                             "us_per_launch": per * 1e6,
                             "bytes_per_launch": alg,
                             "traffic": (TRAFFIC_PER_LAUNCH_512.get(fam)
                                         if tuple(w.ngrid) == (512, 512, 512)
                                         else None)}
    ours = {k: v for k, v in prof.items()
            if k not in ("r2c", "c2r") and k in fam_roof}
    if ours:
        fam = max(ours, key=lambda k: ours[k]["seconds"])
        f = fam_roof[fam]
        roof = {"kernel": fam, "bound": "hbm", "achieved": f["achieved_gbs"],
                "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                "frac": f["frac"], "bytes_per_launch": f["bytes_per_launch"],
                "us_per_launch": f["us_per_launch"],
                "traffic": (TRAFFIC_PER_LAUNCH_512.get(fam)
                            if tuple(w.ngrid) == (512, 512, 512) else None)}

    batched = None if a.no_batched else run_batched(a, None)
    served = None if a.no_served else run_served(a, w, timer)

    # CPU baseline: one whole job through the reference C++ on the same
    # catalogs; its FP64 tables are also the reference the GPU forms'
    # deviations are measured against.
    cpu = None
    vs_reference = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        out = reference_job(w, D, R, threads)
        if out is not None:
            secs, rnn, rrr, phases = out
            cpu = {"value": 1.0 / secs, "unit": "jobs/s", "cores": threads,
                   "kind": "reference",
                   "sample": reference_sample_desc(w, threads, phases),
                   "phases": phases}
            from fftcorr_b200.correlate import compute_xi
            ref = (rnn, rrr, compute_xi(rnn["rhist"].T, rrr["rhist"].T))
            vs_reference = {
                "what": "max |GPU - reference FP64| / rms(row 0) per multipole "
                        "(ell = 0, 2, 4) of xi (compute_xi of NN, RR), the NN and "
                        "RR correlation histograms and P (NN); same catalogs",
                "fp32_mixed": deviations(res32, ref),
                "fp64": deviations(res64, ref) if fp64 else None,
            }

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "jobs/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000.0 * t_dev / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded mock survey catalogs, see config)",
            "config": bench_config(w, world),
            "form": "fp32-mixed, inputs resident in HBM",
            "e2e": {"value": e2e_value, "unit": "jobs/s",
                    "h2d_bytes_per_step": int(D.nbytes + R.nbytes),
                    "d2h_bytes_per_step": int(result_bytes),
                    "ms_per_step": 1000.0 * t_e2e / a.steps,
                    "api": f"fftcorr_b200.serve.Server ({a.e2e_slots} slots), catalogs "
                           "copied from pinned host memory every job, tables "
                           "read back every job"},
            "e2e_sync": {"value": world * a.steps / t_e2e_sync, "unit": "jobs/s",
                         "ms_per_step": 1000.0 * t_e2e_sync / a.steps,
                         "api": "MassAssignor.add_particles + Correlator."
                                "autocorrelate, one job at a time"},
            "fp64_gpu": fp64,
            "roofline": roof,
            "kernel_roofline": fam_roof,
            "kernels": prof,
            "mass_assign_s_per_flush": {"sort": ma_stats.sort_time,
                                        "scatter": ma_stats.window_time},
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "vs_reference_fp64": vs_reference,
            "gpu_launches": launches_dev,
            "catalog_generation_s": t_gen,
            "batched": batched,
            "served": served,
        }
        print(json.dumps(line))
    for p in (dD, dR):
        _lib.call("fc_device_free", ctypes.c_void_p(p))
    dist.close()


if __name__ == "__main__":
    main()
