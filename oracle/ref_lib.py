"""ctypes front end to the compiled reference (oracle/_ref, TEST INFRASTRUCTURE).

The libraries are the unmodified reference C++ classes compiled by
oracle/Makefile against the project FFT shim, reached through the C entry
points of oracle/ref_harness.cc.  Three builds:

  "parity"  libfcref.so       1 thread, -O2 -ffp-contract=off
  "pomp"    libfcref_pomp.so  the parity flags plus OpenMP and the per-slab
                              FFT split; its correlator outputs are bit for
                              bit those of the parity build (pinned by
                              tests/test_oracle.py), so it stands in for it
                              on the large grids
  "omp"     libfcref_omp.so   -O3 -march=x86-64-v3 OpenMP, the build that is
                              timed as the CPU baseline

Only tests, the smoke check and the CPU-baseline leg of bench.py use this
module; the fftcorr_b200 package never imports it.

Reference entry points driven (see ref_harness.cc):
  MassAssignor add_particles_to_buffer + flush  cc/particle_mesh/mass_assignor.h:72-191
  PeriodicCorrelator / Correlator               cc/correlate/correlator.h:254-505
"""
import ctypes
import math
import os

import numpy as np

_REF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")
_FILES = {"parity": "libfcref.so", "pomp": "libfcref_pomp.so", "omp": "libfcref_omp.so"}
_libs = {}


def path(build="parity"):
    return os.path.join(_REF, _FILES[build])


def available(build="parity"):
    return os.path.exists(path(build))


def lib(build="parity"):
    if build not in _libs:
        p = path(build)
        if not os.path.exists(p):
            raise RuntimeError(f"{p} is missing; run `make -C oracle ref`")
        L = ctypes.CDLL(p)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.fcref_mass_assign.argtypes = [dp, ctypes.c_long, ip, dp, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_long,
                                        dp, dp, ctypes.c_int]
        L.fcref_mass_assign.restype = ctypes.c_int
        d = ctypes.c_double
        L.fcref_correlate.argtypes = [ctypes.c_int, dp, dp, ip, d, dp, ctypes.c_int,
                                      d, d, d, d, ctypes.c_int, dp, ip, dp, dp, ip,
                                      dp, dp, ctypes.c_int, dp]
        L.fcref_correlate.restype = ctypes.c_int
        L.fcref_last_error.restype = ctypes.c_char_p
        _libs[build] = L
    return _libs[build]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _check(L, rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what} failed: {L.fcref_last_error().decode()}")


def mass_assign(posw, shape, posmin, cell, scheme, periodic=False,
                buffer_size=1000000, build="parity", grid=None):
    """Reference MassAssignor over an (n, 4) catalog, then flush().

    Returns (grid, stats); stats = [num_added, num_skipped, totw, totwsq,
    sort_time, window_time].  ``grid`` (C-contiguous FP64) receives the
    result when given.  The CLI's particle buffer is 1e6
    (cc/fftcorr.cc:354-355).
    """
    L = lib(build)
    posw = np.ascontiguousarray(posw, dtype=np.float64)
    shape = tuple(int(s) for s in shape)
    if grid is None:
        grid = np.zeros(shape)
    st = np.zeros(6)
    rc = L.fcref_mass_assign(_dp(posw), posw.shape[0],
                             _ip(np.array(shape, dtype=np.intc)),
                             _dp(np.ascontiguousarray(posmin, dtype=np.float64)),
                             float(cell), int(scheme), int(bool(periodic)),
                             int(buffer_size), _dp(grid), _dp(st), 1)
    _check(L, rc, "mass assignment")
    return grid, st


def correlate(survey, grid, cell, posmin, window, rmax, dr, kmax, dk, maxell,
              grid2=None, build="parity"):
    """Reference Correlator (survey) or PeriodicCorrelator; autocorrelate, or
    cross_correlate with grid2.  Returns the result dict (rbins, rcounts,
    rhist, kbins, kcounts, khist, zerolag) plus the reference's own phase
    timers under "timers" (setup, fft_plan, fft, extract, multiply, ylm,
    histogram, total; correlator.h:97-105)."""
    L = lib(build)
    nrows = maxell // 2 + 1
    nr = int(math.floor(rmax / dr))
    nk = int(math.floor(kmax / dk))
    out = {
        "rbins": np.zeros(nr), "rcounts": np.zeros((nrows, nr), dtype=np.intc),
        "rhist": np.zeros((nrows, nr)), "kbins": np.zeros(nk),
        "kcounts": np.zeros((nrows, nk), dtype=np.intc),
        "khist": np.zeros((nrows, nk)), "timers": np.zeros(8),
    }
    zl = ctypes.c_double()
    g1 = np.ascontiguousarray(grid, dtype=np.float64)
    g2 = None if grid2 is None else np.ascontiguousarray(grid2, dtype=np.float64)
    pm = np.ascontiguousarray(posmin if posmin is not None else [0.0, 0.0, 0.0],
                              dtype=np.float64)
    rc = L.fcref_correlate(
        int(bool(survey)), _dp(g1), None if g2 is None else _dp(g2),
        _ip(np.array(g1.shape, dtype=np.intc)), float(cell), _dp(pm), int(window),
        float(rmax), float(dr), float(kmax), float(dk), int(maxell),
        _dp(out["rbins"]), _ip(out["rcounts"]), _dp(out["rhist"]),
        _dp(out["kbins"]), _ip(out["kcounts"]), _dp(out["khist"]),
        ctypes.byref(zl), 1, _dp(out["timers"]))
    _check(L, rc, "correlation")
    out["zerolag"] = zl.value
    return out


def survey_job(D, R, shape, posmin, cell, window, rmax, dr, kmax, dk, maxell,
               scheme=1, build="omp"):
    """One survey xi_ell + P_ell job through the reference classes.

    D is the data catalog and R the randoms with weights already scaled by
    -alpha.  The flow is the one the GPU job runs: D and R are assigned
    into two grids by the reference MassAssignor (CLI buffer 1e6), the NN
    grid is D + R (numpy, as the reference's Python API adds grids), and the
    reference Correlator autocorrelates NN and RR.  Returns (nn, rr, phase
    seconds).
    """
    import time
    t0 = time.perf_counter()
    gD, stD = mass_assign(D, shape, posmin, cell, scheme, False, build=build)
    gR, stR = mass_assign(R, shape, posmin, cell, scheme, False, build=build)
    t1 = time.perf_counter()
    np.add(gD, gR, out=gD)
    t2 = time.perf_counter()
    nn = correlate(True, gD, cell, posmin, window, rmax, dr, kmax, dk, maxell,
                   build=build)
    rr = correlate(True, gR, cell, posmin, window, rmax, dr, kmax, dk, maxell,
                   build=build)
    t3 = time.perf_counter()
    nn["ma_stats"] = stD
    rr["ma_stats"] = stR
    phases = {"mass_assign_s": t1 - t0, "grid_add_s": t2 - t1,
              "correlate_s": t3 - t2, "total_s": t3 - t0}
    return nn, rr, phases
