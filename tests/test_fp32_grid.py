"""FP32 grids (a library extension: the reference's grids are FP64).

An FP32 grid stores FP32 cells.  Mass assignment sums each update in FP64
and rounds once, so a cell that receives k updates differs from the FP64
oracle by at most k half-ulps of its running value.  One flush updates a
cell from at most 12 scatter units (3 x 2 x 2 neighbouring units' footprints
reach it; 8 for the 8-wide wavelet tiles), so the tests allow 1e-6 of the
grid's largest cell (12 x 2^-24 = 7.2e-7, with room for running values
above the final ones).  The grid arithmetic works in FP64 per cell and
rounds once.  Correlations of an
FP32 grid by the FP32-mixed correlators meet the mixed form's target,
max |gpu - oracle| <= 1e-4 rms(row 0) against the oracle's FP64 tables of
the FP64 field, and the FP64 correlators read an FP32 grid through a
widening copy.
"""
import ctypes

import numpy as np
import pytest

from conftest import clustered_catalog, uniform_catalog
from oracle import fc_oracle as O

import fftcorr_b200 as fb
from fftcorr_b200 import _lib
from fftcorr_b200.correlate import NO_CORRECTION, TSC_ALIASED_CORRECTION

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-6
FP32_TOL = 1e-4


def _values(grid):
    out = np.empty(grid.shape)
    _lib.call("fc_grid_download", grid.handle, _lib.dptr(out))
    return out


def _close_rms0(res, ref, label):
    for key in ("rhist", "khist"):
        rms0 = np.sqrt(np.mean(ref[key][0] ** 2))
        err = np.max(np.abs(res[key] - ref[key]))
        assert err <= FP32_TOL * rms0, f"{label} {key}: {err} vs rms {rms0}"
    np.testing.assert_array_equal(res["rcounts"], ref["rcounts"])
    np.testing.assert_array_equal(res["kcounts"], ref["kcounts"])


def test_precision_keyword_and_errors():
    g = fb.ConfigSpaceGrid.from_geometry((8, 8, 8), np.zeros(3), 1.0, precision="fp32")
    assert g.precision == "fp32"
    p = ctypes.c_int()
    _lib.call("fc_grid_precision", g.handle, ctypes.byref(p))
    assert p.value == _lib.FC_FP32_MIXED
    with pytest.raises(ValueError):
        fb.ConfigSpaceGrid.from_geometry((8, 8, 8), np.zeros(3), 1.0, precision="fp16")
    # The FP64-only pointer query refuses an FP32 grid; the typed one works.
    dp = ctypes.c_void_p()
    with pytest.raises(ValueError):
        _lib.call("fc_grid_device_ptr", g.handle, ctypes.byref(dp))
    assert g.device_ptr()


@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
@pytest.mark.parametrize("periodic", [False, True])
def test_mass_assign_into_fp32_grid(scheme, periodic):
    shape, cell = (24, 20, 28), 10.0
    posmin = np.array([-5.0, 3.0, 100.0])
    box = np.array(shape) * cell
    posw = clustered_catalog(30000, posmin, posmin + box, 7 + scheme, ncenters=20,
                             sigma=2 * cell)
    ref, st = O.mass_assign(posw, shape, posmin, cell, scheme, periodic)
    g = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision="fp32")
    ma = fb.MassAssignor(g, scheme, periodic, 0)
    ma.add_particles(posw)
    assert ma.num_added == st[0] and ma.num_skipped == st[1]
    got = _values(g)
    assert np.max(np.abs(got - ref)) <= GRID_TOL * np.max(np.abs(ref))
    # Stored values are FP32 numbers.
    assert np.array_equal(got, got.astype(np.float32).astype(np.float64))
    # Deterministic: the same bits on a second run.
    g.clear()
    ma.clear()
    ma.add_particles(posw)
    assert np.array_equal(_values(g), got)


def test_fp32_grid_arithmetic():
    shape = (16, 12, 10)
    rng = np.random.default_rng(3)
    a = rng.standard_normal(shape)
    b = rng.standard_normal(shape)
    ga = fb.ConfigSpaceGrid.from_geometry(shape, np.zeros(3), 1.0, precision="fp32")
    gb = fb.ConfigSpaceGrid.from_geometry(shape, np.zeros(3), 1.0, precision="fp32")
    g64 = fb.ConfigSpaceGrid.from_geometry(shape, np.zeros(3), 1.0)
    _lib.call("fc_grid_upload", ga.handle, _lib.dptr(a))
    _lib.call("fc_grid_upload", gb.handle, _lib.dptr(b))
    _lib.call("fc_grid_upload", g64.handle, _lib.dptr(b))
    a32 = a.astype(np.float32).astype(np.float64)
    b32 = b.astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(_values(ga), a32)
    s, q = ga.sum_sumsq()
    assert abs(s - a32.sum()) <= 1e-12 * np.abs(a32).sum()
    assert abs(q - (a32 ** 2).sum()) <= 1e-12 * (a32 ** 2).sum()
    # FP64 per cell, one rounding to FP32.
    ga.add_grid(gb, -0.5)
    want = (a32 - 0.5 * b32).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(_values(ga), want)
    ga.add_grid(g64, 2.0)  # FP64 x into an FP32 y
    want = (want + 2.0 * b).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(_values(ga), want)
    g64.add_grid(gb, 1.0)  # FP32 x into an FP64 y
    np.testing.assert_array_equal(_values(g64), b + b32)
    ga *= 3.0
    want = (want * 3.0).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(_values(ga), want)
    ga -= 0.25
    want = (want - 0.25).astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(_values(ga), want)


def _survey_catalogs(shape, cell, posmin, seed):
    box = np.array(shape) * cell
    lo = posmin + 0.15 * box
    hi = posmin + 0.85 * box
    D = clustered_catalog(20000, lo, hi, seed, ncenters=30, sigma=2 * cell)
    R = uniform_catalog(60000, lo, hi, seed + 1, weights="random")
    R[:, 3] *= -D[:, 3].sum() / R[:, 3].sum()
    return D, R


@pytest.mark.parametrize("fft", ["fused", "cufft"])
def test_survey_job_on_fp32_grids(fft, monkeypatch):
    """The benchmark's flow on FP32 grids: D and -alpha R assigned into two
    grids, NN = D + R' formed on the device, both correlated in FP32-mixed
    and FP64 against the oracle's FP64 tables."""
    monkeypatch.setenv("FFTCORR_B200_FFT", fft)
    shape, cell = (48, 48, 48), 12.0
    posmin = np.array([-288.0, -288.0, 30.0])
    D, R = _survey_catalogs(shape, cell, posmin, 71)
    nn_ref, _ = O.mass_assign(np.concatenate([D, R]), shape, posmin, cell, 1, False)
    rr_ref, _ = O.mass_assign(R, shape, posmin, cell, 1, False)
    args = (cell, posmin, TSC_ALIASED_CORRECTION, 96.0, 8.0, 0.15, 0.02, 4)
    refs = [O.survey_correlate(g, *args) for g in (nn_ref, rr_ref)]
    gA = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision="fp32")
    gB = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision="fp32")
    fb.MassAssignor(gA, 1, False, 0).add_particles(D)
    fb.MassAssignor(gB, 1, False, 0).add_particles(R)
    gA.add_grid(gB)
    # D and R' each within GRID_TOL of their largest cells, plus the add's
    # rounding.
    scale = max(np.max(np.abs(nn_ref - rr_ref)), np.max(np.abs(rr_ref)))
    assert np.max(np.abs(_values(gA) - nn_ref)) <= 3 * GRID_TOL * scale
    for precision in ("fp32", "fp64"):
        c = fb.Correlator(shape, *args, precision=precision)
        for g, ref in zip((gA, gB), refs):
            c.autocorrelate(g)
            _close_rms0(c.results(), ref, f"{fft} {precision}")


def test_periodic_on_fp32_grid():
    shape, cell = (40, 40, 40), 10.0
    box = np.array(shape) * cell
    posw = clustered_catalog(60000, [0, 0, 0], box, 72, ncenters=40, sigma=2 * cell)
    ref_grid, st = O.mass_assign(posw, shape, [0, 0, 0], cell, 3, True)
    mean = st[2] / ref_grid.size
    ref_grid = (ref_grid - mean) / mean
    pargs = (cell, NO_CORRECTION, 96.0, 8.0, 0.15, 0.02, 2)
    ref = O.periodic_correlate(ref_grid, *pargs)
    g = fb.ConfigSpaceGrid.from_geometry(shape, np.zeros(3), cell, precision="fp32")
    ma = fb.MassAssignor(g, 3, True, 0)
    ma.add_particles(posw)
    g -= mean
    g *= 1.0 / mean
    for precision in ("fp32", "fp64"):
        c = fb.PeriodicCorrelator(shape, *pargs, precision=precision)
        c.autocorrelate(g)
        _close_rms0(c.results(), ref, f"periodic {precision}")
