"""GPU parity tests: the CUDA path (through the C ABI) against the oracle.

The oracle (oracle/fc_oracle.py, pinned to the reference's golden outputs in
tests/test_oracle.py) and the compiled reference itself (oracle/_ref) are the
checkers.  Tolerances:
  * histogram counts, bin centres, num_added, num_skipped: exact;
  * FP64 grids: max |gpu - oracle| <= 1e-12 * max |oracle| (summation order);
  * FP64 correlator histograms: per multipole row,
    max |gpu - oracle| <= 1e-9 * max |oracle row| (cuFFT vs pocketfft);
  * FP32-mixed histograms: per row, max |gpu - oracle| <= 1e-4 * rms(row 0),
    the precision target of the mixed form.
"""
import numpy as np
import pytest

from conftest import clustered_catalog, uniform_catalog
from oracle import fc_oracle as O

import fftcorr_b200 as fb
from fftcorr_b200 import _lib
from fftcorr_b200.correlate import (NO_CORRECTION, TSC_ALIASED_CORRECTION,
                                    TSC_CORRECTION)

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-9
FP32_TOL = 1e-4


def _grid(shape, posmin, cell):
    return fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell)


def _device_grid_values(grid):
    out = np.empty(grid.shape)
    _lib.call("fc_grid_download", grid.handle, _lib.dptr(out))
    return out


def _assign_gpu(posw, shape, posmin, cell, scheme, periodic, buffer_size=0):
    g = _grid(shape, posmin, cell)
    ma = fb.MassAssignor(g, scheme, periodic, buffer_size)
    ma.add_particles(np.ascontiguousarray(posw))
    return g, ma


def _assert_rows_close(gpu, ref, rtol, label):
    gpu = np.atleast_2d(gpu)
    ref = np.atleast_2d(ref)
    assert gpu.shape == ref.shape, label
    for i in range(ref.shape[0]):
        scale = np.max(np.abs(ref[i])) if ref[i].size else 0.0
        err = np.max(np.abs(gpu[i] - ref[i])) if ref[i].size else 0.0
        assert err <= rtol * scale + 1e-300, f"{label} row {i}: {err} vs {scale}"


def _compare_results(res, ref, rtol, label, fp32=False):
    np.testing.assert_array_equal(res["rbins"], ref["rbins"])
    np.testing.assert_array_equal(res["kbins"], ref["kbins"])
    np.testing.assert_array_equal(res["rcounts"], ref["rcounts"])
    np.testing.assert_array_equal(res["kcounts"], ref["kcounts"])
    if fp32:
        for key in ("rhist", "khist"):
            rms0 = np.sqrt(np.mean(ref[key][0] ** 2))
            err = np.max(np.abs(res[key] - ref[key]))
            assert err <= FP32_TOL * rms0, f"{label} {key}: {err} vs rms {rms0}"
    else:
        _assert_rows_close(res["rhist"], ref["rhist"], rtol, label + " rhist")
        _assert_rows_close(res["khist"], ref["khist"], rtol, label + " khist")
        assert abs(res["zerolag"] - ref["zerolag"]) <= rtol * abs(ref["zerolag"]) + 1e-300


# --------------------------------------------------------------- gridding

@pytest.mark.parametrize("scheme", [0, 1, 2, 3])
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 20, 18), (9, 8, 26)])
def test_mass_assign_matches_oracle(scheme, periodic, shape):
    cell = 10.0
    posmin = np.array([-5.0, 3.0, 100.0])
    box = np.array(shape) * cell
    # Some particles fall outside the box: skipped, or wrapped when periodic.
    posw = uniform_catalog(20000, posmin - 0.1 * box, posmin + 1.1 * box, 7,
                           weights="random")
    g, ma = _assign_gpu(posw, shape, posmin, cell, scheme, periodic)
    ref, st = O.mass_assign(posw, shape, posmin, cell, scheme, periodic)
    got = _device_grid_values(g)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= 1e-12 * scale
    assert ma.num_added == int(st[0])
    assert ma.num_skipped == int(st[1])
    assert ma.totw == pytest.approx(st[2], rel=1e-12)
    assert ma.totwsq == pytest.approx(st[3], rel=1e-12)


@pytest.mark.parametrize("scheme", [1, 2])
@pytest.mark.parametrize("n", [1, 8191, 8192, 8193, 24581])
def test_particle_sort_tiles_and_skipped_particles(scheme, n):
    """The particle sort's edge cases: counts around its 8192-key tiles,
    about two thirds of the particles outside the grid (their keys sort last in
    a digit of their own), and a grid of 576 tiles, so that the unit bits
    (TSC) and the full cell keys (D12) both take two passes."""
    shape, cell = (64, 64, 72), 4.0
    posmin = np.array([1.0, -2.0, 50.0])
    box = np.array(shape) * cell
    posw = uniform_catalog(n, posmin - 0.2 * box, posmin + 1.2 * box, 100 + n,
                           weights="random")
    g, ma = _assign_gpu(posw, shape, posmin, cell, scheme, False)
    ref, st = O.mass_assign(posw, shape, posmin, cell, scheme, False)
    got = _device_grid_values(g)
    assert np.max(np.abs(got - ref)) <= 1e-12 * max(np.max(np.abs(ref)), 1e-300)
    assert ma.num_added == int(st[0])
    assert ma.num_skipped == int(st[1])


@pytest.mark.parametrize("scheme", [0, 1, 3])
def test_cell_sums_follow_input_order(scheme):
    """Bit-level check that each cell sums its particles in input order
    (stable sort, ordered ranking in the scatter).  Three particles at one
    cell centre carry weights whose FP64 sum depends on the order: with
    [1, 2^-60, -1] only orders that leave 2^-60 last give a nonzero cell,
    and with [1, -1, 2^-60] every order but those ending in 2^-60 gives 0
    where input order gives exactly c 2^-60 (c the stencil's product, a
    product of 1/8, 1/2 and 3/4, so every term is exact).  The three are
    spread over different 8192-key sort tiles among 30000 other particles
    whose footprints do not reach them."""
    t = 2.0 ** -60
    shape, cell = (32, 32, 32), 1.0
    rng = np.random.default_rng(23)
    posw = np.empty((30000, 4))
    posw[:, 0] = rng.uniform(14.0, 30.0, 30000)
    posw[:, 1:3] = rng.uniform(0.0, 32.0, (30000, 2))
    posw[:, 3] = rng.uniform(0.5, 1.5, 30000)
    a_idx, b_idx = (5, 15000, 29000), (7, 15002, 29002)
    for i, w in zip(a_idx, (1.0, t, -1.0)):
        posw[i] = (5.5, 5.5, 5.5, w)
    for i, w in zip(b_idx, (1.0, -1.0, t)):
        posw[i] = (5.5, 5.5, 20.5, w)
    g, ma = _assign_gpu(posw, shape, np.zeros(3), cell, scheme, False)
    got = _device_grid_values(g)
    # Stencil weights at a cell centre and their offsets from the home cell.
    wts, off = {0: ([1.0], [0]), 1: ([0.125, 0.75, 0.125], [-1, 0, 1]),
                3: ([0.5, 0.5], [0, 1])}[scheme]
    want = np.zeros(shape)
    for ax, wx in zip(off, wts):
        for ay, wy in zip(off, wts):
            for az, wz in zip(off, wts):
                want[5 + ax, 5 + ay, 20 + az] = wx * wy * wz * t
    np.testing.assert_array_equal(got[:12], want[:12])
    assert ma.num_added == 30000


@pytest.mark.parametrize("scheme", [1, 2])
def test_every_particle_outside_the_grid(scheme):
    shape, cell = (16, 16, 16), 10.0
    posmin = np.zeros(3)
    posw = uniform_catalog(10000, [200.0, 0.0, 0.0], [300.0, 160.0, 160.0], 5,
                           weights="random")
    g, ma = _assign_gpu(posw, shape, posmin, cell, scheme, False)
    assert ma.num_added == 0 and ma.num_skipped == 10000
    assert not np.any(_device_grid_values(g))


@pytest.mark.parametrize("scheme", [1, 2])
def test_tiny_periodic_grid_wraps_onto_itself(scheme):
    # Stencils wider than the grid (test_mass_assignor.py uses a 2^3 grid).
    shape = (2, 3, 2)
    posmin = np.array([2.0, -5.0, 77.0])
    posw = uniform_catalog(500, posmin, posmin + np.array(shape) * 25.0, 3,
                           weights="random")
    g, _ = _assign_gpu(posw, shape, posmin, 25.0, scheme, True)
    ref, _ = O.mass_assign(posw, shape, posmin, 25.0, scheme, True)
    got = _device_grid_values(g)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_mass_assign_matches_compiled_reference():
    """Against the reference's own MassAssignor (oracle/_ref/libfcref.so)."""
    import ctypes
    import os
    path = os.path.join(os.path.dirname(O.__file__), "_ref", "libfcref.so")
    L = ctypes.CDLL(path)
    shape = (24, 16, 20)
    posmin = np.array([0.0, 0.0, 0.0])
    posw = clustered_catalog(50000, [0, 0, 0], np.array(shape) * 5.0, 11)
    for scheme in (0, 1, 2):
        ref = np.zeros(shape)
        st = np.zeros(6)
        shp = np.array(shape, dtype=np.intc)
        rc = L.fcref_mass_assign(
            O._dp(posw), ctypes.c_long(posw.shape[0]), O._ip(shp), O._dp(posmin),
            ctypes.c_double(5.0), scheme, 1, ctypes.c_long(0), O._dp(ref),
            O._dp(st), 1)
        assert rc == 0
        g, ma = _assign_gpu(posw, shape, posmin, 5.0, scheme, True)
        got = _device_grid_values(g)
        assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
        assert ma.num_added == int(st[0])


@pytest.mark.parametrize("cell", [3.450520833333333, 0.1, 7.0 / 3.0])
def test_cell_faces_match_division(cell):
    """Particles within a few ulps of cell faces land in the cells IEEE
    division puts them in (the kernels divide through the reciprocal)."""
    rng = np.random.default_rng(17)
    shape = (16, 16, 16)
    posmin = np.array([-123.456, 0.0, 987.654321])
    n = 60000
    pos = posmin + rng.integers(0, 17, size=(n, 3)) * cell
    pos = pos + rng.integers(-3, 4, size=(n, 3)) * np.spacing(pos)
    posw = np.concatenate([pos, np.ones((n, 1))], axis=1)
    for periodic in (False, True):
        g, ma = _assign_gpu(posw, shape, posmin, cell, 0, periodic)
        ref, st = O.mass_assign(posw, shape, posmin, cell, 0, periodic)
        assert np.array_equal(_device_grid_values(g), ref)
        assert ma.num_added == int(st[0])
        assert ma.num_skipped == int(st[1])


def test_mass_assign_is_deterministic():
    shape = (64, 64, 64)
    posw = clustered_catalog(400000, [0, 0, 0], [640, 640, 640], 5, ncenters=200)
    a, _ = _assign_gpu(posw, shape, [0, 0, 0], 10.0, 1, True)
    b, _ = _assign_gpu(posw, shape, [0, 0, 0], 10.0, 1, True)
    assert np.array_equal(_device_grid_values(a), _device_grid_values(b))


def test_buffered_equals_direct_and_overloads_agree():
    shape = (20, 20, 20)
    posw = uniform_catalog(30000, [0, 0, 0], [200, 200, 200], 9, weights="random")
    direct, _ = _assign_gpu(posw, shape, [0, 0, 0], 10.0, 1, False)
    g = _grid(shape, [0, 0, 0], 10.0)
    ma = fb.MassAssignor(g, 1, False, buffer_size=7000)
    for chunk in np.array_split(posw, 5):
        ma.add_particles_to_buffer(np.ascontiguousarray(chunk))
    ma.flush()
    ref = _device_grid_values(direct)
    assert np.max(np.abs(_device_grid_values(g) - ref)) <= 1e-12 * np.max(np.abs(ref))
    g2 = _grid(shape, [0, 0, 0], 10.0)
    ma2 = fb.MassAssignor(g2, 1, False)
    ma2.add_particles(np.ascontiguousarray(posw[:, :3]),
                      np.ascontiguousarray(posw[:, 3]))
    assert np.max(np.abs(_device_grid_values(g2) - ref)) <= 1e-12 * np.max(np.abs(ref))
    g3 = _grid(shape, [0, 0, 0], 10.0)
    ma3 = fb.MassAssignor(g3, 1, False)
    ma3.add_particles(np.ascontiguousarray(posw[:, :3]), 2.5)
    unit = posw.copy()
    unit[:, 3] = 2.5
    ref3, _ = O.mass_assign(unit, shape, [0, 0, 0], 10.0, 1, False)
    assert np.max(np.abs(_device_grid_values(g3) - ref3)) <= 1e-12 * np.max(np.abs(ref3))
    assert ma3.totw == pytest.approx(2.5 * ma3.num_added)


def test_input_errors_match_reference():
    g = _grid((2, 2, 2), [2, -5, 77], 25.0)
    ma = fb.MassAssignor(g, distribution_scheme=1, buffer_size=100)
    with pytest.raises(RuntimeError):
        ma.add_particles(np.zeros((2, 3, 4)), 5.0)
    with pytest.raises(RuntimeError):
        ma.add_particles(np.zeros((10, 3), dtype=np.float32), 5.0)
    with pytest.raises(RuntimeError):
        ma.add_particles(np.zeros((10, 4))[:, 0:3], 5.0)
    ro = np.zeros((10, 4))
    ro.setflags(write=False)
    with pytest.raises(RuntimeError):
        ma.add_particles(ro)
    with pytest.raises(ValueError):
        ma.add_particles(np.zeros((10, 4)), 1.0)
    with pytest.raises(ValueError):
        ma.add_particles(np.zeros((10, 5)))
    with pytest.raises(ValueError):
        ma.add_particles(np.zeros((10, 3)), np.ones(9))


def test_grid_host_mirror_semantics():
    g = fb.ConfigSpaceGrid([2, 2, 2], [2, -5, 77], [50, 45, 120], cell_size=25)
    d = g.data
    d += 7
    assert np.sum(g) == pytest.approx(56.0)
    ma = fb.MassAssignor(g, 0)
    ma.add_particles(np.array([[10.0, 10.0, 100.0, 12.0]]))
    assert g.data[0, 0, 0] == pytest.approx(19.0)
    assert d is g.data
    g.clear()
    assert np.sum(g) == 0.0
    assert g.to_grid_coords([2, -4, 79]) == pytest.approx([0.0, 0.04, 0.08])
    with pytest.raises(ValueError):
        g.to_grid_coords([1, 0, 77])
    assert g.to_grid_coords([1, 0, 77], periodic_wrap=True)[0] == pytest.approx(
        2 - 1 / 25.0)


# ------------------------------------------------------------ correlators

@pytest.fixture(params=["fused", "cufft"])
def fft_path(request, monkeypatch):
    """Runs a survey test through the hand-written fused FFT passes and
    through the cuFFT path (the correlator reads FFTCORR_B200_FFT when it is
    created)."""
    monkeypatch.setenv("FFTCORR_B200_FFT", request.param)
    return request.param


def _periodic_field(shape, cell, seed, scheme=3):
    box = np.array(shape) * cell
    posw = clustered_catalog(60000, [0, 0, 0], box, seed, ncenters=40,
                             sigma=2 * cell)
    grid, st = O.mass_assign(posw, shape, [0, 0, 0], cell, scheme, True)
    mean = st[2] / grid.size
    grid += -mean
    grid *= 1.0 / mean
    return grid


def _survey_field(shape, cell, posmin, seed):
    box = np.array(shape) * cell
    lo = np.asarray(posmin) + 0.15 * box
    hi = np.asarray(posmin) + 0.85 * box
    D = clustered_catalog(20000, lo, hi, seed, ncenters=30, sigma=2 * cell)
    R = uniform_catalog(60000, lo, hi, seed + 1, weights="random")
    R[:, 3] *= -D[:, 3].sum() / R[:, 3].sum()
    nn, _ = O.mass_assign(np.concatenate([D, R]), shape, posmin, cell, 1, False)
    rr, _ = O.mass_assign(R, shape, posmin, cell, 1, False)
    return nn, rr


@pytest.mark.parametrize("maxell", [0, 2, 4])
@pytest.mark.parametrize("window", [NO_CORRECTION, TSC_CORRECTION,
                                    TSC_ALIASED_CORRECTION])
def test_periodic_correlator_fp64(maxell, window):
    shape, cell = (32, 40, 36), 10.0
    grid = _periodic_field(shape, cell, 21)
    args = (cell, window, 60.0, 7.0, 0.25, 0.02, maxell)
    ref = O.periodic_correlate(grid, *args)
    c = fb.PeriodicCorrelator(shape, *args)
    c.autocorrelate(grid)
    _compare_results(c.results(), ref, FP64_RTOL, "periodic")


@pytest.mark.parametrize("maxell", [0, 2, 4])
def test_survey_correlator_fp64(maxell, fft_path):
    shape, cell = (32, 36, 40), 12.0
    posmin = np.array([-100.0, 250.0, -300.0])
    nn, _ = _survey_field(shape, cell, posmin, 31)
    args = (cell, posmin, TSC_ALIASED_CORRECTION, 70.0, 10.0, 0.12, 0.02, maxell)
    ref = O.survey_correlate(nn, *args)
    c = fb.Correlator(shape, *args)
    ps, xi = c.autocorrelate(nn)
    _compare_results(c.results(), ref, FP64_RTOL, "survey")
    assert list(xi.colnames) == ["r", "xi", "histogram", "count"]
    assert list(ps.colnames) == ["k", "ps", "histogram", "count"]


def test_correlators_read_device_grids(fft_path):
    shape, cell = (32, 32, 32), 15.0
    posmin = np.array([-240.0, -240.0, 10.0])
    nn, _ = _survey_field(shape, cell, posmin, 41)
    g = _grid(shape, posmin, cell)
    _lib.call("fc_grid_upload", g.handle, _lib.dptr(np.ascontiguousarray(nn)))
    args = (cell, posmin, NO_CORRECTION, 90.0, 10.0, 0.1, 0.02, 2)
    c = fb.Correlator(shape, *args)
    c.autocorrelate(g)
    ref = O.survey_correlate(nn, *args)
    _compare_results(c.results(), ref, FP64_RTOL, "survey-device")


def test_cross_correlations(fft_path):
    shape, cell = (24, 24, 32), 10.0
    a = _periodic_field(shape, cell, 51)
    b = _periodic_field(shape, cell, 52, scheme=1)
    args = (cell, NO_CORRECTION, 50.0, 5.0, 0.3, 0.05, 2)
    ref = O.periodic_correlate(a, *args, grid2=b)
    c = fb.PeriodicCorrelator(shape, *args)
    c.cross_correlate(a, b)
    _compare_results(c.results(), ref, FP64_RTOL, "periodic-cross")
    # set_grid2_fft with the FFT of b gives the same answer.
    c2 = fb.PeriodicCorrelator(shape, *args)
    c2.set_grid2_fft(np.fft.rfftn(b))
    c2.cross_correlate(a)
    _compare_results(c2.results(), ref, FP64_RTOL, "periodic-cross-fft")
    posmin = np.array([0.0, -120.0, 40.0])
    sargs = (cell, posmin, NO_CORRECTION, 50.0, 5.0, 0.3, 0.05, 4)
    sref = O.survey_correlate(a, *sargs, grid2=b)
    s = fb.Correlator(shape, *sargs)
    s.set_grid2(b)
    s.cross_correlate(a)
    _compare_results(s.results(), sref, FP64_RTOL, "survey-cross")
    # The survey correlator takes a host FFT of grid2 too (rows padded on
    # the device in the fused path).
    for precision in ("fp64", "fp32"):
        s2 = fb.Correlator(shape, *sargs, precision=precision)
        s2.set_grid2_fft(np.fft.rfftn(b))
        s2.cross_correlate(a)
        _compare_results(s2.results(), sref, FP64_RTOL, "survey-cross-fft",
                         fp32=precision == "fp32")


@pytest.mark.parametrize("shape", [(20, 28, 30), (24, 18, 50), (16, 16, 33),
                                   (64, 128, 256), (128, 96, 128)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_survey_radix_3_5_7_and_odd_sizes(shape, precision):
    """Lengths with factors 3, 5, 7 run through the fused passes; an odd N2
    uses the cuFFT path.  Both must match the oracle."""
    cell = 10.0
    posmin = np.array([-100.0, 50.0, -130.0])
    nn, _ = _survey_field(shape, cell, posmin, 81)
    args = (cell, posmin, TSC_CORRECTION, 45.0, 6.0, 0.2, 0.03, 4)
    ref = O.survey_correlate(nn, *args)
    c = fb.Correlator(shape, *args, precision=precision)
    c.autocorrelate(nn)
    _compare_results(c.results(), ref, FP64_RTOL, "radix", fp32=precision == "fp32")


def test_cross_correlate_without_grid2_fails():
    c = fb.PeriodicCorrelator((16, 16, 16), 10.0, 0, 30.0, 5.0, 0.2, 0.05, 0)
    with pytest.raises(_lib.FcError):
        c.cross_correlate(np.zeros((16, 16, 16)))


@pytest.mark.parametrize("kmax", [0.2, 0.35])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_survey_last_column_group(kmax, precision):
    """The column passes hand the kz = N2/2 column (alone in its 16-column
    group) to CTAs that take it for 16 planes each, unless the k-subgrid
    reaches it: kmax 0.2 keeps it outside, 0.35 (above the Nyquist 0.314)
    spans every kz.  Both must match the oracle."""
    shape, cell = (64, 64, 64), 10.0
    posmin = np.array([-320.0, -320.0, 40.0])
    nn, _ = _survey_field(shape, cell, posmin, 91)
    args = (cell, posmin, TSC_ALIASED_CORRECTION, 60.0, 6.0, kmax, 0.03, 4)
    ref = O.survey_correlate(nn, *args)
    c = fb.Correlator(shape, *args, precision=precision)
    c.autocorrelate(nn)
    _compare_results(c.results(), ref, FP64_RTOL, "last group",
                     fp32=precision == "fp32")


def test_fp32_mixed_within_tolerance(fft_path):
    shape, cell = (48, 48, 48), 12.0
    posmin = np.array([-288.0, -288.0, 30.0])
    nn, rr = _survey_field(shape, cell, posmin, 61)
    args = (cell, posmin, TSC_ALIASED_CORRECTION, 96.0, 8.0, 0.15, 0.02, 4)
    for grid in (nn, rr):
        ref = O.survey_correlate(grid, *args)
        c = fb.Correlator(shape, *args, precision="fp32")
        c.autocorrelate(grid)
        _compare_results(c.results(), ref, 0, "survey-fp32", fp32=True)
    pgrid = _periodic_field(shape, cell, 62)
    pargs = (cell, NO_CORRECTION, 96.0, 8.0, 0.15, 0.02, 4)
    ref = O.periodic_correlate(pgrid, *pargs)
    c = fb.PeriodicCorrelator(shape, *pargs, precision="fp32")
    c.autocorrelate(pgrid)
    _compare_results(c.results(), ref, 0, "periodic-fp32", fp32=True)


def test_correlation_is_deterministic(fft_path):
    shape, cell = (32, 32, 32), 10.0
    posmin = np.array([-160.0, -160.0, 20.0])
    nn, _ = _survey_field(shape, cell, posmin, 71)
    args = (cell, posmin, NO_CORRECTION, 60.0, 6.0, 0.2, 0.02, 4)
    c = fb.Correlator(shape, *args)
    c.autocorrelate(nn)
    a = c.results()
    c.autocorrelate(nn)
    b = c.results()
    assert np.array_equal(a["rhist"], b["rhist"])
    assert np.array_equal(a["khist"], b["khist"])


# ----------------------------------------------------------- histograms

def test_histogram_list_matches_oracle():
    rng = np.random.default_rng(3)
    h = fb.HistogramList(2, -10, 10, 2)
    counts = h.counts
    x = np.array([[1, 7], [3, -5]], dtype=np.double)
    y = np.array([[11, 77], [33, -55]], dtype=np.double)
    h.accumulate(0, x, y)
    assert counts[0].tolist() == [0, 0, 1, 0, 0, 1, 1, 0, 1, 0]
    ref = O.Histogram(2, -10, 10, 2)
    ref.accumulate(0, x, y)
    xs = rng.uniform(-12, 12, 100000)
    ys = rng.normal(size=100000)
    h.accumulate(1, xs, ys)
    ref.accumulate(1, xs, ys)
    np.testing.assert_array_equal(h.counts, ref.counts)
    np.testing.assert_array_equal(h.bins, ref.bins)
    np.testing.assert_allclose(h.hist_values, ref.hist, rtol=1e-12, atol=1e-12)
    with pytest.raises(ValueError):
        h.hist_values[0][0] = 5
    h.reset()
    assert counts.sum() == 0


# --------------------------------------------- golden end-to-end on the GPU

def _gpu_cli(cats, header, ngrid=(256, 256, 256), sep=200.0, dsep=10.0,
             kmax=0.03, dk=0.01, maxell=2, scheme=2, periodic=False):
    posmin, cell = O.cli_box(header[0:3], header[3:6], sep, ngrid, periodic)
    g = _grid(ngrid, posmin, cell)
    ma = fb.MassAssignor(g, scheme, periodic, 1000000)
    for cat in cats:
        ma.add_particles_to_buffer(np.ascontiguousarray(cat))
    ma.flush()
    window = TSC_ALIASED_CORRECTION if scheme == 1 else NO_CORRECTION
    c = fb.Correlator(ngrid, cell, posmin, window, sep, dsep, kmax, dk, maxell)
    c.autocorrelate(g)
    return O.cli_table(c.results(), periodic)


@pytest.mark.parametrize("hemi", ["north", "south"])
def test_golden_tables_through_gpu(hemi, golden_catalogs, golden_tables, fft_path):
    header = golden_catalogs[f"{hemi}_header"]
    DD = golden_catalogs[f"{hemi}_DD"]
    RR = golden_catalogs[f"{hemi}_RR"]
    for name, cats in (("corrDD", [DD, RR]), ("corrRR", [RR])):
        tab = _gpu_cli(cats, header)
        gold = golden_tables[f"{hemi}_{name}"]
        np.testing.assert_array_equal(tab[:, 2], gold[:, 2])
        np.testing.assert_allclose(tab, gold, rtol=1e-7)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_term_shards_sum_to_the_full_correlation(precision, fft_path):
    """(ell, m) terms split over 3 ranks, run one after another on this GPU:
    each share matches the oracle's share of the same terms, and the shares
    sum to the unsharded correlation."""
    from fftcorr_b200.correlate.sharded import owned_terms
    shape, cell = (32, 32, 32), 12.0
    posmin = np.array([-100.0, 250.0, -300.0])
    nn, _ = _survey_field(shape, cell, posmin, 71)
    args = (cell, posmin, TSC_ALIASED_CORRECTION, 70.0, 10.0, 0.12, 0.02, 4)
    c = fb.Correlator(shape, *args, precision=precision)
    c.autocorrelate(nn)
    full = c.results()
    tot = {"rhist": 0.0, "khist": 0.0, "zerolag": 0.0}
    for rank in range(3):
        c.set_term_shard(rank, 3)
        c.autocorrelate(nn)
        part = c.results()
        np.testing.assert_array_equal(part["rcounts"], full["rcounts"])
        np.testing.assert_array_equal(part["kcounts"], full["kcounts"])
        if precision == "fp64":
            terms = {i for i, _, _ in owned_terms(4, rank, 3)}
            ref = O.survey_correlate(nn, *args, terms=terms)
            _compare_results(part, ref, FP64_RTOL, f"shard {rank}")
        for k in tot:
            tot[k] = tot[k] + part[k]
    for k in ("rhist", "khist"):
        scale = np.max(np.abs(full[k]))
        assert np.max(np.abs(tot[k] - full[k])) <= 1e-12 * scale
    assert abs(tot["zerolag"] - full["zerolag"]) <= 1e-12 * abs(full["zerolag"])
    c.set_term_shard(0, 1)
    c.autocorrelate(nn)
    assert np.array_equal(c.results()["rhist"], full["rhist"])


def test_term_shard_arguments():
    c = fb.Correlator((16, 16, 16), 10.0, np.array([-80.0, 5.0, 5.0]), 0, 30.0,
                      5.0, 0.2, 0.05, 2)
    with pytest.raises(ValueError):
        c.set_term_shard(2, 2)
    p = fb.PeriodicCorrelator((16, 16, 16), 10.0, 0, 30.0, 5.0, 0.2, 0.05, 2)
    with pytest.raises(_lib.FcError):
        p.set_term_shard(0, 2)
    p.set_term_shard(0, 1)
