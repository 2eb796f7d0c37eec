"""Pins the oracle before it is trusted (no GPU needed).

1. The oracle restatement (oracle/fc_oracle.py) reproduces the reference's
   golden P_ell / xi_ell tables (test_data/*/nonperiodic/*.out, committed as
   tests/golden/tables.npz) at the reference test's rtol 1e-7, counts exact.
2. The restatement agrees with the compiled reference (oracle/_ref, built
   from the reference sources with the FFTW shim): mass-assigned grids bit
   for bit, histograms bit for bit, correlator outputs to FFT rounding.
3. The compiled reference CLI reproduces a golden table file.
4. compute_xi reproduces the golden xi.txt (test_fftcorr_aniso.py:115-134).
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, clustered_catalog, uniform_catalog
from oracle import fc_oracle as O
from oracle import ref_lib

REF_DIR = os.path.join(ROOT, "oracle", "_ref")
HAVE_REF = os.path.exists(os.path.join(REF_DIR, "libfcref.so"))
needs_ref = pytest.mark.skipif(not HAVE_REF, reason="oracle/_ref not built")


def _fcref():
    return ctypes.CDLL(os.path.join(REF_DIR, "libfcref.so"))


def _ref_correlate(survey, grid, cell, posmin, window, rmax, dr, kmax, dk,
                   maxell, grid2=None):
    L = _fcref()
    nrows = maxell // 2 + 1
    nr = int(np.floor(rmax / dr))
    nk = int(np.floor(kmax / dk))
    out = {
        "rbins": np.zeros(nr), "rcounts": np.zeros((nrows, nr), dtype=np.intc),
        "rhist": np.zeros((nrows, nr)), "kbins": np.zeros(nk),
        "kcounts": np.zeros((nrows, nk), dtype=np.intc),
        "khist": np.zeros((nrows, nk)),
    }
    zl = ctypes.c_double()
    shp = np.array(grid.shape, dtype=np.intc)
    pm = np.ascontiguousarray(posmin, dtype=np.float64)
    g1 = np.ascontiguousarray(grid)
    g2 = None if grid2 is None else np.ascontiguousarray(grid2)
    d = ctypes.c_double
    rc = L.fcref_correlate(
        int(survey), O._dp(g1), None if g2 is None else O._dp(g2), O._ip(shp),
        d(cell), O._dp(pm), int(window), d(rmax), d(dr), d(kmax), d(dk),
        int(maxell), O._dp(out["rbins"]), O._ip(out["rcounts"]),
        O._dp(out["rhist"]), O._dp(out["kbins"]), O._ip(out["kcounts"]),
        O._dp(out["khist"]), ctypes.byref(zl), 1, None)
    assert rc == 0
    out["zerolag"] = zl.value
    return out


@pytest.mark.slow
@pytest.mark.parametrize("hemi", ["north", "south"])
def test_oracle_reproduces_golden_tables(hemi, golden_catalogs, golden_tables):
    header = golden_catalogs[f"{hemi}_header"]
    DD = golden_catalogs[f"{hemi}_DD"]
    RR = golden_catalogs[f"{hemi}_RR"]
    for name, cats in (("corrDD", [DD, RR]), ("corrRR", [RR])):
        res = O.cli_run(cats, (256, 256, 256), 200.0, 10.0, 0.03, 0.01, 2,
                        O.WAVELET, False, header)
        tab = O.cli_table(res, False)
        gold = golden_tables[f"{hemi}_{name}"]
        np.testing.assert_array_equal(tab[:, 2], gold[:, 2])
        np.testing.assert_allclose(tab, gold, rtol=1e-7)


@pytest.mark.parametrize("hemi", ["north", "south"])
def test_compute_xi_reproduces_golden(hemi, golden_tables):
    from fftcorr_b200.correlate.utils import compute_xi
    nn = golden_tables[f"{hemi}_corrDD"]
    rr = golden_tables[f"{hemi}_corrRR"]
    nn = nn[nn[:, 0] == 0]
    rr = rr[rr[:, 0] == 0]
    gold = golden_tables[f"{hemi}_xi"]
    xi = compute_xi(nn[:, 3:], rr[:, 3:])
    np.testing.assert_allclose(nn[:, 1], gold[:, 0])
    np.testing.assert_allclose(xi, gold[:, 1:], rtol=1e-5)


@needs_ref
@pytest.mark.parametrize("scheme", [0, 1, 2])
@pytest.mark.parametrize("periodic", [0, 1])
def test_oracle_grid_bit_identical_to_reference(scheme, periodic):
    L = _fcref()
    shape = (12, 10, 14)
    posmin = np.array([-3.0, 7.0, 20.0])
    cell = 4.0
    box = np.array(shape) * cell
    posw = uniform_catalog(5000, posmin - 0.1 * box, posmin + 1.1 * box, 1,
                           weights="random")
    ref = np.zeros(shape)
    st = np.zeros(6)
    rc = L.fcref_mass_assign(O._dp(posw), ctypes.c_long(len(posw)),
                             O._ip(np.array(shape, dtype=np.intc)), O._dp(posmin),
                             ctypes.c_double(cell), scheme, periodic,
                             ctypes.c_long(0), O._dp(ref), O._dp(st), 1)
    assert rc == 0
    got, gst = O.mass_assign(posw, shape, posmin, cell, scheme, periodic)
    assert np.array_equal(got, ref)
    np.testing.assert_array_equal(gst, st[:4])


@needs_ref
def test_oracle_histogram_bit_identical_to_reference():
    L = _fcref()
    rng = np.random.default_rng(2)
    x = rng.uniform(-3, 25, 20000)
    y = rng.normal(size=20000)
    bins = np.zeros(11)
    counts = np.zeros((2, 11), dtype=np.intc)
    hist = np.zeros((2, 11))
    ih = np.array([0, 1, 1], dtype=np.intc)
    rc = L.fcref_histogram(2, ctypes.c_double(0.0), ctypes.c_double(22.0),
                           ctypes.c_double(2.0), 3, O._ip(ih), O._dp(x), O._dp(y),
                           ctypes.c_long(x.size), O._dp(bins), O._ip(counts),
                           O._dp(hist))
    assert rc == 0
    h = O.Histogram(2, 0.0, 22.0, 2.0)
    for i in ih:
        h.accumulate(int(i), x, y)
    assert np.array_equal(h.bins, bins)
    assert np.array_equal(h.counts, counts)
    assert np.array_equal(h.hist, hist)


@needs_ref
@pytest.mark.parametrize("maxell", [0, 2, 4])
@pytest.mark.parametrize("window", [0, 1, 2])
def test_oracle_periodic_correlator_matches_reference(maxell, window):
    shape, cell = (16, 20, 18), 10.0
    posw = clustered_catalog(20000, [0, 0, 0], np.array(shape) * cell, 4)
    grid, st = O.mass_assign(posw, shape, [0, 0, 0], cell, 1, True)
    grid = grid / (st[2] / grid.size) - 1.0
    args = (cell, window, 50.0, 7.0, 0.25, 0.04, maxell)
    got = O.periodic_correlate(grid, *args)
    ref = _ref_correlate(0, grid, cell, [0, 0, 0], *((window,) + args[2:]))
    _assert_same(got, ref, 1e-10)


@needs_ref
@pytest.mark.parametrize("maxell", [0, 4])
def test_oracle_survey_correlator_matches_reference(maxell):
    shape, cell = (16, 18, 20), 10.0
    posmin = np.array([-60.0, 50.0, -90.0])
    posw = clustered_catalog(20000, posmin, posmin + np.array(shape) * cell, 8)
    posw[10000:, 3] *= -1.0
    grid, _ = O.mass_assign(posw, shape, posmin, cell, 1, False)
    args = (cell, posmin, 2, 60.0, 10.0, 0.2, 0.03, maxell)
    got = O.survey_correlate(grid, *args)
    ref = _ref_correlate(1, grid, *args)
    _assert_same(got, ref, 1e-10)
    # Cross-correlation against a second grid.
    grid2, _ = O.mass_assign(posw[::-1].copy(), shape, posmin, cell, 0, False)
    got = O.survey_correlate(grid, *args, grid2=grid2)
    ref = _ref_correlate(1, grid, *args, grid2=grid2)
    _assert_same(got, ref, 1e-10)


def _assert_same(got, ref, rtol):
    np.testing.assert_array_equal(got["rbins"], ref["rbins"])
    np.testing.assert_array_equal(got["kbins"], ref["kbins"])
    np.testing.assert_array_equal(got["rcounts"], ref["rcounts"])
    np.testing.assert_array_equal(got["kcounts"], ref["kcounts"])
    for key in ("rhist", "khist"):
        for i in range(ref[key].shape[0]):
            scale = np.max(np.abs(ref[key][i]))
            assert np.max(np.abs(got[key][i] - ref[key][i])) <= rtol * scale + 1e-300
    assert got["zerolag"] == pytest.approx(ref["zerolag"], rel=rtol)


@needs_ref
@pytest.mark.slow
def test_reference_cli_reproduces_golden(tmp_path, golden_catalogs, golden_tables):
    hemi = "south"
    for name in ("DD", "RR"):
        hdr = golden_catalogs[f"{hemi}_header"]
        with open(tmp_path / f"corr{name}.dat", "wb") as f:
            hdr.tofile(f)
            golden_catalogs[f"{hemi}_{name}"].tofile(f)
    exe = os.path.join(REF_DIR, "fftcorr")
    cmd = [exe, "-in", "corrDD.dat", "-out", "corrDD.dat.out", "-dr", "10.0",
           "-n", "256", "-ell", "2", "-r", "200.0", "-in2", "corrRR.dat",
           "-wisdom", str(tmp_path / "wisdom")]
    subprocess.run(cmd, cwd=tmp_path, check=True, capture_output=True)
    tab = np.loadtxt(tmp_path / "corrDD.dat.out")
    np.testing.assert_allclose(tab, golden_tables[f"{hemi}_corrDD"], rtol=1e-7)


@pytest.mark.skipif(not (ref_lib.available("parity") and ref_lib.available("pomp")),
                    reason="oracle/_ref not built")
@pytest.mark.parametrize("survey", [0, 1])
def test_openmp_parity_build_matches_serial_parity_build(survey):
    """The OpenMP parity build (the oracle for the large grids) gives the
    serial parity build's correlator outputs bit for bit: the per-slab FFT
    split runs the same 1-D transforms and every cell's arithmetic is
    unchanged, only spread over threads."""
    rng = np.random.default_rng(11)
    shape, cell = (40, 32, 48), 9.0
    grid = rng.standard_normal(shape)
    args = (cell, [-150.0, 40.0, -200.0], 2, 80.0, 5.0, 0.3, 0.01, 4)
    a = ref_lib.correlate(survey, grid, *args, build="parity")
    b = ref_lib.correlate(survey, grid, *args, build="pomp")
    for key in ("rbins", "rcounts", "rhist", "kbins", "kcounts", "khist", "zerolag"):
        assert np.array_equal(a[key], b[key]), key
