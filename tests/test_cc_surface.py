"""The C++ class surface (include/fftcorr_cc): the reference's class names and
signatures as the Cython package binds them (fftcorr/*/*.pxd), implemented
over the C ABI.

* Without a GPU: the headers and tests/cc/test_cc_surface.cc compile as
  C++11 (the reference's Cython extensions build with -std=c++11).
* On the GPU: the test program runs ConfigSpaceGrid, MassAssignor (all
  four add overloads, buffered and direct), Correlator (auto and cross),
  PeriodicCorrelator and HistogramList, and its outputs are checked against
  the oracle with the tolerances of tests/test_gpu_parity.py (counts and
  bins exact, FP64 grids 1e-12 and histograms 1e-9 of the row maximum);
  argument errors raise the reference's std::invalid_argument.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, clustered_catalog
from oracle import fc_oracle as O
from oracle import ref_lib

SRC = os.path.join(ROOT, "tests", "cc", "test_cc_surface.cc")
INC = [os.path.join(ROOT, "include", "fftcorr_cc"), os.path.join(ROOT, "include")]
LIBDIR = os.path.join(ROOT, "fftcorr_b200")


def _compile(out, syntax_only=False):
    cmd = ["g++", "-std=c++11", "-O2", "-Wall", "-Werror"]
    for d in INC:
        cmd += ["-I", d]
    cmd.append(SRC)
    if syntax_only:
        cmd.append("-fsyntax-only")
    else:
        cmd += ["-o", out, "-L", LIBDIR, "-lfftcorr_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cc_surface_compiles_as_cxx11():
    _compile(None, syntax_only=True)


SHAPE = (32, 36, 40)
CELL = 10.0
POSMIN = np.array([-120.0, 300.0, -150.0])


def _read(d, name, dtype, shape):
    return np.fromfile(os.path.join(d, name + ".bin"), dtype=dtype).reshape(shape)


def _results(d, tag, maxell, ref):
    nrows = maxell // 2 + 1
    nr, nk = ref["rbins"].size, ref["kbins"].size
    return {
        "rbins": _read(d, tag + "_rbins", np.float64, (nr,)),
        "rcounts": _read(d, tag + "_rcounts", np.int32, (nrows, nr)),
        "rhist": _read(d, tag + "_rhist", np.float64, (nrows, nr)),
        "kbins": _read(d, tag + "_kbins", np.float64, (nk,)),
        "kcounts": _read(d, tag + "_kcounts", np.int32, (nrows, nk)),
        "khist": _read(d, tag + "_khist", np.float64, (nrows, nk)),
        "zerolag": float(_read(d, tag + "_zerolag", np.float64, (1,))[0]),
    }


def _assert_close(got, ref, label):
    for key in ("rbins", "kbins", "rcounts", "kcounts"):
        np.testing.assert_array_equal(got[key], ref[key], err_msg=f"{label} {key}")
    for key in ("rhist", "khist"):
        for i in range(ref[key].shape[0]):
            scale = float(np.max(np.abs(ref[key][i])))
            err = float(np.max(np.abs(got[key][i] - ref[key][i])))
            assert err <= 1e-9 * scale + 1e-300, f"{label} {key}[{i}]"
    assert abs(got["zerolag"] - ref["zerolag"]) <= 1e-9 * abs(ref["zerolag"])


@pytest.mark.gpu
@pytest.mark.skipif(not ref_lib.available("parity"), reason="oracle/_ref not built")
def test_cc_surface_matches_oracle(tmp_path):
    exe = str(tmp_path / "test_cc_surface")
    _compile(exe)
    box = np.array(SHAPE) * CELL
    posw = clustered_catalog(30000, POSMIN - 0.05 * box, POSMIN + 1.05 * box, 17)
    posw[15000:, 3] *= -posw[:15000, 3].sum() / posw[15000:, 3].sum()
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array(SHAPE, dtype=np.int32).tofile(f)
        POSMIN.tofile(f)
        np.array([CELL]).tofile(f)
        np.array([posw.shape[0]], dtype=np.int64).tofile(f)
        posw.tofile(f)
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([exe, str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    d = str(out)

    ref_grid, st = O.mass_assign(posw, SHAPE, POSMIN, CELL, O.TRIANGULAR_SHAPED_CLOUD)
    grid = _read(d, "grid", np.float64, SHAPE)
    scale = float(np.max(np.abs(ref_grid)))
    assert float(np.max(np.abs(grid - ref_grid))) <= 1e-12 * scale
    stats = _read(d, "stats", np.float64, (4,))
    assert stats[0] == st[0] and stats[1] == st[1]
    np.testing.assert_allclose(stats[2:], st[2:], rtol=1e-12)
    unit = posw.copy()
    unit[:, 3] = 1.0
    ref_grid2, _ = O.mass_assign(unit, SHAPE, POSMIN, CELL, O.NEAREST_CELL)
    grid2 = _read(d, "grid2", np.float64, SHAPE)
    assert np.array_equal(grid2, ref_grid2)

    coords = _read(d, "coords", np.float64, (3,))
    np.testing.assert_array_equal(coords, [1.5, 2.25, 0.5])
    assert _read(d, "inside", np.int32, (1,))[0] == 1

    sargs = (CELL, POSMIN, 2, 60.0, 10.0, 0.2, 0.04, 4)
    ref = ref_lib.correlate(True, ref_grid, *sargs)
    _assert_close(_results(d, "survey", 4, ref), ref, "survey")
    refx = ref_lib.correlate(True, ref_grid, *sargs, grid2=ref_grid2)
    _assert_close(_results(d, "cross", 4, refx), refx, "cross")
    pargs = (CELL, None, 0, 60.0, 10.0, 0.2, 0.04, 2)
    refp = ref_lib.correlate(False, ref_grid2, *pargs)
    _assert_close(_results(d, "periodic", 2, refp), refp, "periodic")

    h = O.Histogram(2, -10.0, 10.0, 2.0)
    m = 1000
    x = -12.0 + 24.0 * (np.arange(m) + 0.5) / m
    y = 0.001 * np.arange(m) - 0.3
    h.accumulate(0, x, y)
    h.accumulate(1, y, x)
    h.accumulate(1, x, x)
    nb = h.bins.size
    np.testing.assert_array_equal(_read(d, "hist_bins", np.float64, (nb,)), h.bins)
    np.testing.assert_array_equal(_read(d, "hist_counts", np.int32, (2, nb)), h.counts)
    np.testing.assert_allclose(_read(d, "hist_values", np.float64, (2, nb)), h.hist,
                               rtol=1e-12, atol=1e-12)

    assert _read(d, "errors", np.int32, (5,)).tolist() == [1, 1, 1, 1, 1]


def _reference_tree():
    import __graft_entry__
    ref = os.environ.get("FFTCORR_REFERENCE", __graft_entry__.REFERENCE)
    return ref if os.path.isdir(os.path.join(ref, "fftcorr")) else None


@pytest.mark.skipif(_reference_tree() is None, reason="reference tree not present")
def test_reference_cython_package_compiles_against_cc_surface(tmp_path):
    """The reference's own .pyx/.pxd files, unmodified (copied to a scratch
    directory at test time), cythonized and compiled as C++11 against
    include/fftcorr_cc instead of the reference's cc/ tree: every class,
    method and enum the Cython package binds resolves to this surface."""
    import shutil
    import sysconfig
    pytest.importorskip("Cython")
    numpy_inc = np.get_include()
    pkg = tmp_path / "pkg"
    shutil.copytree(os.path.join(_reference_tree(), "fftcorr"), pkg / "fftcorr")
    inc = INC[0]
    incs = [sysconfig.get_paths()["include"], numpy_inc, inc] + [
        os.path.join(inc, d) for d in ("array", "grid", "particle_mesh", "correlate",
                                       "histogram", "fftw")] + [
        INC[1], str(pkg / "fftcorr" / "array")]
    modules = ["array/row_major_array", "grid/config_space_grid", "grid/utils",
               "particle_mesh/mass_assignor", "correlate/correlator",
               "histogram/histogram_list", "fftw/fftw"]
    for m in modules:
        cpp = str(tmp_path / (os.path.basename(m) + ".cpp"))
        subprocess.run(["cython", "--cplus", "-3", "-I", str(pkg),
                        str(pkg / "fftcorr" / (m + ".pyx")), "-o", cpp],
                       check=True, capture_output=True, text=True)
        cmd = ["g++", "-std=c++11", "-fsyntax-only", cpp]
        for d in incs:
            cmd += ["-I", d]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, f"{m}: {r.stderr[-2000:]}"
