"""GPU parity at the benchmark configurations, against the compiled reference.

Each case builds the seeded synthetic catalogs of the configuration, runs the
whole chain (mass assignment, normalisation where the CLI does it, the
correlator) through the CUDA library, and compares with the reference C++
classes (oracle/_ref) run on the same catalogs:

  * 128^3 periodic box, L = 1000 Mpc/h, 100k uniform points with unit
    weights, rmax 200 / dr 10, kmax 0.03 / dk 0.01 (the CLI defaults),
    ell_max 0; CIC against the oracle's CIC restatement (the reference has
    no CIC), NGP and TSC against the reference MassAssignor.  The grid is
    normalised as the CLI does for periodic runs (cc/fftcorr.cc:369-375).
  * 256^3 survey sector (r 500-1500 Mpc/h, RA/Dec +-30 deg, observer at the
    origin), 2M clustered data + 20M uniform randoms, weights U[0.5, 1.5],
    TSC with the aliased window correction, ell <= 4, rmax 200 / dr 5.
  * 512^3, the same sector with 20M data + 100M randoms, kmax 0.3 / dk
    0.005, FP64 and FP32-mixed (the benchmark job,
    cc/correlate/correlator.h:406-497 at full size).

Tolerances (the same as tests/test_gpu_parity.py):
  * bin centres and counts, num_added / num_skipped: exact;
  * FP64 grids: max |gpu - ref| <= 1e-12 * max |ref| (the reference's
    unstable std::sort orders a cell's particles differently);
  * FP64 histograms: per multipole row, max |gpu - ref| <= 1e-9 * max |ref row|;
  * FP32-mixed: every xi_ell (from NN and RR by compute_xi) within
    1e-4 * rms(xi_0) of the reference's FP64 xi, every P_ell row within
    1e-4 * rms(P_0) and every NN / RR row within 1e-4 * rms(row 0).

The reference correlators run in the parity build with OpenMP
(oracle/_ref/libfcref_pomp.so), which tests/test_oracle.py pins bit for bit
to the single-threaded parity build.
"""
import numpy as np
import pytest

from oracle import fc_oracle as O
from oracle import ref_lib

import fftcorr_b200 as fb
from fftcorr_b200 import _lib, mocks
from fftcorr_b200.correlate import NO_CORRECTION, TSC_ALIASED_CORRECTION, compute_xi

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_lib.available("pomp"),
                                 reason="oracle/_ref not built")]

FP64_RTOL = 1e-9
FP32_TOL = 1e-4
GRID_RTOL = 1e-12


def _download(grid):
    out = np.empty(grid.shape)
    _lib.call("fc_grid_download", grid.handle, _lib.dptr(out))
    return out


def _assert_grid_close(gpu, ref, label):
    scale = float(np.max(np.abs(ref)))
    err = float(np.max(np.abs(gpu - ref)))
    assert err <= GRID_RTOL * scale, f"{label}: {err} vs {scale}"


def _assert_geometry_equal(res, ref):
    np.testing.assert_array_equal(res["rbins"], ref["rbins"])
    np.testing.assert_array_equal(res["kbins"], ref["kbins"])
    np.testing.assert_array_equal(res["rcounts"], ref["rcounts"])
    np.testing.assert_array_equal(res["kcounts"], ref["kcounts"])


def _assert_fp64_close(res, ref, label):
    _assert_geometry_equal(res, ref)
    for key in ("rhist", "khist"):
        for i in range(ref[key].shape[0]):
            scale = float(np.max(np.abs(ref[key][i])))
            err = float(np.max(np.abs(res[key][i] - ref[key][i])))
            assert err <= FP64_RTOL * scale + 1e-300, f"{label} {key}[{i}]: {err} vs {scale}"
    assert abs(res["zerolag"] - ref["zerolag"]) <= FP64_RTOL * abs(ref["zerolag"])


def maxdev_over_rms0(got, ref):
    """max |got_l - ref_l| / rms(ref_0) for every multipole row l."""
    got, ref = np.atleast_2d(got), np.atleast_2d(ref)
    rms0 = float(np.sqrt(np.mean(ref[0] ** 2)))
    return [float(np.max(np.abs(got[i] - ref[i]))) / rms0 for i in range(ref.shape[0])]


def _assert_fp32_close(res, ref, label):
    _assert_geometry_equal(res, ref)
    for key in ("rhist", "khist"):
        dev = maxdev_over_rms0(res[key], ref[key])
        assert max(dev) <= FP32_TOL, f"{label} {key}: {dev}"


# ------------------------------------------------ 128^3 periodic box, ell 0

BOX = 1000.0
N1 = (128, 128, 128)
CELL1 = BOX / 128
PERIODIC_ARGS = (CELL1, NO_CORRECTION, 200.0, 10.0, 0.03, 0.01, 0)


@pytest.fixture(scope="module")
def box_catalog():
    rng = np.random.default_rng(1)
    posw = np.empty((100_000, 4))
    posw[:, :3] = rng.random((100_000, 3)) * BOX
    posw[:, 3] = 1.0
    return posw


def _normalise_like_cli(grid, totw):
    mean = totw / grid.size
    grid += -mean
    grid *= 1.0 / mean
    return grid


@pytest.mark.parametrize("scheme", [0, 1, 3])
def test_periodic_box_128(box_catalog, scheme):
    posmin = np.zeros(3)
    if scheme == O.CLOUD_IN_CELL:
        ref_grid, st = O.mass_assign(box_catalog, N1, posmin, CELL1, scheme, True)
    else:
        ref_grid, st = ref_lib.mass_assign(box_catalog, N1, posmin, CELL1, scheme,
                                           True, build="parity")
    g = fb.ConfigSpaceGrid.from_geometry(N1, posmin, CELL1)
    ma = fb.MassAssignor(g, scheme, True, 1000000)
    ma.add_particles(box_catalog)
    assert ma.num_added == int(st[0]) == 100_000
    assert ma.num_skipped == int(st[1]) == 0
    assert ma.totw == st[2]
    _assert_grid_close(_download(g), ref_grid, f"box grid scheme {scheme}")
    _normalise_like_cli(ref_grid, st[2])
    mean = ma.totw / float(np.prod(N1))
    g += -mean
    g *= 1.0 / mean
    window = TSC_ALIASED_CORRECTION if scheme == 1 else NO_CORRECTION
    args = (CELL1, window) + PERIODIC_ARGS[2:]
    ref = ref_lib.correlate(False, ref_grid, CELL1, None, *args[1:], build="pomp")
    for precision in ("fp64", "fp32"):
        c = fb.PeriodicCorrelator(N1, *args, precision=precision)
        c.autocorrelate(g)
        res = c.results()
        if precision == "fp64":
            _assert_fp64_close(res, ref, f"box scheme {scheme}")
        else:
            _assert_fp32_close(res, ref, f"box scheme {scheme} fp32")


# -------------------------------------------------------- survey sectors

def _sector_case(ngrid, nd, nr, kmax, dk):
    sector = mocks.Sector()
    shape = (ngrid,) * 3
    posmin, cell = mocks.survey_box(sector, 200.0, shape)
    D = mocks.sector_clustered(nd, 2, sector=sector)
    R = mocks.sector_randoms(nr, 3, sector=sector)
    R[:, 3] *= -(D[:, 3].sum() / R[:, 3].sum())
    args = (cell, posmin, TSC_ALIASED_CORRECTION, 200.0, 5.0, kmax, dk, 4)
    nn, rr, _ = ref_lib.survey_job(D, R, shape, posmin, cell, TSC_ALIASED_CORRECTION,
                                   200.0, 5.0, kmax, dk, 4, build="pomp")
    return {"shape": shape, "posmin": posmin, "cell": cell, "D": D, "R": R,
            "args": args, "nn": nn, "rr": rr,
            "xi": compute_xi(nn["rhist"].T, rr["rhist"].T)}


def _gpu_sector_job(case, precision):
    shape, posmin, cell = case["shape"], case["posmin"], case["cell"]
    # Grids of the form's precision, as the benchmark job uses them (FP32
    # cells for the FP32-mixed form).
    gA = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision=precision)
    gB = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision=precision)
    tsc = fb.DistributionScheme.TRIANGULAR_SHAPED_CLOUD
    maA = fb.MassAssignor(gA, tsc, False, 0)
    maB = fb.MassAssignor(gB, tsc, False, 0)
    maA.add_particles(case["D"])
    maB.add_particles(case["R"])
    for ma, st in ((maA, case["nn"]["ma_stats"]), (maB, case["rr"]["ma_stats"])):
        assert ma.num_added == int(st[0])
        assert ma.num_skipped == int(st[1])
    grids = (_download(gA), _download(gB)) if precision == "fp64" else None
    gA.add_grid(gB)
    c = fb.Correlator(shape, *case["args"], precision=precision)
    c.autocorrelate(gA)
    nn = c.results()
    c.autocorrelate(gB)
    rr = c.results()
    return nn, rr, compute_xi(nn["rhist"].T, rr["rhist"].T), grids


def _check_sector(case, precision, label):
    nn, rr, xi, grids = _gpu_sector_job(case, precision)
    if precision == "fp64":
        _assert_fp64_close(nn, case["nn"], label + " NN")
        _assert_fp64_close(rr, case["rr"], label + " RR")
        dev = maxdev_over_rms0(xi.T, case["xi"].T)
        assert max(dev) <= 1e-8, f"{label} xi: {dev}"
    else:
        _assert_fp32_close(nn, case["nn"], label + " NN fp32")
        _assert_fp32_close(rr, case["rr"], label + " RR fp32")
        dev = maxdev_over_rms0(xi.T, case["xi"].T)
        assert max(dev) <= FP32_TOL, f"{label} xi fp32: {dev}"
    return grids


@pytest.fixture(scope="module")
def sector256():
    return _sector_case(256, 2_000_000, 20_000_000, 0.03, 0.01)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_survey_sector_256(sector256, precision):
    grids = _check_sector(sector256, precision, "sector256")
    if grids is not None:
        # Grids against the reference MassAssignor (run in the parity
        # build with OpenMP: its parallel merge sort orders a cell's
        # particles differently from the stable GPU sort, so the sums
        # agree to rounding).
        shape, posmin, cell = sector256["shape"], sector256["posmin"], sector256["cell"]
        refA, _ = ref_lib.mass_assign(sector256["D"], shape, posmin, cell, 1, False,
                                      build="pomp")
        _assert_grid_close(grids[0], refA, "sector256 D grid")


@pytest.fixture(scope="module")
def sector512():
    return _sector_case(512, 20_000_000, 100_000_000, 0.3, 0.005)


@pytest.mark.slow
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_survey_sector_512_benchmark_job(sector512, precision):
    _check_sector(sector512, precision, "sector512")
