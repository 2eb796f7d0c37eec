"""The batched form (fftcorr_b200.batch.PeriodicBatch, fc_batch_* in
include/fc_api.h) against the single-box path and the oracle.

Per box the batch must give what MassAssignor + the CLI's periodic
normalisation + PeriodicCorrelator give on that box alone.  In the same
precision that is the same bits: the graph runs the same kernels on the same
data, only the launch shapes (per-cell independent) and the stream differ,
and the batched histogram kernel reduces the same chunks in the same order.
FP64 batches are also checked against the oracle (rtol 1e-9 per multipole
row, as the single-box FP64 parity tests), FP32 batches within 1e-4 of the
monopole rms.
"""
import numpy as np
import pytest

from conftest import clustered_catalog
from oracle import fc_oracle as O

import fftcorr_b200 as fb
from fftcorr_b200.batch import PeriodicBatch
from fftcorr_b200.correlate import NO_CORRECTION

pytestmark = pytest.mark.gpu

RMAX, DR, KMAX, DK = 60.0, 5.0, 0.2, 0.02


def _boxes():
    spec = [((32, 32, 32), 400.0, 30000, 1), ((48, 48, 48), 600.0, 80000, 2),
            ((24, 36, 30), 10.0 * 24, 20000, 3), ((32, 32, 32), 500.0, 5000, 4),
            ((40, 40, 40), 480.0, 120000, 5), ((27, 27, 27), 270.0, 15000, 6)]
    boxes = []
    for shape, lx, n, seed in spec:
        cell = lx / shape[0]
        hi = np.array(shape) * cell
        posw = clustered_catalog(n, [0, 0, 0], hi, seed, ncenters=30)
        posw[:, 3] = np.random.default_rng(seed).uniform(0.5, 1.5, n)
        boxes.append((shape, cell, posw))
    return boxes


def _single_box(shape, cell, posw, precision, maxell=2):
    # The batch's grids have its precision (FP32 cells in the FP32 form).
    g = fb.ConfigSpaceGrid.from_geometry(shape, [0, 0, 0], cell, precision=precision)
    ma = fb.MassAssignor(g, fb.DistributionScheme.CLOUD_IN_CELL, True, 0)
    ma.add_particles(np.ascontiguousarray(posw))
    mean = ma.totw / (shape[0] * shape[1] * shape[2])
    g -= mean
    g *= 1.0 / mean
    corr = fb.PeriodicCorrelator(shape, cell, NO_CORRECTION, RMAX, DR, KMAX, DK,
                                 maxell, precision=precision)
    corr.autocorrelate(g)
    return corr.results(), ma


def _batch(boxes, precision, **kw):
    return PeriodicBatch(boxes, fb.DistributionScheme.CLOUD_IN_CELL, RMAX, DR,
                         KMAX, DK, 2, NO_CORRECTION, precision, **kw)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_equals_single_box_path(precision):
    boxes = _boxes()
    b = _batch(boxes, precision)
    b.run()
    for i, (shape, cell, posw) in enumerate(boxes):
        ref, ma = _single_box(shape, cell, posw, precision)
        got = b.results(i)
        for key in ("rbins", "kbins", "rcounts", "kcounts", "rhist", "khist"):
            np.testing.assert_array_equal(got[key], ref[key], err_msg=f"box {i} {key}")
        assert got["zerolag"] == ref["zerolag"]
        st = b.stats(i)
        assert st["num_added"] == ma.num_added and st["totw"] == ma.totw


def test_fp64_batch_matches_oracle():
    boxes = _boxes()[:3]
    b = _batch(boxes, "fp64")
    b.run()
    for i, (shape, cell, posw) in enumerate(boxes):
        grid, st = O.mass_assign(posw, shape, [0, 0, 0], cell, 3, True)
        delta = O.normalise_periodic(grid, st[2])
        ref = O.periodic_correlate(delta, cell, NO_CORRECTION, RMAX, DR, KMAX, DK, 2)
        got = b.results(i)
        np.testing.assert_array_equal(got["rcounts"], ref["rcounts"])
        np.testing.assert_array_equal(got["kcounts"], ref["kcounts"])
        for key in ("rhist", "khist"):
            for row in range(ref[key].shape[0]):
                scale = np.max(np.abs(ref[key][row]))
                assert np.max(np.abs(got[key][row] - ref[key][row])) <= 1e-9 * scale


def test_fp32_batch_within_tolerance_of_fp64():
    boxes = _boxes()[3:]
    b32 = _batch(boxes, "fp32")
    b64 = _batch(boxes, "fp64")
    b32.run()
    b64.run()
    for i in range(len(boxes)):
        r32, r64 = b32.results(i), b64.results(i)
        for key in ("rhist", "khist"):
            rms0 = np.sqrt(np.mean(r64[key][0] ** 2))
            assert np.max(np.abs(r32[key] - r64[key])) <= 1e-4 * rms0


def test_replays_are_identical_and_info_is_sane():
    boxes = _boxes()
    b = _batch(boxes, "fp32")
    b.run()
    first = [b.results(i) for i in range(len(boxes))]
    b.launch()
    t = b.wait()
    assert t > 0
    for i in range(len(boxes)):
        np.testing.assert_array_equal(b.results(i)["rhist"], first[i]["rhist"])
        np.testing.assert_array_equal(b.results(i)["khist"], first[i]["khist"])
    info = b.info
    assert info["nboxes"] == len(boxes)
    assert 1 <= info["lanes"] <= len(boxes)
    assert info["kernel_nodes"] >= info["own_kernel_nodes"] > 0
    assert info["hist_items"] > 0
    ps, xi = b.tables(0)
    assert list(xi.keys()) == ["r", "xi", "histogram", "count"]


def test_tuning_table_round_trip(tmp_path):
    from fftcorr_b200 import fftw
    boxes = _boxes()[:2]
    a = _batch(boxes, "fp32")
    a.run()
    assert fftw.wisdom_entries() > 0
    path = str(tmp_path / "tune.txt")
    fftw.export_wisdom_to_file(path)
    fftw.forget_wisdom()
    assert fftw.wisdom_entries() == 0
    fftw.import_wisdom_from_file(path)
    n = fftw.wisdom_entries()
    assert n > 0
    # A batch built from the imported table times nothing new and agrees.
    b = _batch(boxes, "fp32", tune=False)
    b.run()
    assert fftw.wisdom_entries() == n
    for i in range(len(boxes)):
        np.testing.assert_array_equal(a.results(i)["rhist"], b.results(i)["rhist"])


def test_fixed_lane_counts_agree():
    boxes = _boxes()
    ref = None
    for lanes in (1, 3):
        b = _batch(boxes, "fp32", lanes=lanes)
        b.run()
        assert b.info["lanes"] == lanes
        out = [b.results(i)["rhist"] for i in range(len(boxes))]
        if ref is None:
            ref = out
        else:
            for x, y in zip(out, ref):
                np.testing.assert_array_equal(x, y)


def test_batch_rejects_bad_input():
    with pytest.raises(ValueError):
        PeriodicBatch([], precision="fp32")
    with pytest.raises(ValueError):
        _batch([((16, 16, 16), -1.0, np.zeros((10, 4)))], "fp32")
    with pytest.raises(ValueError):
        _batch([((16, 16, 16), 10.0, np.zeros((10, 3)))], "fp32")
