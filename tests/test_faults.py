"""Failure paths, made on the host (fc_fault_inject / fc_set_device_budget):
the planned failure is raised where the real one would surface, before the
CUDA or cuFFT call, so no GPU faults.

The reference fails on an allocation or a plan it cannot make
(cc/grid/fft_grid.cc:126,153).  Each failure must:
* surface as the mapped exception type (MemoryError for an allocation,
  FcError for a cuFFT plan);
* leave no device memory behind (fc_device_bytes before == after);
* leave the library usable: the same call succeeds once the fault is gone,
  with results equal to the oracle's.
A serving job that fails mid-stream reports its status while the jobs
around it complete, and a bounded wait that runs out returns FC_ERR_TIMEOUT.
"""
import ctypes

import numpy as np
import pytest

from conftest import clustered_catalog
from oracle import fc_oracle as O

import fftcorr_b200 as fb
from fftcorr_b200 import _lib
from fftcorr_b200.serve import CAT_CLUSTERED_BOX, JobSpec, Server, catalog_spec

pytestmark = pytest.mark.gpu


def _device_bytes():
    b = ctypes.c_size_t()
    _lib.call("fc_device_bytes", ctypes.byref(b))
    return b.value


@pytest.fixture(autouse=True)
def _disarm():
    yield
    _lib.call("fc_fault_inject", _lib.FC_FAULT_DEVICE_ALLOC, 0)
    _lib.call("fc_fault_inject", _lib.FC_FAULT_FFT_PLAN, 0)
    _lib.call("fc_set_device_budget", 0)


def _catalog(shape, cell, posmin, seed):
    box = np.array(shape) * cell
    return clustered_catalog(20000, posmin, posmin + box, seed)


def test_unknown_fault_kind_is_rejected():
    with pytest.raises(ValueError):
        _lib.call("fc_fault_inject", 99, 1)


def test_device_budget_refuses_a_grid_then_allows_it():
    shape, cell, posmin = (64, 64, 64), 5.0, np.zeros(3)
    before = _device_bytes()
    _lib.call("fc_set_device_budget", before + (1 << 20))
    with pytest.raises(MemoryError):
        fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell)
    assert _device_bytes() == before
    _lib.call("fc_set_device_budget", 0)
    g = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell)
    posw = _catalog(shape, cell, posmin, 3)
    ma = fb.MassAssignor(g, 1, False, 0)
    ma.add_particles(posw)
    ref, _ = O.mass_assign(posw, shape, posmin, cell, 1, False)
    got = np.asarray(g)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("nth", [1, 2, 5])
def test_allocation_failure_in_a_correlator_leaves_nothing_behind(nth):
    shape, cell = (32, 32, 32), 10.0
    posmin = np.array([-160.0, -160.0, 20.0])
    args = (cell, posmin, 2, 60.0, 10.0, 0.2, 0.04, 2)
    before = _device_bytes()
    _lib.call("fc_fault_inject", _lib.FC_FAULT_DEVICE_ALLOC, nth)
    with pytest.raises(MemoryError):
        fb.Correlator(shape, *args)
    assert _device_bytes() == before
    grid, _ = O.mass_assign(_catalog(shape, cell, posmin, 4), shape, posmin, cell, 1)
    c = fb.Correlator(shape, *args)
    c.autocorrelate(grid)
    ref = O.survey_correlate(grid, *args)
    res = c.results()
    np.testing.assert_array_equal(res["rcounts"], ref["rcounts"])
    assert np.max(np.abs(res["rhist"] - ref["rhist"])) <= 1e-9 * np.max(np.abs(ref["rhist"]))


def test_fft_plan_failure_is_reported_and_the_next_plan_works():
    shape, cell = (32, 40, 36), 10.0
    args = (cell, 0, 60.0, 7.0, 0.25, 0.02, 2)
    before = _device_bytes()
    _lib.call("fc_fault_inject", _lib.FC_FAULT_FFT_PLAN, 1)
    with pytest.raises(_lib.FcError) as e:
        fb.PeriodicCorrelator(shape, *args)
    assert e.value.code == _lib.FC_ERR_CUFFT
    assert _device_bytes() == before
    grid = np.random.default_rng(5).standard_normal(shape)
    c = fb.PeriodicCorrelator(shape, *args)
    c.autocorrelate(grid)
    ref = O.periodic_correlate(grid, *args)
    np.testing.assert_array_equal(c.results()["rcounts"], ref["rcounts"])


def test_assignor_survives_a_failed_add():
    shape, cell, posmin = (32, 32, 32), 10.0, np.zeros(3)
    posw = _catalog(shape, cell, posmin, 6)
    g = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell)
    ma = fb.MassAssignor(g, 1, False, 0)
    _lib.call("fc_fault_inject", _lib.FC_FAULT_DEVICE_ALLOC, 1)
    with pytest.raises(MemoryError):
        ma.add_particles(posw)
    ma.clear()
    g.clear()
    ma.add_particles(posw)
    assert ma.num_added == len(posw)
    ref, _ = O.mass_assign(posw, shape, posmin, cell, 1, False)
    assert np.max(np.abs(np.asarray(g) - ref)) <= 1e-12 * np.max(np.abs(ref))


def _box_job(n, seed):
    data = catalog_spec(CAT_CLUSTERED_BOX, n=20000, boxsize=400.0, ncentres=50,
                        sigma=5.0, seed=seed)
    return JobSpec("periodic", (n, n, n), 400.0 / n, data, rmax=60.0, dr=5.0,
                   kmax=0.2, dk=0.02, maxell=2, precision="fp64")


def test_serving_job_failure_is_isolated():
    srv = Server(8 << 30, slots=1)
    try:
        a = srv.submit(_box_job(32, 1))
        assert srv.wait(a, timeout=120)
        ta = srv.tables(a)
        # The next correlator the server builds (a new shape) cannot plan
        # its FFT: that job fails with its status, the others complete.
        _lib.call("fc_fault_inject", _lib.FC_FAULT_FFT_PLAN, 1)
        b = srv.submit(_box_job(40, 2))
        c = srv.submit(_box_job(32, 1))
        assert srv.wait(b, timeout=120) and srv.wait(c, timeout=120)
        assert srv.info(b)["status"] == _lib.FC_ERR_CUFFT
        with pytest.raises(_lib.FcError):
            srv.tables(b)
        assert srv.info(c)["status"] == 0
        tc = srv.tables(c)
        for x, y in zip(ta, tc):
            assert np.array_equal(np.asarray(x["histogram"]), np.asarray(y["histogram"]))
        # With the fault gone the same shape builds and runs.
        d = srv.submit(_box_job(40, 2))
        assert srv.wait(d, timeout=120)
        assert srv.info(d)["status"] == 0
    finally:
        srv.close()


def test_bounded_wait_runs_out_with_timeout_status():
    srv = Server(8 << 30, slots=1)
    try:
        t = srv.submit(_box_job(64, 3))
        done = ctypes.c_int(7)
        rc = _lib.load().fc_server_wait(srv._handle, t, 0.0, ctypes.byref(done))
        if rc == _lib.FC_ERR_TIMEOUT:
            assert done.value == 0
        else:
            assert rc == 0 and done.value == 1   # it had already finished
        assert srv.wait(t, timeout=120)
    finally:
        srv.close()
