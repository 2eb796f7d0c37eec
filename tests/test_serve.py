"""The serving form (fftcorr_b200.serve, fc_server_* in include/fc_api.h).

Each job's result must be the same alone and in a mix of concurrently
running jobs: the same kernels run on the same data, so the tables are
compared bit for bit.  A job's result must also equal the single-job path
through the reference-style API (MassAssignor + normalisation + correlator).
Admission never lets the accounted device bytes exceed the budget.
"""
import ctypes

import numpy as np
import pytest

from conftest import clustered_catalog

import fftcorr_b200 as fb
from fftcorr_b200 import _lib, mocks
from fftcorr_b200.correlate import NO_CORRECTION, TSC_ALIASED_CORRECTION
from fftcorr_b200.serve import (CAT_CLUSTERED_BOX, CAT_HOST, CAT_SECTOR_CLUSTERED,
                                CAT_SECTOR_UNIFORM, JobSpec, Server, catalog_spec)

pytestmark = pytest.mark.gpu

GB = 1 << 30


def _periodic(n, L, npart, seed, precision="fp32", maxell=2, scheme=3):
    data = catalog_spec(CAT_CLUSTERED_BOX, n=npart, boxsize=L, ncentres=50,
                        sigma=5.0, seed=seed)
    return JobSpec("periodic", (n, n, n), L / n, data, scheme=scheme,
                   rmax=60.0, dr=5.0, kmax=0.2, dk=0.02, maxell=maxell,
                   precision=precision)


def _survey(n, nd, nr, seed, precision="fp32", maxell=2):
    sector = mocks.Sector()
    posmin, cell = mocks.survey_box(sector, 200.0, (n, n, n))
    data = catalog_spec(CAT_SECTOR_CLUSTERED, n=nd, ncentres=200, sigma=5.0,
                        wmin=0.5, wmax=1.5, seed=seed)
    rand = catalog_spec(CAT_SECTOR_UNIFORM, n=nr, wmin=0.5, wmax=1.5, seed=seed + 1)
    return JobSpec("survey", (n, n, n), cell, data, rand, posmin=posmin,
                   scheme=fb.DistributionScheme.TRIANGULAR_SHAPED_CLOUD,
                   window=TSC_ALIASED_CORRECTION, rmax=200.0, dr=20.0,
                   kmax=0.05, dk=0.01, maxell=maxell, precision=precision)


def _mix():
    return [_periodic(32, 400.0, 20000, 1), _survey(48, 30000, 90000, 2),
            _periodic(48, 600.0, 60000, 3, precision="fp64", maxell=0, scheme=1),
            _survey(40, 20000, 50000, 4, precision="fp64", maxell=4),
            _periodic(40, 500.0, 40000, 5, maxell=4),
            _survey(48, 30000, 90000, 6),
            _periodic(32, 400.0, 20000, 7)]


def _collect(server, tickets, specs):
    out = []
    for t, s in zip(tickets, specs):
        assert server.wait(t, timeout=300)
        inf = server.info(t)
        assert inf["status"] == 0, inf["message"]
        r = [server.results(t, 0)]
        if s.kind == "survey":
            r.append(server.results(t, 1))
        out.append(r)
    return out


def test_results_same_alone_and_in_the_mix():
    specs = _mix()
    alone = Server(40 * GB, slots=1)
    ref = []
    for s in specs:
        t = alone.submit(s)
        ref += _collect(alone, [t], [s])
    alone.close()
    mix = Server(40 * GB, slots=4)
    tickets = [mix.submit(s) for s in specs]
    got = _collect(mix, tickets, specs)
    st = mix.stats()
    mix.close()
    assert st["peak_running"] >= 2          # jobs really overlapped
    assert st["completed"] == len(specs)
    for i, (a, b) in enumerate(zip(ref, got)):
        for ra, rb in zip(a, b):
            for key in ("rcounts", "kcounts", "rhist", "khist"):
                np.testing.assert_array_equal(ra[key], rb[key], err_msg=f"job {i} {key}")
            assert ra["zerolag"] == rb["zerolag"]


def test_periodic_job_equals_direct_api():
    n, L = 40, 500.0
    posw = clustered_catalog(50000, [0, 0, 0], [L, L, L], 9, ncenters=40)
    spec = JobSpec("periodic", (n, n, n), L / n, catalog_spec(CAT_HOST, posw=posw),
                   rmax=60.0, dr=5.0, kmax=0.2, dk=0.02, maxell=2, precision="fp32")
    srv = Server(8 * GB, slots=2)
    t = srv.submit(spec)
    got = _collect(srv, [t], [spec])[0][0]
    srv.close()
    # A served FP32-mixed job works on FP32 grids.
    g = fb.ConfigSpaceGrid.from_geometry((n, n, n), [0, 0, 0], L / n, precision="fp32")
    ma = fb.MassAssignor(g, fb.DistributionScheme.CLOUD_IN_CELL, True, 0)
    ma.add_particles(posw)
    mean = ma.totw / n ** 3
    g -= mean
    g *= 1.0 / mean
    corr = fb.PeriodicCorrelator((n, n, n), L / n, NO_CORRECTION, 60.0, 5.0, 0.2,
                                 0.02, 2, precision="fp32")
    corr.autocorrelate(g)
    ref = corr.results()
    for key in ("rcounts", "kcounts", "rhist", "khist"):
        np.testing.assert_array_equal(got[key], ref[key])


def test_survey_job_equals_direct_api():
    from fftcorr_b200 import catalog
    spec = _survey(40, 20000, 60000, 11, maxell=2)
    srv = Server(8 * GB, slots=2)
    t = srv.submit(spec)
    nn, rr = _collect(srv, [t], [spec])[0]
    srv.close()
    j = spec.job
    D = catalog.DeviceCatalog(j.data.n)
    _lib.call("fc_catalog_generate", j.data, ctypes.c_void_p(D.ptr))
    R = catalog.DeviceCatalog(j.randoms.n)
    _lib.call("fc_catalog_generate", j.randoms, ctypes.c_void_p(R.ptr))
    shape, posmin, cell = tuple(j.shape), tuple(j.posmin), j.cell
    gA = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision="fp32")
    gB = fb.ConfigSpaceGrid.from_geometry(shape, posmin, cell, precision="fp32")
    tsc = fb.DistributionScheme.TRIANGULAR_SHAPED_CLOUD
    mA = fb.MassAssignor(gA, tsc, False, 0)
    mB = fb.MassAssignor(gB, tsc, False, 0)
    mA.add_particles_device(D.ptr, D.n)
    mB.add_particles_device(R.ptr, R.n)
    gB *= -(mA.totw / mB.totw)
    gA.add_grid(gB)
    corr = fb.Correlator(shape, cell, posmin, TSC_ALIASED_CORRECTION, 200.0, 20.0,
                         0.05, 0.01, 2, precision="fp32")
    corr.autocorrelate(gA)
    ref_nn = corr.results()
    corr.autocorrelate(gB)
    ref_rr = corr.results()
    for got, ref in ((nn, ref_nn), (rr, ref_rr)):
        for key in ("rcounts", "kcounts", "rhist", "khist"):
            np.testing.assert_array_equal(got[key], ref[key])


def test_admission_by_footprint():
    a = _periodic(48, 600.0, 50000, 21)
    fp = a.footprint
    # A job larger than the whole budget is refused at submission.
    small = Server(fp // 2, slots=2)
    with pytest.raises(_lib.AdmissionError):
        small.submit(a)
    small.close()
    # Room for one such job at a time: both run, one after the other.
    srv = Server(int(fp * 1.5), slots=3)
    specs = [a, _periodic(48, 600.0, 50000, 22)]
    tickets = [srv.submit(s) for s in specs]
    _collect(srv, tickets, specs)
    st = srv.stats()
    srv.close()
    assert st["peak_running"] == 1
    assert st["peak_bytes"] <= st["budget"]


def test_resident_objects_are_reused():
    srv = Server(8 * GB, slots=1)
    for seed in (31, 32, 33):
        s = _periodic(32, 400.0, 10000, seed)
        _collect(srv, [srv.submit(s)], [s])
    st = srv.stats()
    srv.close()
    assert st["resident_objects"] == 2      # one grid + one correlator
    assert st["evictions"] == 0


def test_failed_job_reports_its_status():
    srv = Server(8 * GB, slots=2)
    bad = _survey(32, 1000, 1000, 41)
    bad.job.randoms.wmin = 0.0
    bad.job.randoms.wmax = 0.0
    t = srv.submit(bad)
    assert srv.wait(t, timeout=120)
    inf = srv.info(t)
    assert inf["status"] == _lib.FC_ERR_INVALID
    with pytest.raises(ValueError):
        srv.results(t)
    good = _periodic(32, 400.0, 10000, 42)
    _collect(srv, [srv.submit(good)], [good])
    srv.close()
