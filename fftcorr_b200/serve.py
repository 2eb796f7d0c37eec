"""Serving form: a request loop over correlation jobs with continuous
batching and admission by HBM footprint (fc_server_* in include/fc_api.h).

A job is one catalog's run of the reference pipeline (cc/fftcorr.cc:233-463):
periodic -- assign, delta = (rho - mean) / mean, PeriodicCorrelator; survey --
NN grid D - alpha R (alpha = sum w_D / sum w_R, randoms negated as
fftcorr/fftcorr.py:538 does), Correlator, and optionally the RR grid for
compute_xi.  `slots` workers take queued jobs as soon as a slot and memory
are free, so jobs that arrive while others run overlap on the GPU; grids and
correlators (FFT plans, bin indices) stay resident per configuration.

Catalogs are described by value (`catalog_spec`): a host or device array,
or a seeded device-generated catalog, so a stream of requests need not hold
every catalog in memory.
"""
import ctypes

import numpy as np

from fftcorr_b200 import _lib
from fftcorr_b200.correlate.correlator import (NO_CORRECTION, _PRECISIONS,
                                               BaseCorrelator)
from fftcorr_b200.particle_mesh import DistributionScheme

CAT_DEVICE, CAT_HOST, CAT_UNIFORM_BOX, CAT_CLUSTERED_BOX = 0, 1, 2, 3
CAT_SECTOR_UNIFORM, CAT_SECTOR_CLUSTERED = 4, 5


def catalog_spec(kind, n=0, posw=None, boxsize=0.0, ncentres=10000, sigma=5.0,
                 rmin=500.0, rmax=1500.0, ra_deg=30.0, dec_deg=30.0,
                 wmin=1.0, wmax=1.0, wsign=1.0, seed=0):
    """A catalog for a job.  kind CAT_HOST takes an (n, 4) FP64 array (kept
    alive by the returned spec), CAT_DEVICE a DeviceCatalog."""
    c = _lib.CatalogSpec()
    c.kind = int(kind)
    keep = None
    if kind == CAT_HOST:
        keep = np.ascontiguousarray(posw, dtype=np.float64)
        if keep.ndim != 2 or keep.shape[1] != 4:
            raise ValueError("posw must be (n, 4)")
        n = keep.shape[0]
        c.posw = keep.ctypes.data
    elif kind == CAT_DEVICE:
        keep = posw
        n = posw.n
        c.posw = posw.ptr
    c.n = int(n)
    c.boxsize = float(boxsize)
    c.ncentres = int(ncentres)
    c.sigma = float(sigma)
    c.rmin, c.rmax = float(rmin), float(rmax)
    c.ra_half, c.dec_half = np.deg2rad(ra_deg), np.deg2rad(dec_deg)
    c.wmin, c.wmax, c.wsign = float(wmin), float(wmax), float(wsign)
    c.seed = int(seed) & (2 ** 64 - 1)
    return c, keep


class JobSpec:
    """A correlation request (see module docstring)."""

    def __init__(self, kind, shape, cell, data, randoms=None, posmin=(0, 0, 0),
                 scheme=DistributionScheme.CLOUD_IN_CELL, window=NO_CORRECTION,
                 rmax=200.0, dr=5.0, kmax=0.1, dk=0.005, maxell=2,
                 precision="fp32", want_rr=True):
        if kind not in ("periodic", "survey"):
            raise ValueError("kind must be 'periodic' or 'survey'")
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be 'fp64' or 'fp32', got {precision!r}")
        j = _lib.Job()
        _lib.call("fc_job_init", ctypes.byref(j))
        j.kind = _lib.FC_PERIODIC if kind == "periodic" else _lib.FC_SURVEY
        j.shape[:] = [int(s) for s in _lib.int3(shape)]
        j.cell = float(cell)
        j.posmin[:] = [float(p) for p in _lib.dbl3(posmin)]
        j.scheme, j.window = int(scheme), int(window)
        j.rmax, j.dr, j.kmax, j.dk = float(rmax), float(dr), float(kmax), float(dk)
        j.maxell = int(maxell)
        j.precision = _PRECISIONS[precision]
        j.want_rr = 1 if want_rr else 0
        j.data, self._keep_d = data
        if randoms is not None:
            j.randoms, self._keep_r = randoms
        else:
            self._keep_r = None
        self.job = j
        self.kind = kind

    @property
    def footprint(self):
        b = ctypes.c_size_t()
        _lib.call("fc_job_footprint", ctypes.byref(self.job), ctypes.byref(b))
        return b.value


class Server:
    def __init__(self, hbm_budget, slots=2, max_bypass=8):
        self._handle = None
        h = ctypes.c_void_p()
        _lib.call("fc_server_create", int(hbm_budget), int(slots), int(max_bypass),
                  ctypes.byref(h))
        self._handle = h
        self._specs = {}

    def close(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            _lib.load().fc_server_destroy(h)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, spec):
        t = ctypes.c_uint64()
        _lib.call("fc_server_submit", self._handle, ctypes.byref(spec.job),
                  ctypes.byref(t))
        self._specs[t.value] = spec  # keeps host catalogs alive
        return t.value

    def wait(self, ticket, timeout=None):
        """True when the job has finished; False when `timeout` seconds ran
        out first."""
        done = ctypes.c_int()
        rc = _lib.load().fc_server_wait(self._handle, int(ticket),
                                        -1.0 if timeout is None else float(timeout),
                                        ctypes.byref(done))
        if rc == _lib.FC_ERR_TIMEOUT:
            return False
        _lib.check(rc)
        return bool(done.value)

    def info(self, ticket):
        i = _lib.JobInfo()
        _lib.call("fc_server_job_info", self._handle, int(ticket), ctypes.byref(i))
        out = {name: getattr(i, name) for name, _ in i._fields_
               if name not in ("data", "randoms", "message", "phase_s")}
        out["phase_s"] = dict(zip(("data_catalog", "data_assign", "random_catalog",
                                   "random_assign", "combine", "correlate_nn",
                                   "correlate_rr", "build"), list(i.phase_s)))
        out["message"] = i.message.decode("utf-8", "replace")
        out["data_totw"] = i.data.totw
        out["data_added"] = i.data.num_added
        out["randoms_totw"] = i.randoms.totw
        return out

    def results(self, ticket, which=0):
        """Raw outputs (as Correlator.results()); which 0 = NN, 1 = RR."""
        inf = self.info(ticket)
        nrows, nr, nk = inf["nrows"], inf["nr"], inf["nk"]
        rb, kb = np.zeros(nr), np.zeros(nk)
        rc = np.zeros((nrows, nr), dtype=np.intc)
        kc = np.zeros((nrows, nk), dtype=np.intc)
        rh, kh = np.zeros((nrows, nr)), np.zeros((nrows, nk))
        zl = ctypes.c_double()
        _lib.call("fc_server_job_results", self._handle, int(ticket), int(which),
                  _lib.dptr(rb), _lib.iptr(rc), _lib.dptr(rh), _lib.dptr(kb),
                  _lib.iptr(kc), _lib.dptr(kh), ctypes.byref(zl))
        return {"rbins": rb, "rcounts": rc, "rhist": rh, "kbins": kb,
                "kcounts": kc, "khist": kh, "zerolag": zl.value}

    def tables(self, ticket, which=0, squeeze=True):
        res = self.results(ticket, which)
        return (BaseCorrelator._power_spectrum(None, res, squeeze),
                BaseCorrelator._correlation(None, res, squeeze))

    def release(self, ticket):
        _lib.call("fc_server_release", self._handle, int(ticket))
        self._specs.pop(ticket, None)

    def stats(self):
        s = _lib.ServerStats()
        _lib.call("fc_server_stats", self._handle, ctypes.byref(s))
        return {name: getattr(s, name) for name, _ in s._fields_}
