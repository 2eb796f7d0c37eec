"""Batched form: many periodic boxes in one captured CUDA graph.

Each box goes through what a single-box script does with the reference's
API -- MassAssignor(grid, scheme, periodic_wrap=True) on its particles, the
CLI's periodic normalisation (cc/fftcorr.cc:369-375: subtract the mean cell
density, divide by it), PeriodicCorrelator.autocorrelate
(cc/correlate/correlator.h:273-357) -- but the whole batch is enqueued once
on several streams, captured into a CUDA graph and replayed with one launch.
The histograms of every box are reduced by one persistent kernel at the end.
Results per box are the same bits as the single-box path in the same
precision (fc_batch_* in include/fc_api.h).

Launch shapes, the stream count and the histogram CTA count come from the
library's tuning table, filled by timing candidates on first use; it can be
saved and restored with fftcorr_b200.fftw.export_wisdom_to_file /
import_wisdom_from_file.
"""
import ctypes

import numpy as np

from fftcorr_b200 import _lib
from fftcorr_b200.correlate.correlator import (NO_CORRECTION, _PRECISIONS,
                                               BaseCorrelator)
from fftcorr_b200.particle_mesh import DistributionScheme


class _Box:
    def __init__(self, shape, cell_size, particles):
        from fftcorr_b200.catalog.device import DeviceCatalog
        self.shape = tuple(int(s) for s in _lib.int3(shape))
        self.cell_size = float(cell_size)
        if isinstance(particles, DeviceCatalog):
            self.catalog = particles
        else:
            p = np.ascontiguousarray(particles, dtype=np.float64)
            if p.ndim != 2 or p.shape[1] != 4:
                raise ValueError("particles must be (n, 4) x, y, z, w")
            self.catalog = DeviceCatalog(p.shape[0])
            if p.shape[0]:
                _lib.call("fc_memcpy_htod", ctypes.c_void_p(self.catalog.ptr),
                          p.ctypes.data_as(ctypes.c_void_p), p.nbytes)


class PeriodicBatch:
    """boxes: sequence of (shape, cell_size, particles), particles an (n, 4)
    FP64 array (uploaded once and kept on the device) or a DeviceCatalog
    (used in place; it must outlive the batch)."""

    def __init__(self, boxes, distribution_scheme=DistributionScheme.CLOUD_IN_CELL,
                 rmax=200.0, dr=5.0, kmax=0.1, dk=0.005, maxell=2,
                 window_correct=NO_CORRECTION, precision="fp32", lanes=0,
                 tune=True):
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be 'fp64' or 'fp32', got {precision!r}")
        self._handle = None
        self._boxes = [_Box(*b) for b in boxes]
        if not self._boxes:
            raise ValueError("a batch needs at least one box")
        arr = (_lib.BatchBox * len(self._boxes))()
        for i, b in enumerate(self._boxes):
            arr[i].shape[:] = list(b.shape)
            arr[i].cell_size = b.cell_size
            arr[i].posw_device = b.catalog.ptr
            arr[i].n = b.catalog.n
        prm = _lib.BatchParams()
        _lib.call("fc_batch_params_default", ctypes.byref(prm))
        prm.scheme = int(distribution_scheme)
        prm.window = int(window_correct)
        prm.rmax, prm.dr, prm.kmax, prm.dk = float(rmax), float(dr), float(kmax), float(dk)
        prm.maxell = int(maxell)
        prm.precision = _PRECISIONS[precision]
        prm.lanes = int(lanes)
        prm.tune = 1 if tune else 0
        h = ctypes.c_void_p()
        _lib.call("fc_batch_create", arr, len(self._boxes), ctypes.byref(prm),
                  ctypes.byref(h))
        self._handle = h
        self.last_seconds = None

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().fc_batch_destroy(h)
            except Exception:
                pass
            self._handle = None

    def __len__(self):
        return len(self._boxes)

    def run(self):
        """Replays the graph and waits; returns its device time in seconds."""
        s = ctypes.c_double()
        _lib.call("fc_batch_run", self._handle, ctypes.byref(s))
        self.last_seconds = s.value
        return s.value

    def launch(self):
        _lib.call("fc_batch_launch", self._handle)

    def wait(self):
        s = ctypes.c_double()
        _lib.call("fc_batch_wait", self._handle, ctypes.byref(s))
        self.last_seconds = s.value
        return s.value

    @property
    def info(self):
        i = _lib.BatchInfo()
        _lib.call("fc_batch_info", self._handle, ctypes.byref(i))
        return {name: getattr(i, name) for name, _ in i._fields_}

    def results(self, box):
        """Raw outputs of one box, as Correlator.results()."""
        nrows, nr, nk = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.call("fc_batch_box_dims", self._handle, int(box), ctypes.byref(nrows),
                  ctypes.byref(nr), ctypes.byref(nk))
        nrows, nr, nk = nrows.value, nr.value, nk.value
        rb, kb = np.zeros(nr), np.zeros(nk)
        rc = np.zeros((nrows, nr), dtype=np.intc)
        kc = np.zeros((nrows, nk), dtype=np.intc)
        rh, kh = np.zeros((nrows, nr)), np.zeros((nrows, nk))
        zl = ctypes.c_double()
        _lib.call("fc_batch_results", self._handle, int(box), _lib.dptr(rb),
                  _lib.iptr(rc), _lib.dptr(rh), _lib.dptr(kb), _lib.iptr(kc),
                  _lib.dptr(kh), ctypes.byref(zl))
        return {"rbins": rb, "rcounts": rc, "rhist": rh, "kbins": kb,
                "kcounts": kc, "khist": kh, "zerolag": zl.value}

    def tables(self, box, squeeze=True):
        """(ps_table, xi_table) of one box, as PeriodicCorrelator returns."""
        res = self.results(box)
        return (BaseCorrelator._power_spectrum(None, res, squeeze),
                BaseCorrelator._correlation(None, res, squeeze))

    def stats(self, box):
        s = _lib.AssignStats()
        _lib.call("fc_batch_box_stats", self._handle, int(box), ctypes.byref(s))
        return {"num_added": s.num_added, "num_skipped": s.num_skipped,
                "totw": s.totw, "totwsq": s.totwsq}
