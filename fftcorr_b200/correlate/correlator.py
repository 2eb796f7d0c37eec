"""PeriodicCorrelator and Correlator running on the GPU.

Mirrors fftcorr/correlate/correlator.pyx:12-183 (constructors,
from_grid_spec, autocorrelate / cross_correlate / set_grid2 / set_grid2_fft
and the (power spectrum, correlation) tables) over the C ABI's
fc_correlator, which implements cc/correlate/correlator.h:18-505.

Extensions beyond the reference: a ``precision`` keyword ("fp64", the
reference's arithmetic, or "fp32" for FP32 grids and FFTs with FP64
coordinates, Y_lm normalisation and histograms); grids may be passed as
device-resident ConfigSpaceGrid objects, which avoids any host transfer; and
``zerolag`` (cc/correlate/correlator.h:80) is exposed.
"""
import ctypes
import enum

import numpy as np

from fftcorr_b200 import _lib
from fftcorr_b200.table import make_table


class WindowCorrection(enum.IntEnum):
    """cc/correlate/window_correct.h:8-12."""
    NO_CORRECTION = 0
    TSC_CORRECTION = 1
    TSC_ALIASED_CORRECTION = 2


NO_CORRECTION = WindowCorrection.NO_CORRECTION
TSC_CORRECTION = WindowCorrection.TSC_CORRECTION
TSC_ALIASED_CORRECTION = WindowCorrection.TSC_ALIASED_CORRECTION

_PRECISIONS = {"fp64": _lib.FC_FP64, "fp32": _lib.FC_FP32_MIXED,
               _lib.FC_FP64: _lib.FC_FP64, _lib.FC_FP32_MIXED: _lib.FC_FP32_MIXED}


def _is_grid(obj):
    return hasattr(obj, "handle") and hasattr(obj, "_before_device")


class BaseCorrelator:
    _kind = None

    def _create(self, shape, cell_size, posmin, window_correct, rmax, dr, kmax,
                dk, maxell, fftw_flags, precision):
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be 'fp64' or 'fp32', got {precision!r}")
        self._handle = None
        shape = _lib.int3(shape)
        pm = _lib.dbl3(posmin if posmin is not None else (0.0, 0.0, 0.0))
        h = ctypes.c_void_p()
        _lib.call("fc_corr_create", self._kind, _lib.iptr(shape), float(cell_size),
                  _lib.dptr(pm), int(window_correct), float(rmax), float(dr),
                  float(kmax), float(dk), int(maxell), int(fftw_flags),
                  _PRECISIONS[precision], ctypes.byref(h))
        self._handle = h
        self._shape = tuple(int(s) for s in shape)
        nrows, nr, nk = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        rs = np.zeros(3, dtype=np.intc)
        ks = np.zeros(3, dtype=np.intc)
        _lib.call("fc_corr_dims", self._handle, ctypes.byref(nrows), ctypes.byref(nr),
                  ctypes.byref(nk), _lib.iptr(rs), _lib.iptr(ks))
        self._nrows, self._nr, self._nk = nrows.value, nr.value, nk.value
        self.rshape = tuple(rs)
        self.kshape = tuple(ks)
        self.precision = "fp64" if _PRECISIONS[precision] == _lib.FC_FP64 else "fp32"

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().fc_corr_destroy(h)
            except Exception:
                pass
            self._handle = None

    @property
    def handle(self):
        return self._handle

    # ----------------------------------------------------------- results
    def results(self):
        """Raw outputs: dict of rbins, rcounts, rhist, kbins, kcounts, khist,
        zerolag (the C++ accessors of correlator.h:80-95)."""
        rb = np.zeros(self._nr)
        rc = np.zeros((self._nrows, self._nr), dtype=np.intc)
        rh = np.zeros((self._nrows, self._nr))
        kb = np.zeros(self._nk)
        kc = np.zeros((self._nrows, self._nk), dtype=np.intc)
        kh = np.zeros((self._nrows, self._nk))
        zl = ctypes.c_double()
        _lib.call("fc_corr_results", self._handle, _lib.dptr(rb), _lib.iptr(rc),
                  _lib.dptr(rh), _lib.dptr(kb), _lib.iptr(kc), _lib.dptr(kh),
                  ctypes.byref(zl))
        return {"rbins": rb, "rcounts": rc, "rhist": rh, "kbins": kb,
                "kcounts": kc, "khist": kh, "zerolag": zl.value}

    @property
    def zerolag(self):
        return self.results()["zerolag"]

    def timings(self):
        t = _lib.CorrTimings()
        _lib.call("fc_corr_timings_get", self._handle, ctypes.byref(t))
        return {name: getattr(t, name) for name, _ in t._fields_}

    def _correlation(self, res, squeeze=True):
        r = res["rbins"]
        histogram = res["rhist"]
        counts = res["rcounts"]
        with np.errstate(divide="ignore", invalid="ignore"):
            xi = histogram / counts
        if squeeze:
            xi = np.squeeze(xi)
            histogram = np.squeeze(histogram)
        return make_table((r, np.transpose(xi), np.transpose(histogram), counts[0, :]),
                          ("r", "xi", "histogram", "count"))

    def _power_spectrum(self, res, squeeze=True):
        k = res["kbins"]
        histogram = res["khist"]
        counts = res["kcounts"]
        with np.errstate(divide="ignore", invalid="ignore"):
            ps = histogram / counts
        if squeeze:
            ps = np.squeeze(ps)
            histogram = np.squeeze(histogram)
        return make_table((k, np.transpose(ps), np.transpose(histogram), counts[0, :]),
                          ("k", "ps", "histogram", "count"))

    def _tables(self, squeeze):
        res = self.results()
        return self._power_spectrum(res, squeeze), self._correlation(res, squeeze)

    def set_term_shard(self, rank, world):
        """Compute only the (ell, m) terms i with i % world == rank (survey
        correlators); see fftcorr_b200.correlate.sharded."""
        _lib.call("fc_corr_set_term_shard", self._handle, int(rank), int(world))

    # -------------------------------------------------------------- inputs
    def _host_grid(self, grid):
        grid = np.ascontiguousarray(grid, dtype=np.float64)
        if grid.shape != self._shape:
            raise ValueError(f"grid shape {grid.shape} does not match {self._shape}")
        return grid

    def set_grid2(self, grid2):
        if _is_grid(grid2):
            grid2._before_device()
            _lib.call("fc_corr_set_grid2_grid", self._handle, grid2.handle)
            return
        g = self._host_grid(grid2)
        _lib.call("fc_corr_set_grid2", self._handle, _lib.dptr(g))

    def set_grid2_fft(self, grid2_fft):
        g = np.ascontiguousarray(grid2_fft, dtype=np.complex128)
        want = (self._shape[0], self._shape[1], self._shape[2] // 2 + 1)
        if g.shape != want:
            raise ValueError(f"grid2_fft shape {g.shape} does not match {want}")
        _lib.call("fc_corr_set_grid2_fft", self._handle,
                  g.view(np.float64).ctypes.data_as(_lib.c_double_p))

    def autocorrelate(self, grid, squeeze=True):
        if _is_grid(grid):
            grid._before_device()
            _lib.call("fc_corr_autocorrelate_grid", self._handle, grid.handle)
        else:
            g = self._host_grid(grid)
            _lib.call("fc_corr_autocorrelate", self._handle, _lib.dptr(g))
        return self._tables(squeeze)

    def cross_correlate(self, grid1, grid2=None, squeeze=True):
        if grid2 is not None:
            self.set_grid2(grid2)
        if _is_grid(grid1):
            grid1._before_device()
            _lib.call("fc_corr_cross_correlate_grid", self._handle, grid1.handle)
        else:
            g = self._host_grid(grid1)
            _lib.call("fc_corr_cross_correlate", self._handle, _lib.dptr(g))
        return self._tables(squeeze)


class PeriodicCorrelator(BaseCorrelator):
    _kind = _lib.FC_PERIODIC

    def __init__(self, shape, cell_size, window_correct, rmax, dr, kmax, dk,
                 maxell, fftw_flags=0, precision="fp64"):
        self._create(shape, cell_size, None, window_correct, rmax, dr, kmax, dk,
                     maxell, fftw_flags, precision)

    @classmethod
    def from_grid_spec(cls, grid, rmax, dr, kmax, dk, maxell,
                       window_correct=NO_CORRECTION, fftw_flags=0,
                       precision="fp64"):
        return cls(shape=grid.shape, cell_size=grid.cell_size,
                   window_correct=window_correct, rmax=rmax, dr=dr, kmax=kmax,
                   dk=dk, maxell=maxell, fftw_flags=fftw_flags,
                   precision=precision)


class Correlator(BaseCorrelator):
    _kind = _lib.FC_SURVEY

    def __init__(self, shape, cell_size, posmin, window_correct, rmax, dr, kmax,
                 dk, maxell, fftw_flags=0, precision="fp64"):
        self._create(shape, cell_size, posmin, window_correct, rmax, dr, kmax, dk,
                     maxell, fftw_flags, precision)

    @classmethod
    def from_grid_spec(cls, grid, rmax, dr, kmax, dk, maxell,
                       window_correct=NO_CORRECTION, fftw_flags=0,
                       precision="fp64"):
        return cls(shape=grid.shape, cell_size=grid.cell_size,
                   posmin=grid.posmin, window_correct=window_correct, rmax=rmax,
                   dr=dr, kmax=kmax, dk=dk, maxell=maxell, fftw_flags=fftw_flags,
                   precision=precision)


def footprint_bytes(kind, shape, cell_size, rmax, kmax, maxell, precision="fp64"):
    """Device bytes a correlator of this configuration holds."""
    out = ctypes.c_size_t()
    _lib.call("fc_corr_footprint", int(kind), _lib.iptr(_lib.int3(shape)),
              float(cell_size), float(rmax), float(kmax), int(maxell),
              _PRECISIONS[precision], ctypes.byref(out))
    return out.value
