"""HistogramList with counts and sums accumulated on the GPU.

Mirrors fftcorr/histogram/histogram_list.pyx:9-44 over the C ABI's fc_hist
(cc/histogram/histogram_list.h:10-68).  ``bins``, ``counts`` and
``hist_values`` are read-only numpy arrays that are refreshed in place after
every accumulate/reset, so references taken earlier stay current, like the
reference's views of C++ memory.
"""
import ctypes

import numpy as np

from fftcorr_b200 import _lib
from fftcorr_b200.array_checks import as_row_major


def _readonly(a):
    a.setflags(write=False)
    return a


class HistogramList:
    def __init__(self, n, minval, maxval, binsize):
        self._handle = None
        h = ctypes.c_void_p()
        _lib.call("fc_hist_create", int(n), float(minval), float(maxval),
                  float(binsize), ctypes.byref(h))
        self._handle = h
        nb = ctypes.c_int()
        _lib.call("fc_hist_nbins", self._handle, ctypes.byref(nb))
        self._n = int(n)
        self._nbins = nb.value
        self._bins = np.zeros(self._nbins)
        self._counts = np.zeros((self._n, self._nbins), dtype=np.intc)
        self._hist_values = np.zeros((self._n, self._nbins))
        self._refresh()

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().fc_hist_destroy(h)
            except Exception:
                pass
            self._handle = None

    def _refresh(self):
        for a in (self._bins, self._counts, self._hist_values):
            a.setflags(write=True)
        _lib.call("fc_hist_get", self._handle, _lib.dptr(self._bins),
                  _lib.iptr(self._counts), _lib.dptr(self._hist_values))
        for a in (self._bins, self._counts, self._hist_values):
            _readonly(a)

    @property
    def bins(self):
        return self._bins

    @property
    def counts(self):
        return self._counts

    @property
    def hist_values(self):
        return self._hist_values

    def accumulate(self, ih, x, y):
        if x.shape != y.shape:
            raise ValueError("x and y should have the same dimensions")
        x = x.flatten()
        y = y.flatten()
        as_row_major(x, 1)
        as_row_major(y, 1)
        _lib.call("fc_hist_accumulate", self._handle, int(ih), _lib.dptr(x),
                  _lib.dptr(y), x.size)
        self._refresh()

    def reset(self):
        _lib.call("fc_hist_reset", self._handle)
        self._refresh()
