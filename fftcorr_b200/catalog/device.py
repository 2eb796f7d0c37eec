"""Synthetic catalogs generated in device memory (fc_catalog_* in
include/fc_api.h): counter-based Philox4x32-10 streams keyed by a seed, so a
catalog is reproducible and independent of how it is batched.  The rows are
(x, y, z, w) FP64, ready for MassAssignor.add_particles_device or a batch.
"""
import ctypes

import numpy as np

from fftcorr_b200 import _lib


class DeviceCatalog:
    """An (n, 4) FP64 particle array owned in device memory."""

    def __init__(self, n):
        self.n = int(n)
        if self.n < 0:
            raise ValueError("n must be >= 0")
        p = ctypes.c_void_p()
        _lib.call("fc_device_malloc", max(1, self.n) * 32, ctypes.byref(p))
        self.ptr = p.value

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr:
            try:
                _lib.call("fc_device_free", ctypes.c_void_p(ptr))
            except Exception:
                pass
            self.ptr = None

    def to_host(self):
        """Copies the rows back (for tests and small catalogs)."""
        out = np.empty((self.n, 4), dtype=np.float64)
        if self.n:
            _lib.call("fc_memcpy_dtoh", out.ctypes.data_as(ctypes.c_void_p),
                      ctypes.c_void_p(self.ptr), out.nbytes)
        return out


def uniform(n, lo, hi, seed, wmin=1.0, wmax=1.0):
    cat = DeviceCatalog(n)
    _lib.call("fc_catalog_uniform", ctypes.c_void_p(cat.ptr), cat.n,
              _lib.dptr(_lib.dbl3(lo)), _lib.dptr(_lib.dbl3(hi)), float(wmin),
              float(wmax), int(seed))
    return cat


def clustered_box(n, boxsize, seed, ncentres=10000, sigma=5.0, wmin=1.0,
                  wmax=1.0):
    cat = DeviceCatalog(n)
    _lib.call("fc_catalog_clustered_box", ctypes.c_void_p(cat.ptr), cat.n,
              float(boxsize), int(ncentres), float(sigma), float(wmin),
              float(wmax), int(seed))
    return cat


def sector(n, seed, rmin=500.0, rmax=1500.0, ra_deg=30.0, dec_deg=30.0,
           wmin=0.5, wmax=1.5, wsign=1.0):
    cat = DeviceCatalog(n)
    _lib.call("fc_catalog_sector", ctypes.c_void_p(cat.ptr), cat.n, float(rmin),
              float(rmax), np.deg2rad(ra_deg), np.deg2rad(dec_deg), float(wmin),
              float(wmax), float(wsign), int(seed))
    return cat
