"""MassAssignor running on the GPU.

Mirrors fftcorr/particle_mesh/mass_assignor.pyx:17-108 (argument handling,
metadata bookkeeping, properties) over the C ABI's fc_assignor, which
implements cc/particle_mesh/mass_assignor.h:30-234: particles are keyed by
cell, radix-sorted and scattered deterministically into the grid's device
buffer.
"""
import ctypes
import enum

import numpy as np

from fftcorr_b200 import _lib
from fftcorr_b200.array_checks import as_row_major


class DistributionScheme(enum.IntEnum):
    """cc/particle_mesh/distribution_functions.h:11-15, plus trilinear CIC."""
    NEAREST_CELL = 0
    TRIANGULAR_SHAPED_CLOUD = 1
    WAVELET = 2
    CLOUD_IN_CELL = 3


NEAREST_CELL = DistributionScheme.NEAREST_CELL
TRIANGULAR_SHAPED_CLOUD = DistributionScheme.TRIANGULAR_SHAPED_CLOUD
WAVELET = DistributionScheme.WAVELET
CLOUD_IN_CELL = DistributionScheme.CLOUD_IN_CELL


class MassAssignor:
    def __init__(self, grid, distribution_scheme, periodic_wrap=False,
                 buffer_size=0):
        scheme = int(distribution_scheme)
        if ("distribution_scheme" in grid.metadata and
                grid.metadata["distribution_scheme"] != scheme):
            grid.metadata["distribution_scheme"] = -1
        else:
            grid.metadata["distribution_scheme"] = scheme
        self._grid = grid  # kept alive for the assignor's lifetime
        self._handle = None
        h = ctypes.c_void_p()
        _lib.call("fc_assignor_create", grid.handle, scheme,
                  int(bool(periodic_wrap)), int(buffer_size), ctypes.byref(h))
        self._handle = h

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().fc_assignor_destroy(h)
            except Exception:
                pass
            self._handle = None

    @property
    def buffer_size(self):
        v = ctypes.c_int64()
        _lib.call("fc_assignor_buffer_size", self._handle, ctypes.byref(v))
        return v.value

    def clear(self):
        _lib.call("fc_assignor_clear", self._handle)

    def add_particles(self, particles, weight=None):
        self.add_particles_to_buffer(particles, weight)
        self.flush()

    def add_particles_to_buffer(self, particles, weight=None):
        as_row_major(particles, 2)
        g = self._grid
        if particles.shape[1] == 4:
            if weight is not None:
                raise ValueError("Cannot pass weights twice")
            g._before_device()
            _lib.call("fc_assignor_add_posw", self._handle, _lib.dptr(particles),
                      particles.shape[0])
            g._after_device()
            return
        if particles.shape[1] != 3:
            raise ValueError(
                "Particles must have shape (n, 3) or (n, 4). "
                f"Got: {particles.shape}")
        if weight is None:
            weight = 1.0
        weight = np.asarray(weight)
        if not weight.shape:
            g._before_device()
            _lib.call("fc_assignor_add_pos_weight", self._handle,
                      _lib.dptr(particles), float(weight), particles.shape[0])
            g._after_device()
            return
        if weight.shape != (particles.shape[0],):
            raise ValueError(
                "Weight must be 1D with the same length as particles. "
                f"Got {weight.shape} and {particles.shape}")
        as_row_major(weight, 1)
        g._before_device()
        _lib.call("fc_assignor_add_pos_weights", self._handle, _lib.dptr(particles),
                  _lib.dptr(weight), particles.shape[0])
        g._after_device()

    def add_particles_device(self, posw_device_ptr, n):
        """Assigns n particles whose (n, 4) posw array is in device memory."""
        self._grid._before_device()
        _lib.call("fc_assignor_add_posw_device", self._handle,
                  ctypes.c_void_p(posw_device_ptr), int(n))
        self._grid._after_device()

    def flush(self):
        self._grid._before_device()
        _lib.call("fc_assignor_flush", self._handle)
        self._grid._after_device()

    def _stats(self):
        s = _lib.AssignStats()
        _lib.call("fc_assignor_stats", self._handle, ctypes.byref(s))
        return s

    @property
    def num_added(self):
        return int(self._stats().num_added)

    @property
    def num_skipped(self):
        return int(self._stats().num_skipped)

    @property
    def totw(self):
        return self._stats().totw

    @property
    def totwsq(self):
        return self._stats().totwsq

    @property
    def sort_time(self):
        return self._stats().sort_time

    @property
    def window_time(self):
        return self._stats().window_time
