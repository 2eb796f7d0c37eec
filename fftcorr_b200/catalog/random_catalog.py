"""add_random_particles (fftcorr/catalog/random_catalog.py:8-87) with the
random positions drawn on the GPU.

Same signature, argument checks and counters as the reference: n points
uniform over the grid's [posmin, posmax) box, weight particle_weight (or
total_weight / n), optionally moved by a displacement field, assigned with
the given window and periodic wrap.  The positions come from the library's
Philox4x32-10 generator keyed by seed instead of numpy's PCG64, so they are
never copied from the host; the catalog matches the reference's in
distribution, not value by value, and does not depend on batch_size.
"""
import logging

import numpy as np

from fftcorr_b200 import _lib
from fftcorr_b200.particle_mesh import MassAssignor


def add_random_particles(n, grid, window_type, particle_weight=None,
                         total_weight=None, periodic_wrap=False, disp=None,
                         seed=None, batch_size=int(1e8), buffer_size=int(1e7)):
    if total_weight is not None:
        if particle_weight is not None:
            raise ValueError(
                "particle_weight and total_weight cannot both be set")
        particle_weight = total_weight / n
    if particle_weight is None:
        particle_weight = 1.0
    logging.info(f"Particle weight: {particle_weight:.6g}")
    dptr = None
    if disp is not None:
        disp = np.ascontiguousarray(disp, dtype=np.float64)
        if disp.shape != tuple(grid.shape) + (3,):
            raise ValueError(f"disp must have shape {tuple(grid.shape) + (3,)}")
        dptr = _lib.dptr(disp)
    if seed is None:
        seed = int(np.random.default_rng().integers(0, 2**63))
    ma = MassAssignor(grid, window_type, periodic_wrap, buffer_size)
    grid._before_device()
    _lib.call("fc_assignor_add_random", ma._handle, int(n), float(particle_weight),
              dptr, int(seed) & (2**64 - 1), int(batch_size))
    ma.flush()
    grid._after_device()
    assert ma.num_added + ma.num_skipped == n
    logging.info(f"Added {ma.num_added:,} randoms ({ma.num_skipped:,} skipped). "
                 f"Total weight: {ma.totw:.4g}")
    return ma
