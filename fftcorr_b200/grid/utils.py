"""apply_displacement_field (fftcorr/grid/utils.pyx:21-55) on the GPU.

out[i] = pos[i] + disp[cell of pos[i]] where the cell is that of
ConfigSpaceGrid.get_grid_coords (with periodic wrap when asked), truncated
to integers; a position with no cell raises the reference's ValueError.
"""
import numpy as np

from fftcorr_b200 import _lib


def apply_displacement_field(grid, pos, disp, periodic_wrap=False, out=None):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    if pos.ndim != 2 or pos.shape[1] != 3:
        raise ValueError("pos must have shape (n, 3)")
    disp = np.ascontiguousarray(disp, dtype=np.float64)
    if disp.shape != tuple(grid.shape) + (3,):
        raise ValueError(f"disp must have shape {tuple(grid.shape) + (3,)}")
    res = np.empty_like(pos)
    try:
        _lib.call("fc_apply_displacement", grid.handle, _lib.dptr(pos),
                  pos.shape[0], _lib.dptr(disp), 1 if periodic_wrap else 0,
                  _lib.dptr(res))
    except ValueError:
        raise ValueError(
            "Failed to apply displacement field: coordinates out of bounds? "
            "Try setting periodic_wrap=True.") from None
    if out is None:
        return res
    out[...] = res
    return out
