from fftcorr_b200.grid.config_space_grid import ConfigSpaceGrid
from fftcorr_b200.grid.utils import apply_displacement_field

__all__ = ["ConfigSpaceGrid", "apply_displacement_field"]
