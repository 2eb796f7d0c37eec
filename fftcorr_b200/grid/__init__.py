from fftcorr_b200.grid.config_space_grid import ConfigSpaceGrid

__all__ = ["ConfigSpaceGrid"]
