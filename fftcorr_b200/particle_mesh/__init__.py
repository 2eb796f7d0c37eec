from fftcorr_b200.particle_mesh.mass_assignor import (
    CLOUD_IN_CELL, NEAREST_CELL, TRIANGULAR_SHAPED_CLOUD, WAVELET,
    DistributionScheme, MassAssignor)

__all__ = ["MassAssignor", "DistributionScheme", "NEAREST_CELL",
           "TRIANGULAR_SHAPED_CLOUD", "WAVELET", "CLOUD_IN_CELL"]
