from fftcorr_b200.catalog.device import (DeviceCatalog, clustered_box, sector,
                                         uniform)
from fftcorr_b200.catalog.random_catalog import add_random_particles

__all__ = ["DeviceCatalog", "uniform", "clustered_box", "sector",
           "add_random_particles"]
