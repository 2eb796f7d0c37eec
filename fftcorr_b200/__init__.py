"""fftcorr_b200: B200-native (sm_100a) anisotropic correlation function and
power spectrum pipeline (Slepian & Eisenstein Y_lm multipoles), a drop-in for
the fftcorr package's ConfigSpaceGrid / MassAssignor / Correlator /
PeriodicCorrelator / HistogramList API.

The compute runs in the CUDA library libfftcorr_b200.so (C ABI in
include/fc_api.h); this package is the Python face of it.
"""
from fftcorr_b200.correlate import (Correlator, PeriodicCorrelator, compute_xi,
                                    WindowCorrection)
from fftcorr_b200.grid import ConfigSpaceGrid
from fftcorr_b200.histogram import HistogramList
from fftcorr_b200.particle_mesh import DistributionScheme, MassAssignor

__all__ = ["ConfigSpaceGrid", "MassAssignor", "DistributionScheme",
           "Correlator", "PeriodicCorrelator", "compute_xi", "WindowCorrection",
           "HistogramList"]
