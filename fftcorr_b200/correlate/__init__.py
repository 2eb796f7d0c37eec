from fftcorr_b200.correlate.correlator import (
    NO_CORRECTION, TSC_ALIASED_CORRECTION, TSC_CORRECTION, BaseCorrelator,
    Correlator, PeriodicCorrelator, WindowCorrection)
from fftcorr_b200.correlate.utils import compute_xi

__all__ = ["Correlator", "PeriodicCorrelator", "BaseCorrelator", "compute_xi",
           "WindowCorrection", "NO_CORRECTION", "TSC_CORRECTION",
           "TSC_ALIASED_CORRECTION"]
