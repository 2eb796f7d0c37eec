from fftcorr_b200.histogram.histogram_list import HistogramList

__all__ = ["HistogramList"]
