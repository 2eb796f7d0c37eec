"""numpy -> C array checks with the reference adaptor's rules and messages.

Mirrors as_RowMajorArrayPtr in fftcorr/array/numpy_adaptor.h:45-72: the array
must have the expected number of dimensions, dtype float64, be C-contiguous
and writeable, else RuntimeError.
"""
import numpy as np


def as_row_major(arr, ndim, dtype=np.float64):
    if not isinstance(arr, np.ndarray):
        raise RuntimeError("Expected a numpy array.")
    if arr.ndim != ndim:
        raise RuntimeError("Number of dimensions of numpy array is not equal to N.")
    if arr.dtype != np.dtype(dtype):
        raise RuntimeError("Numpy array does not have the expected type.")
    if not arr.flags.c_contiguous:
        raise RuntimeError("Numpy array is not C-contiguous.")
    if not arr.flags.writeable:
        raise RuntimeError("Numpy array is not writeable.")
    return arr
