"""FFTW wisdom functions (fftcorr/fftw/fftw.pyx:1-14).

The reference saves and loads FFTW's planner wisdom so later runs skip the
planner.  The GPU library's counterpart is its launch-tuning table: the
thread and wave counts, lane count and histogram CTA count that the batched
form's autotuner measured for each grid size.  These functions keep the
reference's signatures and errors and move that table to and from a text
file.  A file written by FFTW itself (it starts with "(fftw-") is accepted
by import and contributes nothing.
"""
from fftcorr_b200 import _lib


def export_wisdom_to_file(filename):
    try:
        _lib.call("fc_tune_export", str(filename).encode())
    except ValueError as e:
        raise IOError("Failed to export wisdom file") from e


def import_wisdom_from_file(filename):
    try:
        with open(filename, "r") as f:
            head = f.read(6)
    except OSError as e:
        raise IOError("Failed to import wisdom file") from e
    if head.startswith("(fftw"):
        return
    try:
        _lib.call("fc_tune_import", str(filename).encode())
    except ValueError as e:
        raise IOError("Failed to import wisdom file") from e


def forget_wisdom():
    _lib.call("fc_tune_forget")


def wisdom_entries():
    """Number of entries in the launch-tuning table."""
    import ctypes
    n = ctypes.c_int()
    _lib.call("fc_tune_count", ctypes.byref(n))
    return n.value
