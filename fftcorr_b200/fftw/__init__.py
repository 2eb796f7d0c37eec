"""FFTW wisdom functions (fftcorr/fftw/fftw.pyx:1-14).

The GPU path plans its transforms with cuFFT when a correlator is created and
keeps the plans for the correlator's lifetime, so there is no wisdom to save.
These keep the reference's signatures: exporting writes a small marker file,
importing succeeds when the file can be read, forgetting does nothing.
"""


def export_wisdom_to_file(filename):
    try:
        with open(filename, "w") as f:
            f.write("(fftcorr_b200: cuFFT plans are kept per correlator)\n")
    except OSError as e:
        raise IOError("Failed to export wisdom file") from e


def import_wisdom_from_file(filename):
    try:
        with open(filename, "r"):
            pass
    except OSError as e:
        raise IOError("Failed to import wisdom file") from e


def forget_wisdom():
    pass
