// types.h -- scalar types of the fftcorr C++ class surface.
//
// Same names and meaning as the reference's cc/types.h:1-16 (Float is the
// grid and histogram type, Complex the FFT element, uint64 sizes), so that
// the Cython declarations (fftcorr/types.pxd) match these headers.
#ifndef FFTCORR_CC_TYPES_H
#define FFTCORR_CC_TYPES_H

#include <complex>

typedef double Float;
typedef std::complex<Float> Complex;
typedef unsigned long long int uint64;

#endif  // FFTCORR_CC_TYPES_H
