// distribution_functions.h -- the mass-assignment scheme enum.
//
// Same enumerators and values as the reference's
// cc/particle_mesh/distribution_functions.h:11-15 (bound by
// fftcorr/particle_mesh/distribution_scheme.pxd as
// DistributionScheme::kNearestCell etc.).  kCloudInCell (trilinear, 2^3
// taps) is an addition of this library.  The stencils themselves run on
// the GPU behind fc_api.h.
#ifndef FFTCORR_CC_DISTRIBUTION_FUNCTIONS_H
#define FFTCORR_CC_DISTRIBUTION_FUNCTIONS_H

#include "../types.h"

enum DistributionScheme {
  kNearestCell = 0,
  kTriangularShapedCloud = 1,
  kWavelet = 2,
  kCloudInCell = 3,
};

#endif  // FFTCORR_CC_DISTRIBUTION_FUNCTIONS_H
