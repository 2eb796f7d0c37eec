/* fftw3.h -- the three wisdom functions fftcorr/fftw/fftw.pxd binds,
 * mapped onto this library's persisted launch-tuning table (the analogue
 * of FFTW wisdom for the hand-written passes; fc_tune_* in fc_api.h).
 * Return values follow FFTW: nonzero on success. */
#ifndef FFTCORR_CC_FFTW3_H
#define FFTCORR_CC_FFTW3_H

#include "../../fc_api.h"

static inline int fftw_export_wisdom_to_filename(const char *filename) {
  return fc_tune_export(filename) == FC_OK;
}
static inline int fftw_import_wisdom_from_filename(const char *filename) {
  return fc_tune_import(filename) == FC_OK;
}
static inline void fftw_forget_wisdom(void) { fc_tune_forget(); }

#endif /* FFTCORR_CC_FFTW3_H */
