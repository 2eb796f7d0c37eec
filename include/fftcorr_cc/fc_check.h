// fc_check.h -- turns C ABI status codes into the exception types the
// reference's C++ classes throw, so code written against the reference
// (and the Cython `except +` declarations) sees the same error behaviour:
//   FC_ERR_INVALID, FC_ERR_UNSUPPORTED  -> std::invalid_argument
//   FC_ERR_RANGE                        -> std::out_of_range
//   FC_ERR_ALLOC, FC_ERR_ADMISSION      -> std::bad_alloc
//   FC_ERR_STATE                        -> std::logic_error
//   anything else (CUDA, cuFFT, ...)    -> std::runtime_error
// The message is fc_last_error() of the failing call.
#ifndef FFTCORR_CC_FC_CHECK_H
#define FFTCORR_CC_FC_CHECK_H

#include <new>
#include <stdexcept>
#include <string>

#include "../fc_api.h"

namespace fftcorr_cc {

inline void fc_check(int status, const char *what) {
  if (status == FC_OK) return;
  const std::string msg = std::string(what) + ": " + fc_last_error();
  switch (status) {
    case FC_ERR_INVALID:
    case FC_ERR_UNSUPPORTED:
      throw std::invalid_argument(msg);
    case FC_ERR_RANGE:
      throw std::out_of_range(msg);
    case FC_ERR_ALLOC:
    case FC_ERR_ADMISSION:
      throw std::bad_alloc();
    case FC_ERR_STATE:
      throw std::logic_error(msg);
    default:
      throw std::runtime_error(msg);
  }
}

}  // namespace fftcorr_cc

#endif  // FFTCORR_CC_FC_CHECK_H
