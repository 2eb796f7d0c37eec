// array.h -- abstract contiguous array (reference cc/array/array.h:10-17).
// HistogramList::accumulate takes its x and y as Array<Float> views
// (fftcorr/array/array.pxd, fftcorr/histogram/histogram_list.pxd:12).
#ifndef FFTCORR_CC_ARRAY_H
#define FFTCORR_CC_ARRAY_H

#include "../types.h"

template <typename dtype>
class Array {
 public:
  virtual ~Array() = default;
  virtual uint64 size() const = 0;
  virtual dtype *data() = 0;
  virtual const dtype *data() const = 0;
};

#endif  // FFTCORR_CC_ARRAY_H
