// histogram_list.h -- HistogramList over the B200 library.
//
// Interface of the reference's cc/histogram/histogram_list.h:10-68 as bound
// by fftcorr/histogram/histogram_list.pxd:5-13:
//   HistogramList(int n, Float minval, Float maxval, Float binsize)
//   nbins(), bins(), counts(), hist_values(),
//   accumulate(int ih, const Array<Float> &x, const Array<Float> &y), reset()
// n rows of floor((maxval - minval) / binsize) bins with midpoints
// minval + (i + 1/2) binsize; accumulate adds each y to the bin of its x in
// row ih (exact integer counts, FP64 sums in a fixed order) on the GPU.  The
// returned arrays are host copies refreshed after every accumulate/reset.
#ifndef FFTCORR_CC_HISTOGRAM_LIST_H
#define FFTCORR_CC_HISTOGRAM_LIST_H

#include <stdexcept>

#include "../array/array.h"
#include "../array/row_major_array.h"
#include "../fc_check.h"
#include "../types.h"

class HistogramList {
 public:
  HistogramList(int n, Float minval, Float maxval, Float binsize) : n_(n) {
    fftcorr_cc::fc_check(fc_hist_create(n, minval, maxval, binsize, &h_),
                         "HistogramList");
    fftcorr_cc::fc_check(fc_hist_nbins(h_, &nbins_), "HistogramList");
    bins_.allocate({nbins_});
    counts_.allocate({n_, nbins_});
    hist_.allocate({n_, nbins_});
    fetch();
  }
  ~HistogramList() { fc_hist_destroy(h_); }
  HistogramList(const HistogramList &) = delete;
  HistogramList &operator=(const HistogramList &) = delete;

  int nbins() const { return nbins_; }
  const RowMajorArrayPtr<Float, 1> &bins() const { return bins_; }
  const RowMajorArrayPtr<int, 2> &counts() const { return counts_; }
  const RowMajorArrayPtr<Float, 2> &hist_values() const { return hist_; }

  void accumulate(int ih, const Array<Float> &x, const Array<Float> &y) {
    if (x.size() != y.size())
      throw std::invalid_argument("x and y must have the same size");
    fftcorr_cc::fc_check(
        fc_hist_accumulate(h_, ih, x.data(), y.data(), (int64_t)x.size()),
        "HistogramList::accumulate");
    fetch();
  }
  void reset() {
    fftcorr_cc::fc_check(fc_hist_reset(h_), "HistogramList::reset");
    fetch();
  }

 private:
  void fetch() {
    fftcorr_cc::fc_check(fc_hist_get(h_, bins_.data(), counts_.data(), hist_.data()),
                         "HistogramList");
  }

  int n_;
  int nbins_ = 0;
  fc_hist *h_ = nullptr;
  RowMajorArray<Float, 1> bins_;
  RowMajorArray<int, 2> counts_;
  RowMajorArray<Float, 2> hist_;
};

#endif  // FFTCORR_CC_HISTOGRAM_LIST_H
