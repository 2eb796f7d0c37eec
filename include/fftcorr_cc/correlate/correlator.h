// correlator.h -- BaseCorrelator, PeriodicCorrelator and Correlator over
// the B200 library.
//
// Interface of the reference's cc/correlate/correlator.h:18-505 as bound by
// fftcorr/correlate/correlator.pxd:10-66:
//   PeriodicCorrelator(shape, cell_size, window_correct, rmax, dr, kmax, dk,
//                      maxell, fftw_flags)
//   Correlator(shape, cell_size, posmin, window_correct, rmax, dr, kmax, dk,
//              maxell, fftw_flags)
//   set_grid2(grid2), set_grid2_fft(grid2_fft), autocorrelate(grid1),
//   cross_correlate(grid1), cross_correlate(grid1, grid2), zerolag(),
//   correlation_r(), correlation_counts(), correlation_histogram(),
//   power_spectrum_k(), power_spectrum_counts(), power_spectrum_histogram()
// and the WindowCorrection enum of cc/correlate/window_correct.h:8-12.
// Grids are host row-major arrays (N0, N1, N2); grid2_fft is the
// (N0, N1, N2/2+1) complex half spectrum.  The correlation runs on the GPU
// in FP64 (the precision of the reference's Float); fftw_flags is accepted
// and ignored.  The result arrays are host copies refreshed after each
// correlation and are valid until the next one, as in the reference.
#ifndef FFTCORR_CC_CORRELATOR_H
#define FFTCORR_CC_CORRELATOR_H

#include <array>
#include <stdexcept>

#include "../array/row_major_array.h"
#include "../fc_check.h"
#include "../grid/config_space_grid.h"
#include "../histogram/histogram_list.h"
#include "../types.h"

enum WindowCorrection {
  kNoCorrection = 0,
  kTscCorrection = 1,
  kTscAliasedCorrection = 2,
};

class BaseCorrelator {
 public:
  virtual ~BaseCorrelator() { fc_corr_destroy(corr_); }
  BaseCorrelator(const BaseCorrelator &) = delete;
  BaseCorrelator &operator=(const BaseCorrelator &) = delete;

  void set_grid2(const RowMajorArrayPtr<Float, 3> &grid2) {
    check_shape(grid2.shape(), shape_[2], "grid2");
    fftcorr_cc::fc_check(fc_corr_set_grid2(corr_, grid2.data()), "set_grid2");
  }
  void set_grid2_fft(const RowMajorArrayPtr<Complex, 3> &grid2_fft) {
    check_shape(grid2_fft.shape(), shape_[2] / 2 + 1, "grid2_fft");
    fftcorr_cc::fc_check(
        fc_corr_set_grid2_fft(corr_, reinterpret_cast<const double *>(grid2_fft.data())),
        "set_grid2_fft");
  }
  void autocorrelate(const RowMajorArrayPtr<Float, 3> &grid1) {
    check_shape(grid1.shape(), shape_[2], "grid1");
    fftcorr_cc::fc_check(fc_corr_autocorrelate(corr_, grid1.data()),
                         "autocorrelate");
    fetch();
  }
  void cross_correlate(const RowMajorArrayPtr<Float, 3> &grid1) {
    check_shape(grid1.shape(), shape_[2], "grid1");
    fftcorr_cc::fc_check(fc_corr_cross_correlate(corr_, grid1.data()),
                         "cross_correlate");
    fetch();
  }
  void cross_correlate(const RowMajorArrayPtr<Float, 3> &grid1,
                       const RowMajorArrayPtr<Float, 3> &grid2) {
    set_grid2(grid2);
    cross_correlate(grid1);
  }

  Float zerolag() const { return zerolag_; }
  const RowMajorArrayPtr<Float, 1> &correlation_r() const { return rbins_; }
  const RowMajorArrayPtr<int, 2> &correlation_counts() const { return rcounts_; }
  const RowMajorArrayPtr<Float, 2> &correlation_histogram() const { return rhist_; }
  const RowMajorArrayPtr<Float, 1> &power_spectrum_k() const { return kbins_; }
  const RowMajorArrayPtr<int, 2> &power_spectrum_counts() const { return kcounts_; }
  const RowMajorArrayPtr<Float, 2> &power_spectrum_histogram() const {
    return khist_;
  }
  // Device time of the last correlation (the reference's total_time()).
  Float total_time() const {
    fc_corr_timings t;
    fftcorr_cc::fc_check(fc_corr_timings_get(corr_, &t), "timings");
    return t.total_time;
  }

 protected:
  BaseCorrelator(int kind, const std::array<int, 3> &shape, Float cell_size,
                 const Float *posmin, int window_correct, Float rmax, Float dr,
                 Float kmax, Float dk, int maxell, unsigned fftw_flags)
      : shape_(shape) {
    fftcorr_cc::fc_check(
        fc_corr_create(kind, shape.data(), cell_size, posmin, window_correct,
                       rmax, dr, kmax, dk, maxell, fftw_flags, FC_FP64, &corr_),
        kind == FC_SURVEY ? "Correlator" : "PeriodicCorrelator");
    int nrows = 0, nr = 0, nk = 0, rs[3], ks[3];
    fftcorr_cc::fc_check(fc_corr_dims(corr_, &nrows, &nr, &nk, rs, ks),
                         "correlator dims");
    rbins_.allocate({nr});
    rcounts_.allocate({nrows, nr});
    rhist_.allocate({nrows, nr});
    kbins_.allocate({nk});
    kcounts_.allocate({nrows, nk});
    khist_.allocate({nrows, nk});
    fetch();  // bin centres are set at construction, as in the reference
  }

 private:
  void check_shape(const std::array<int, 3> &s, int last, const char *what) {
    if (s[0] != shape_[0] || s[1] != shape_[1] || s[2] != last)
      throw std::invalid_argument(std::string(what) +
                                  " has the wrong shape for this correlator");
  }
  void fetch() {
    fftcorr_cc::fc_check(
        fc_corr_results(corr_, rbins_.data(), rcounts_.data(), rhist_.data(),
                        kbins_.data(), kcounts_.data(), khist_.data(), &zerolag_),
        "correlator results");
  }

  std::array<int, 3> shape_;
  fc_correlator *corr_ = nullptr;
  RowMajorArray<Float, 1> rbins_, kbins_;
  RowMajorArray<int, 2> rcounts_, kcounts_;
  RowMajorArray<Float, 2> rhist_, khist_;
  Float zerolag_ = 0.0;
};

class PeriodicCorrelator : public BaseCorrelator {
 public:
  PeriodicCorrelator(const std::array<int, 3> &shape, Float cell_size,
                     int window_correct, Float rmax, Float dr, Float kmax,
                     Float dk, int maxell, unsigned fftw_flags)
      : BaseCorrelator(FC_PERIODIC, shape, cell_size, nullptr, window_correct,
                       rmax, dr, kmax, dk, maxell, fftw_flags) {}
};

class Correlator : public BaseCorrelator {
 public:
  Correlator(const std::array<int, 3> &shape, Float cell_size,
             const std::array<Float, 3> &posmin, int window_correct, Float rmax,
             Float dr, Float kmax, Float dk, int maxell, unsigned fftw_flags)
      : BaseCorrelator(FC_SURVEY, shape, cell_size, posmin.data(), window_correct,
                       rmax, dr, kmax, dk, maxell, fftw_flags) {}
};

#endif  // FFTCORR_CC_CORRELATOR_H
