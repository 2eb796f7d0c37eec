// ref_harness.cc -- C-callable entry points into the UNMODIFIED reference
// fftcorr C++ classes, compiled straight from the reference tree.
//
// TEST INFRASTRUCTURE ONLY.  The oracle Makefile compiles this file with
// -I<reference>/cc so that the reference headers are used where they lie;
// nothing from the reference is copied.  Tests and the CPU-baseline leg of
// bench.py call these functions through ctypes to obtain the reference's own
// FP64 results (mass-assigned grids, histograms, P_ell and xi_ell tables).
//
// Reference classes driven here:
//   ConfigSpaceGrid     cc/grid/config_space_grid.h:10-57
//   MassAssignor        cc/particle_mesh/mass_assignor.h:30-234
//   PeriodicCorrelator  cc/correlate/correlator.h:254-358
//   Correlator          cc/correlate/correlator.h:360-505
//   HistogramList       cc/histogram/histogram_list.h:10-68
//   setup_wavelet/wave  cc/particle_mesh/d12.h:13-155
#include <fcntl.h>
#include <unistd.h>

#include <array>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <string>

#include "array/row_major_array.h"
#include "correlate/correlator.h"
#include "grid/config_space_grid.h"
#include "histogram/histogram_list.h"
#include "particle_mesh/distribution_functions.h"
#include "particle_mesh/mass_assignor.h"

namespace {

std::string g_last_error;
bool g_wavelet_ready = false;

void ensure_wavelet() {
  if (!g_wavelet_ready) {
    setup_wavelet();
    g_wavelet_ready = true;
  }
}

// Silences the reference's progress printing on stdout/stderr for the
// duration of one call when quiet != 0.
class QuietScope {
 public:
  explicit QuietScope(int quiet) : active_(quiet != 0) {
    if (!active_) return;
    fflush(stdout);
    fflush(stderr);
    saved_out_ = dup(1);
    saved_err_ = dup(2);
    int devnull = open("/dev/null", O_WRONLY);
    dup2(devnull, 1);
    dup2(devnull, 2);
    close(devnull);
  }
  ~QuietScope() {
    if (!active_) return;
    fflush(stdout);
    fflush(stderr);
    dup2(saved_out_, 1);
    dup2(saved_err_, 2);
    close(saved_out_);
    close(saved_err_);
  }

 private:
  bool active_;
  int saved_out_ = -1;
  int saved_err_ = -1;
};

template <typename F>
int guarded(F f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char *fcref_last_error() { return g_last_error.c_str(); }

// Copies the transposed D12 lookup table (wave[], 8 x 64 doubles) built by
// setup_wavelet(), cc/particle_mesh/d12.h:149-155.
int fcref_d12_table(double *out, int n) {
  ensure_wavelet();
  if (n != WCELLS * WAVESAMPLE) return -1;
  std::memcpy(out, wave, sizeof(double) * WCELLS * WAVESAMPLE);
  return 0;
}

// ConfigSpaceGrid::get_grid_coords, cc/grid/config_space_grid.h:31-46.
int fcref_grid_coords(const int *shape, const double *posmin, double cell,
                      const double *pos, int periodic, double *out) {
  ConfigSpaceGrid grid({shape[0], shape[1], shape[2]},
                       {posmin[0], posmin[1], posmin[2]}, cell);
  return grid.get_grid_coords(pos, periodic != 0, out) ? 1 : 0;
}

// MassAssignor over an (n, 4) posw array, then flush().  stats receives
// num_added, num_skipped, totw, totwsq, sort_time, window_time
// (mass_assignor.h:52-58): six doubles.
int fcref_mass_assign(const double *posw, long n, const int *shape,
                      const double *posmin, double cell, int scheme,
                      int periodic, long buffer_size, double *grid_out,
                      double *stats, int quiet) {
  QuietScope q(quiet);
  ensure_wavelet();
  return guarded([&] {
    ConfigSpaceGrid grid({shape[0], shape[1], shape[2]},
                         {posmin[0], posmin[1], posmin[2]}, cell);
    MassAssignor ma(grid, DistributionScheme(scheme), periodic != 0,
                    (uint64)buffer_size);
    RowMajorArrayPtr<Float, 2> p({(int)n, 4}, const_cast<double *>(posw));
    ma.add_particles_to_buffer(p);
    ma.flush();
    std::memcpy(grid_out, grid.data().data(), sizeof(double) * grid.size());
    stats[0] = (double)ma.num_added();
    stats[1] = (double)ma.num_skipped();
    stats[2] = ma.totw();
    stats[3] = ma.totwsq();
    stats[4] = ma.sort_time();
    stats[5] = ma.window_time();
  });
}

// Runs PeriodicCorrelator (survey == 0) or Correlator (survey != 0).
// grid2 == NULL runs autocorrelate(grid1), otherwise
// cross_correlate(grid1, grid2).  Output arrays are sized by the caller:
// nrows = maxell/2 + 1, nr = floor(rmax/dr), nk = floor(kmax/dk)
// (histogram_list.h:15).  timers (8 doubles, may be NULL) receives the
// reference's own phase timers (correlator.h:97-105): setup, fft_plan, fft,
// extract, multiply, ylm, histogram, total, in seconds.
int fcref_correlate(int survey, const double *grid1, const double *grid2,
                    const int *shape, double cell, const double *posmin,
                    int window, double rmax, double dr, double kmax, double dk,
                    int maxell, double *rbins, int *rcounts, double *rhist,
                    double *kbins, int *kcounts, double *khist,
                    double *zerolag, int quiet, double *timers) {
  QuietScope q(quiet);
  return guarded([&] {
    std::array<int, 3> shp = {shape[0], shape[1], shape[2]};
    std::unique_ptr<BaseCorrelator> corr;
    if (survey) {
      corr.reset(new Correlator(shp, cell, {posmin[0], posmin[1], posmin[2]},
                                WindowCorrection(window), rmax, dr, kmax, dk,
                                maxell, FFTW_ESTIMATE));
    } else {
      corr.reset(new PeriodicCorrelator(shp, cell, WindowCorrection(window),
                                        rmax, dr, kmax, dk, maxell,
                                        FFTW_ESTIMATE));
    }
    RowMajorArrayPtr<Float, 3> g1(shp, const_cast<double *>(grid1));
    if (grid2) {
      RowMajorArrayPtr<Float, 3> g2(shp, const_cast<double *>(grid2));
      corr->cross_correlate(g1, g2);
    } else {
      corr->autocorrelate(g1);
    }
    const auto &rb = corr->correlation_r();
    const auto &rc = corr->correlation_counts();
    const auto &rh = corr->correlation_histogram();
    const auto &kb = corr->power_spectrum_k();
    const auto &kc = corr->power_spectrum_counts();
    const auto &kh = corr->power_spectrum_histogram();
    std::memcpy(rbins, rb.data(), sizeof(double) * rb.size());
    std::memcpy(rcounts, rc.data(), sizeof(int) * rc.size());
    std::memcpy(rhist, rh.data(), sizeof(double) * rh.size());
    std::memcpy(kbins, kb.data(), sizeof(double) * kb.size());
    std::memcpy(kcounts, kc.data(), sizeof(int) * kc.size());
    std::memcpy(khist, kh.data(), sizeof(double) * kh.size());
    *zerolag = corr->zerolag();
    if (timers) {
      timers[0] = corr->setup_time();
      timers[1] = corr->fft_plan_time();
      timers[2] = corr->fft_time();
      timers[3] = corr->extract_time();
      timers[4] = corr->multiply_time();
      timers[5] = corr->ylm_time();
      timers[6] = corr->histogram_time();
      timers[7] = corr->total_time();
    }
  });
}

// HistogramList(n, minval, maxval, binsize).accumulate(ih, x, y) for each of
// ncalls row indices ih[c] over the same x/y arrays, then copies the state.
int fcref_histogram(int n, double minval, double maxval, double binsize,
                    int ncalls, const int *ih, const double *x,
                    const double *y, long len, double *bins, int *counts,
                    double *hist) {
  return guarded([&] {
    HistogramList h(n, minval, maxval, binsize);
    Array1D<Float> xa((int)len), ya((int)len);
    std::memcpy(xa.data(), x, sizeof(double) * len);
    std::memcpy(ya.data(), y, sizeof(double) * len);
    for (int c = 0; c < ncalls; ++c) h.accumulate(ih[c], xa, ya);
    std::memcpy(bins, h.bins().data(), sizeof(double) * h.nbins());
    std::memcpy(counts, h.counts().data(), sizeof(int) * h.counts().size());
    std::memcpy(hist, h.hist_values().data(),
                sizeof(double) * h.hist_values().size());
  });
}

}  // extern "C"
