/*
 * oracle_grid.c -- CPU restatement (plain C, FP64) of the reference's mass
 * assignment and histogram arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this; the fftcorr_b200 library never
 * does.  It is compiled -ffp-contract=off so every product is rounded the way
 * the reference's parity build rounds it.
 *
 * Particles are processed in input order, which is what the reference's
 * MassAssignor does with buffer_size == 0 (mass_assignor.h:112-116), so for
 * that setting the grid is bit-identical to the reference's.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

enum { NEAREST_CELL = 0, TSC = 1, WAVELET = 2, CIC = 3 };

/* ConfigSpaceGrid::get_grid_coords, cc/grid/config_space_grid.h:31-46:
 * x = (p - posmin) / cell; outside [0, n) -> skip, or fmod wrap. */
int fco_grid_coords(const double *pos, const double *posmin, double cell,
                    const int *shape, int periodic, double *out) {
  for (int i = 0; i < 3; ++i) {
    double x = (pos[i] - posmin[i]) / cell;
    const double xmax = shape[i];
    if (x < 0 || x >= xmax) {
      if (!periodic) return 0;
      x = fmod(x, xmax);
      if (x < 0) x += xmax;
    }
    out[i] = x;
  }
  return 1;
}

static inline long wrap(long i, long n) {
  long r = i % n;
  return r < 0 ? r + n : r;
}

/* Adds one particle at grid coordinates x with weight w.
 *   NGP: distribution_functions.h:25-32
 *   TSC: distribution_functions.h:34-160 (27 taps, offsets -1..1, wrapped;
 *        x weights carry the particle weight, products ((wx*wy)*wz))
 *   D12: distribution_functions.h:162-217 with d12.h (8 taps per axis,
 *        offsets -1..6, sub-cell sample floor(frac*64), Dx = wave*w,
 *        Dxy = Dx*wavey, value = wavez*Dxy)
 *   CIC: trilinear, 8 taps (offsets 0..1), same product order as TSC.  The
 *        reference has no CIC; this follows the textbook definition. */
static void add_particle(double *grid, const int *shape, const double *x,
                         double w, int scheme, const double *wave) {
  const long n0 = shape[0], n1 = shape[1], n2 = shape[2];
  long ix = (long)floor(x[0]);
  long iy = (long)floor(x[1]);
  long iz = (long)floor(x[2]);
  if (scheme == NEAREST_CELL) {
    grid[(wrap(ix, n0) * n1 + wrap(iy, n1)) * n2 + wrap(iz, n2)] += w;
    return;
  }
  double wx[8], wy[8], wz[8];
  int width, omin;
  if (scheme == TSC) {
    const double rx = x[0] - ix, ry = x[1] - iy, rz = x[2] - iz;
    wx[0] = 0.5 * (1 - rx) * (1 - rx) * w;
    wx[1] = (0.5 + rx - rx * rx) * w;
    wx[2] = 0.5 * rx * rx * w;
    wy[0] = 0.5 * (1 - ry) * (1 - ry);
    wy[1] = 0.5 + ry - ry * ry;
    wy[2] = 0.5 * ry * ry;
    wz[0] = 0.5 * (1 - rz) * (1 - rz);
    wz[1] = 0.5 + rz - rz * rz;
    wz[2] = 0.5 * rz * rz;
    width = 3;
    omin = -1;
  } else if (scheme == CIC) {
    const double rx = x[0] - ix, ry = x[1] - iy, rz = x[2] - iz;
    wx[0] = (1 - rx) * w;
    wx[1] = rx * w;
    wy[0] = 1 - ry;
    wy[1] = ry;
    wz[0] = 1 - rz;
    wz[1] = rz;
    width = 2;
    omin = 0;
  } else {
    const int sx = (int)floor((x[0] - ix) * 64);
    const int sy = (int)floor((x[1] - iy) * 64);
    const int sz = (int)floor((x[2] - iz) * 64);
    for (int o = 0; o < 8; ++o) {
      wx[o] = wave[sx * 8 + o] * w;
      wy[o] = wave[sy * 8 + o];
      wz[o] = wave[sz * 8 + o];
    }
    width = 8;
    omin = -1;
  }
  for (int a = 0; a < width; ++a) {
    const long gx = wrap(ix + omin + a, n0);
    for (int b = 0; b < width; ++b) {
      const long gy = wrap(iy + omin + b, n1);
      const double wxy = wx[a] * wy[b];
      double *row = grid + (gx * n1 + gy) * n2;
      for (int c = 0; c < width; ++c) {
        const long gz = wrap(iz + omin + c, n2);
        if (scheme == WAVELET)
          row[gz] += wz[c] * wxy;
        else
          row[gz] += wxy * wz[c];
      }
    }
  }
}

/* MassAssignor::add_particles_to_buffer + flush with buffer_size 0
 * (mass_assignor.h:72-125).  stats: num_added, num_skipped, totw, totwsq,
 * accumulated in input order.  wave: the transposed 8x64 D12 table (only
 * read for scheme 2). */
int fco_mass_assign(const double *posw, long n, const int *shape,
                    const double *posmin, double cell, int scheme,
                    int periodic, const double *wave, double *grid,
                    double *stats) {
  if (scheme < 0 || scheme > 3) return -1;
  if (scheme == WAVELET && !wave) return -2;
  for (long p = 0; p < n; ++p) {
    const double *row = posw + 4 * p;
    double x[3];
    if (!fco_grid_coords(row, posmin, cell, shape, periodic, x)) {
      stats[1] += 1;
      continue;
    }
    const double w = row[3];
    add_particle(grid, shape, x, w, scheme, wave);
    stats[0] += 1;
    stats[2] += w;
    stats[3] += w * w;
  }
  return 0;
}

/* Cell key of each particle, in the reference's row-major flat index
 * (RowMajorArrayPtr::get_index of floor(x), mass_assignor.h:119), or -1
 * for skipped particles. */
void fco_cell_index(const double *posw, long n, const int *shape,
                    const double *posmin, double cell, int periodic,
                    int64_t *out) {
  for (long p = 0; p < n; ++p) {
    double x[3];
    if (!fco_grid_coords(posw + 4 * p, posmin, cell, shape, periodic, x)) {
      out[p] = -1;
      continue;
    }
    out[p] = ((int64_t)floor(x[0]) * shape[1] + (int64_t)floor(x[1])) *
                 shape[2] +
             (int64_t)floor(x[2]);
  }
}

/* HistogramList::accumulate, cc/histogram/histogram_list.h:33-45:
 * bin = floor((x - minval) / binsize), skipped outside [0, nbins). */
void fco_hist_accumulate(double minval, double binsize, int nbins,
                         const double *x, const double *y, long len,
                         int *count, double *hist) {
  for (long j = 0; j < len; ++j) {
    const int bin = (int)floor((x[j] - minval) / binsize);
    if (bin >= nbins || bin < 0) continue;
    ++count[bin];
    hist[bin] += y[j];
  }
}

/* Bin index of every value, -1 when outside [0, nbins). */
void fco_bin_index(double minval, double binsize, int nbins, const double *x,
                   long len, int *out) {
  for (long j = 0; j < len; ++j) {
    const int bin = (int)floor((x[j] - minval) / binsize);
    out[j] = (bin >= nbins || bin < 0) ? -1 : bin;
  }
}
