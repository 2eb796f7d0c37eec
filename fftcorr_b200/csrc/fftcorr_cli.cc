// fftcorr_cli.cc -- the `fftcorr` command-line driver on the GPU library.
//
// Drop-in for the reference CLI (cc/fftcorr.cc:233-463): the same flags and
// defaults, the same binary catalog format (cc/catalog_reader.h:16-71: a
// 64-byte header posmin[3], posmax[3], max_sep, pad, then x, y, z, w
// doubles per particle), the same box padding and cell-size rule, the same
// periodic normalisation, and the same stdout tables (print_hist,
// cc/fftcorr.cc:213-228: "%1d %7.4f %8.0f" then " %16.9e" per multipole; P
// rows prefixed 1 and divided by the counts, xi rows prefixed 0 and divided
// only for periodic boxes), so harnesses that parse the reference's output
// run unchanged.  Everything heavy runs through include/fc_api.h.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fc_api.h"

namespace {

void usage() {
  std::fprintf(stderr,
               "FFTCORR: Error in command-line\n"
               "   -n <int> (or -ngrid): FFT linear grid size for a cubic box\n"
               "   -n3 <int> <int> <int> (or -ngrid3): FFT grid sizes for a "
               "rectangle (outranks -n)\n"
               "   -ell <int> (or -maxell): Multipole to compute.\n"
               "   -r <float> (or -sep): Max separation.\n"
               "   -dr <float> (or -dsep): Binning of separation.\n"
               "   -kmax <float> (or -k): Maximum wavenumber for power spectrum.\n"
               "   -dk <float>: Binning of wavenumber.\n"
               "   -periodic (or -p): Cubic periodic box; the density is "
               "normalised by its mean.\n"
               "   -dist <int> (or -d): Distribution scheme (0 nearest cell, 1 "
               "TSC, 2 D12 wavelet, 3 CIC).\n"
               "   -cell <float> (or -c): Cell size (not with -periodic).\n"
               "   -in <filename> (or -i): Input file name\n"
               "   -in2 <filename> (or -i2): Second input file name\n"
               "   -out <filename> (or -o): Output file name, default stdout\n"
               "   -wisdom <filename> (or -wf): accepted, unused (cuFFT/GPU "
               "plans live with the correlator)\n"
               "   -fp32: FP32-mixed transforms (FP64 coordinates, Y_lm "
               "normalisation and histograms)\n");
  std::exit(1);
}

void check(int rc, const char *what) {
  if (rc != 0) {
    std::fprintf(stderr, "fftcorr: %s failed: %s\n", what, fc_last_error());
    std::exit(2);
  }
}

[[noreturn]] void fail(const char *msg) {
  std::fprintf(stderr, "fftcorr: %s\n", msg);
  std::exit(1);
}

double now() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Reads the 64-byte catalog header (catalog_reader.h:16-43).
void read_header(const char *fn, double posmin[3], double posmax[3]) {
  FILE *fp = std::fopen(fn, "rb");
  if (!fp) fail("cannot open input file");
  double buf[8];
  if (std::fread(buf, sizeof(double), 8, fp) != 8) fail("short header");
  std::fclose(fp);
  for (int i = 0; i < 7; ++i)
    if (!(std::fabs(buf[i]) < 1e10)) fail("header value too large");
  for (int i = 0; i < 3; ++i) {
    posmin[i] = buf[i];
    posmax[i] = buf[3 + i];
  }
  std::fprintf(stderr, "Reading survey box from header of %s\n", fn);
  std::fprintf(stderr, "posmin = [%.4f, %.4f, %.4f]\n", posmin[0], posmin[1],
               posmin[2]);
  std::fprintf(stderr, "posmax = [%.4f, %.4f, %.4f]\n", posmax[0], posmax[1],
               posmax[2]);
}

// Streams the particles of one file into the assignor and flushes it
// (catalog_reader.h:45-71).  Returns the number of particles read.
long read_galaxies(const char *fn, fc_assignor *ma, double *io_time) {
  std::fprintf(stdout, "# Reading from file named %s\n", fn);
  FILE *fp = std::fopen(fn, "rb");
  if (!fp) fail("cannot open input file");
  double hdr[8];
  if (std::fread(hdr, sizeof(double), 8, fp) != 8) fail("short header");
  const size_t chunk = (size_t)1 << 22;  // particles per read
  std::vector<double> buf(4 * chunk);
  long count = 0;
  for (;;) {
    const double t0 = now();
    const size_t got = std::fread(buf.data(), 4 * sizeof(double), chunk, fp);
    *io_time += now() - t0;
    if (got == 0) break;
    check(fc_assignor_add_posw(ma, buf.data(), (int64_t)got), "mass assignment");
    count += (long)got;
    if (got < chunk) break;
  }
  std::fclose(fp);
  std::fprintf(stdout, "# Found %ld galaxies in this file\n", count);
  check(fc_assignor_flush(ma), "flush");
  return count;
}

// print_hist (cc/fftcorr.cc:213-228).
void print_hist(const std::vector<double> &bins, const std::vector<int> &counts,
                const std::vector<double> &hist, int nrows, FILE *fp,
                int prefix, bool normalize) {
  const int nb = (int)bins.size();
  for (int j = 0; j < nb; ++j) {
    const double count = counts[j];
    const double denom = normalize && count != 0 ? count : 1.0;
    std::fprintf(fp, "%1d ", prefix);
    std::fprintf(fp, "%7.4f %8.0f", bins[j], count);
    for (int i = 0; i < nrows; ++i)
      std::fprintf(fp, " %16.9e", hist[(size_t)i * nb + j] / denom);
    std::fprintf(fp, "\n");
  }
}

}  // namespace

int main(int argc, char **argv) {
  const double t_start = now();
  double sep = -123.0, dsep = 10.0, kmax = 0.03, dk = 0.01;
  int maxell = 0, ngrid_cube = 256, dist = 2;
  bool periodic = false, fp32 = false;
  int ngrid[3] = {-1, -1, -1};
  double cell = -123.0;
  const char *infile = "/tmp/corrRR.dat";
  const char *infile2 = nullptr;
  const char *outfile = nullptr;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> const char * {
      if (i + 1 >= argc) usage();
      return argv[++i];
    };
    if (a == "-ngrid" || a == "-n") ngrid_cube = std::atoi(next());
    else if (a == "-ngrid3" || a == "-n3") {
      ngrid[0] = std::atoi(next());
      ngrid[1] = std::atoi(next());
      ngrid[2] = std::atoi(next());
    } else if (a == "-maxell" || a == "-ell") maxell = std::atoi(next());
    else if (a == "-sep" || a == "-r") sep = std::atof(next());
    else if (a == "-dsep" || a == "-dr") dsep = std::atof(next());
    else if (a == "-kmax" || a == "-k") kmax = std::atof(next());
    else if (a == "-dk") dk = std::atof(next());
    else if (a == "-cell" || a == "-c") cell = std::atof(next());
    else if (a == "-in" || a == "-i") infile = next();
    else if (a == "-in2" || a == "-i2") infile2 = next();
    else if (a == "-out" || a == "-o") outfile = next();
    else if (a == "-periodic" || a == "-p") periodic = true;
    else if (a == "-dist" || a == "-d") dist = std::atoi(next());
    else if (a == "-wisdom" || a == "-wf") next();
    else if (a == "-fp32") fp32 = true;
    else usage();
  }
  // The reference asserts these (cc/fftcorr.cc:298-316).
  if (!(ngrid_cube > 0)) fail("ngrid must be positive");
  if (!(maxell >= 0 && maxell % 2 == 0)) fail("maxell must be even");
  if (!(sep > 0.0)) fail("sep must be positive");
  if (!(dsep > 0.0)) fail("dsep must be positive");
  if (!(kmax != 0.0)) fail("kmax must be nonzero");
  if (!(dk > 0.0)) fail("dk must be positive");
  if (periodic && cell >= 0) fail("cell size cannot be set for a periodic box");
  if (outfile && !std::freopen(outfile, "w", stdout)) fail("cannot open output");
  if (ngrid[0] <= 0) ngrid[0] = ngrid[1] = ngrid[2] = ngrid_cube;
  for (int i = 0; i < 3; ++i)
    if (ngrid[i] <= 0) fail("grid sizes must be positive");
  std::fprintf(stdout, "# Running on the GPU (fftcorr_b200 %d).\n", fc_version());

  double posmin[3], posmax[3];
  read_header(infile, posmin, posmax);
  if (!periodic) {
    const double pad = sep / 1.5;
    for (int i = 0; i < 3; ++i) {
      posmin[i] -= pad;
      posmax[i] += pad;
    }
  }
  for (int i = 0; i < 3; ++i)
    cell = std::max(cell, (posmax[i] - posmin[i]) / ngrid[i]);
  std::fprintf(stdout, "# Adopted cell_size=%f for ngrid=[%d, %d, %d]\n", cell,
               ngrid[0], ngrid[1], ngrid[2]);
  std::fprintf(stdout, "# Adopted boxsize: %6.1f %6.1f %6.1f\n", cell * ngrid[0],
               cell * ngrid[1], cell * ngrid[2]);

  fc_grid *grid = nullptr;
  check(fc_grid_create(ngrid, posmin, cell, &grid), "grid");
  fc_assignor *ma = nullptr;
  check(fc_assignor_create(grid, dist, periodic ? 1 : 0, 1000000, &ma),
        "mass assignor");
  double io_time = 0.0;
  const double t_grid0 = now();
  long cnt = read_galaxies(infile, ma, &io_time);
  if (infile2) cnt += read_galaxies(infile2, ma, &io_time);
  const double grid_time = now() - t_grid0 - io_time;

  fc_assign_stats st;
  check(fc_assignor_stats(ma, &st), "stats");
  std::fprintf(stdout, "# Found %llu particles. Total weight %10.4e.\n",
               (unsigned long long)st.num_added, st.totw);
  double totw2 = 0, sumsq = 0;
  check(fc_grid_sum(grid, &totw2, &sumsq), "grid sum");
  std::fprintf(stdout, "# Sum of grid is %10.4e (delta = %10.4e)\n", totw2,
               totw2 - st.totw);
  std::fprintf(stdout, "# Sum of squares of grid is %10.4e \n", sumsq);
  const double ncells = (double)ngrid[0] * ngrid[1] * ngrid[2];
  if (periodic) {
    const double mean = st.totw / ncells;
    std::fprintf(stdout, "# Normalizing by mean cell density %10.4e\n", mean);
    check(fc_grid_add_scalar(grid, -mean), "add_scalar");
    check(fc_grid_multiply_by(grid, 1.0 / mean), "multiply_by");
  }
  double totwsq = st.totwsq;
  double sumsq_dens = 0;
  check(fc_grid_sum(grid, nullptr, &sumsq_dens), "grid sum");
  std::fprintf(stdout, "# Sum of squares of density = %14.7e\n", sumsq_dens);
  std::fprintf(stdout,
               "# Sum of squares of weights (divide by I for Pshot) = %14.7e\n",
               totwsq);
  switch (dist) {
    case 0: std::fprintf(stdout, "# Using nearest cell method\n"); break;
    case 1:
      totwsq *= 0.55 * 0.55 * 0.55;
      std::fprintf(stdout, "# Using triangular cloud-in-cell\n");
      break;
    case 2: std::fprintf(stdout, "# Using D12 wavelet\n"); break;
    default: std::fprintf(stdout, "# Using trilinear cloud-in-cell\n"); break;
  }
  const double vcell = cell * cell * cell;
  std::fprintf(stdout, "# Estimate of I (denominator) = %14.7e - %14.7e = %14.7e\n",
               sumsq_dens / vcell, totwsq / vcell, (sumsq_dens - totwsq) / vcell);

  const int window = dist == 1 ? FC_TSC_ALIASED_CORRECTION : FC_NO_CORRECTION;
  fc_correlator *corr = nullptr;
  check(fc_corr_create(periodic ? FC_PERIODIC : FC_SURVEY, ngrid, cell, posmin,
                       window, sep, dsep, kmax, dk, maxell, 0,
                       fp32 ? FC_FP32_MIXED : FC_FP64, &corr),
        "correlator");
  check(fc_corr_autocorrelate_grid(corr, grid), "correlation");

  int nrows = 0, nr = 0, nk = 0;
  check(fc_corr_dims(corr, &nrows, &nr, &nk, nullptr, nullptr), "dims");
  std::vector<double> rbins(nr), rhist((size_t)nrows * nr), kbins(nk),
      khist((size_t)nrows * nk);
  std::vector<int> rcounts((size_t)nrows * nr), kcounts((size_t)nrows * nk);
  double zerolag = 0;
  check(fc_corr_results(corr, rbins.data(), rcounts.data(), rhist.data(),
                        kbins.data(), kcounts.data(), khist.data(), &zerolag),
        "results");
  std::fprintf(stdout, "# Anisotropic power spectrum:\n");
  print_hist(kbins, kcounts, khist, nrows, stdout, 1, true);
  std::fprintf(stdout, "# Anisotropic correlations:\n");
  print_hist(rbins, rcounts, rhist, nrows, stdout, 0, periodic);
  std::fprintf(stdout, "#\n# Zero-lag correlations are %14.7e\n", zerolag);
  double sum_ell0 = 0.0;
  for (int j = 0; j < nk; ++j) sum_ell0 += khist[j];
  std::fprintf(stdout, "#\n# Integral of power spectrum is %14.7e\n",
               sum_ell0 / (cell * cell * cell * ncells));

  fc_corr_timings tm;
  check(fc_corr_timings_get(corr, &tm), "timings");
  const double total = now() - t_start;
  std::fflush(stdout);
  std::fprintf(stderr, "#\n# Timing Report: \n");
  std::fprintf(stderr, "# IO time:         %8.4f s, %6.3f Mparticles/sec\n",
               io_time, cnt / std::max(io_time, 1e-9) / 1e6);
  std::fprintf(stderr, "# Grid time:    %8.4f s, %6.3f Mparticles/sec\n",
               grid_time, cnt / std::max(grid_time, 1e-9) / 1e6);
  std::fprintf(stderr, "#            Sorting:   %8.4f s\n", st.sort_time);
  std::fprintf(stderr, "#            Window:   %8.4f s\n", st.window_time);
  std::fprintf(stderr, "# Correlate: Total time:   %8.4f s (%d transforms)\n",
               tm.total_time, tm.n_fft);
  std::fprintf(stderr, "# Total time:       %8.4f s\n", total);
  fc_corr_destroy(corr);
  fc_assignor_destroy(ma);
  fc_grid_destroy(grid);
  return 0;
}
