// Drives the C++ class surface (include/fftcorr_cc) the way the reference's
// Cython package and CLI call the reference classes, and writes every
// result for tests/test_cc_surface.py to compare with the oracle.
//
//   test_cc_surface IN_FILE OUT_DIR
//
// IN_FILE: int32 shape[3], float64 posmin[3], float64 cell, int64 n, then
// n rows of (x, y, z, w) float64.  OUT_DIR receives raw arrays (*.bin).
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "correlate/correlator.h"
#include "grid/config_space_grid.h"
#include "histogram/histogram_list.h"
#include "particle_mesh/mass_assignor.h"

namespace {

std::string g_out;

template <typename T>
void save(const char *name, const T *p, size_t n) {
  const std::string path = g_out + "/" + name + ".bin";
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f || std::fwrite(p, sizeof(T), n, f) != n) {
    std::fprintf(stderr, "cannot write %s\n", path.c_str());
    std::exit(2);
  }
  std::fclose(f);
}

void save_results(const std::string &tag, const BaseCorrelator &c) {
  const std::string t = tag + "_";
  save((t + "rbins").c_str(), c.correlation_r().data(), c.correlation_r().size());
  save((t + "rcounts").c_str(), c.correlation_counts().data(),
       c.correlation_counts().size());
  save((t + "rhist").c_str(), c.correlation_histogram().data(),
       c.correlation_histogram().size());
  save((t + "kbins").c_str(), c.power_spectrum_k().data(), c.power_spectrum_k().size());
  save((t + "kcounts").c_str(), c.power_spectrum_counts().data(),
       c.power_spectrum_counts().size());
  save((t + "khist").c_str(), c.power_spectrum_histogram().data(),
       c.power_spectrum_histogram().size());
  const Float z = c.zerolag();
  save((t + "zerolag").c_str(), &z, 1);
}

template <typename E, typename F>
int throws(F f) {
  try {
    f();
  } catch (const E &) {
    return 1;
  } catch (...) {
    return 0;
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s IN_FILE OUT_DIR\n", argv[0]);
    return 2;
  }
  g_out = argv[2];
  FILE *f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  std::array<int, 3> shape;
  std::array<Float, 3> posmin;
  Float cell;
  long long n;
  if (std::fread(shape.data(), sizeof(int), 3, f) != 3 ||
      std::fread(posmin.data(), sizeof(Float), 3, f) != 3 ||
      std::fread(&cell, sizeof(Float), 1, f) != 1 ||
      std::fread(&n, sizeof(long long), 1, f) != 1)
    return 2;
  std::vector<Float> posw((size_t)n * 4);
  if (std::fread(posw.data(), sizeof(Float), posw.size(), f) != posw.size()) return 2;
  std::fclose(f);

  // MassAssignor: the first half as (n, 4) rows, a quarter as (n, 3) rows
  // with a weight array, the rest one particle at a time; then flush.
  ConfigSpaceGrid grid(shape, posmin, cell);
  MassAssignor ma(grid, kTriangularShapedCloud, false, 1000000);
  const int h = (int)(n / 2), q = (int)(n / 4);
  ma.add_particles_to_buffer(RowMajorArrayPtr<Float, 2>({h, 4}, posw.data()));
  std::vector<Float> pos3((size_t)q * 3), w3((size_t)q);
  for (int i = 0; i < q; ++i) {
    for (int a = 0; a < 3; ++a) pos3[3 * i + a] = posw[4 * (size_t)(h + i) + a];
    w3[i] = posw[4 * (size_t)(h + i) + 3];
  }
  ma.add_particles_to_buffer(RowMajorArrayPtr<Float, 2>({q, 3}, pos3.data()),
                             RowMajorArrayPtr<Float, 1>({q}, w3.data()));
  for (long long i = h + q; i < n; ++i)
    ma.add_particle_to_buffer(&posw[4 * (size_t)i], posw[4 * (size_t)i + 3]);
  ma.flush();
  save("grid", grid.data().data(), grid.data().size());
  const double stats[4] = {(double)ma.num_added(), (double)ma.num_skipped(),
                           ma.totw(), ma.totwsq()};
  save("stats", stats, 4);

  // A second grid: nearest cell, every particle through the constant-weight
  // overload with weight 1, buffer 0 (applied at once).
  ConfigSpaceGrid grid2(shape, posmin, cell);
  {
    MassAssignor ngp(grid2, kNearestCell, false, 0);
    std::vector<Float> pos((size_t)n * 3);
    for (long long i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) pos[3 * (size_t)i + a] = posw[4 * (size_t)i + a];
    ngp.add_particles_to_buffer(RowMajorArrayPtr<Float, 2>({(int)n, 3}, pos.data()),
                                1.0);
  }
  save("grid2", grid2.data().data(), grid2.data().size());

  Float coords[3];
  const Float inside_pt[3] = {posmin[0] + 1.5 * cell, posmin[1] + 2.25 * cell,
                              posmin[2] + 0.5 * cell};
  const int in = grid.get_grid_coords(inside_pt, false, coords) ? 1 : 0;
  save("coords", coords, 3);

  Correlator survey(shape, cell, posmin, kTscAliasedCorrection, 60.0, 10.0, 0.2,
                    0.04, 4, 0);
  survey.autocorrelate(grid.data());
  save_results("survey", survey);
  survey.cross_correlate(grid.data(), grid2.data());
  save_results("cross", survey);

  PeriodicCorrelator periodic(shape, cell, kNoCorrection, 60.0, 10.0, 0.2, 0.04,
                              2, 0);
  periodic.autocorrelate(grid2.data());
  save_results("periodic", periodic);

  HistogramList hl(2, -10.0, 10.0, 2.0);
  const int m = 1000;
  Array1D<Float> x(m), y(m);
  for (int i = 0; i < m; ++i) {
    x[i] = -12.0 + 24.0 * (i + 0.5) / m;
    y[i] = 0.001 * i - 0.3;
  }
  hl.accumulate(0, x, y);
  hl.accumulate(1, y, x);
  hl.accumulate(1, x, x);
  save("hist_bins", hl.bins().data(), hl.bins().size());
  save("hist_counts", hl.counts().data(), hl.counts().size());
  save("hist_values", hl.hist_values().data(), hl.hist_values().size());

  // Error behaviour: the reference's exception types.
  int err[5];
  err[0] = throws<std::invalid_argument>([&] {
    ma.add_particles_to_buffer(RowMajorArrayPtr<Float, 2>({q, 3}, pos3.data()));
  });
  err[1] = throws<std::invalid_argument>([&] {
    ma.add_particles_to_buffer(RowMajorArrayPtr<Float, 2>({q, 3}, pos3.data()),
                               RowMajorArrayPtr<Float, 1>({q - 1}, w3.data()));
  });
  err[2] = throws<std::invalid_argument>(
      [&] { ConfigSpaceGrid bad({shape[0], -1, shape[2]}, posmin, cell); });
  err[3] = throws<std::invalid_argument>([&] {
    RowMajorArray<Float, 3> small({shape[0], shape[1], shape[2] - 1});
    survey.autocorrelate(small);
  });
  err[4] = throws<std::invalid_argument>([&] {
    PeriodicCorrelator p(shape, cell, kNoCorrection, 60.0, 10.0, 0.2, 0.04, 3, 0);
  });
  save("errors", err, 5);
  save("inside", &in, 1);
  std::printf("ok\n");
  return 0;
}
