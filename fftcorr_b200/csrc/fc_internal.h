// fc_internal.h -- objects behind the opaque C handles of fc_api.h.
#pragma once

#include <atomic>
#include <vector>

#include "fc_common.cuh"

namespace fc {

// Blocks of the deterministic two-pass grid reductions (8 waves of 148).
constexpr int kSumBlocks = 1184;

const char *last_error_cstr();
std::atomic<unsigned long long> &launch_counter();

// ConfigSpaceGrid (cc/grid/config_space_grid.h:10-57): an N0 x N1 x N2
// row-major FP64 grid resident in HBM, with the geometry that maps survey
// coordinates onto it.  Work on the grid is ordered on its stream.
struct Grid {
  int shape[3];
  double posmin[3];
  double cell_size;
  int device = 0;
  cudaStream_t stream = nullptr;
  DeviceBuffer data;
  DeviceBuffer scratch;

  Grid(const int shp[3], const double pmin[3], double cell);
  ~Grid();
  void clear();
  size_t size() const { return (size_t)shape[0] * shape[1] * shape[2]; }
  double *ptr() const { return data.as<double>(); }
};

inline Grid *as_grid(fc_grid *g) {
  FC_REQUIRE(g, FC_ERR_INVALID, "null grid handle");
  return reinterpret_cast<Grid *>(g);
}
inline const Grid *as_grid(const fc_grid *g) {
  FC_REQUIRE(g, FC_ERR_INVALID, "null grid handle");
  return reinterpret_cast<const Grid *>(g);
}

// ConfigSpaceGrid::get_grid_coords on the host (config_space_grid.h:31-46).
inline bool host_grid_coords(const double *pos, const double *posmin,
                             double cell, const int *shape, bool periodic,
                             double *out) {
  for (int i = 0; i < 3; ++i) {
    double x = (pos[i] - posmin[i]) / cell;
    const double xmax = shape[i];
    if (x < 0 || x >= xmax) {
      if (!periodic) return false;
      x = fmod(x, xmax);
      if (x < 0) x += xmax;
    }
    out[i] = x;
  }
  return true;
}

void device_fill(double *a, size_t n, double v, cudaStream_t s);
// Deterministic FP64 sum and sum of squares of a[0..n).  scratch holds
// 2*kSumBlocks + 2 doubles; the results land in scratch[2*kSumBlocks + {0,1}].
void device_sum_sumsq(const double *a, size_t n, double *scratch,
                      cudaStream_t s);

// Makes stream `waiter` wait for all work queued so far on `producer`.
inline void stream_after(cudaStream_t waiter, cudaStream_t producer) {
  if (waiter == producer) return;
  cudaEvent_t ev;
  FC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  FC_CUDA(cudaEventRecord(ev, producer));
  FC_CUDA(cudaStreamWaitEvent(waiter, ev, 0));
  cudaEventDestroy(ev);
}

// ----------------------------------------------- batched-form building blocks
// Enqueue-only entry points used by the batched form (fc_batch.cu): once
// prepared they allocate nothing and never synchronise the host, so a whole
// batch can be captured into one CUDA graph.
struct Assignor;
Assignor *assignor_new(Grid *g, int scheme, bool periodic);
void assignor_delete(Assignor *a);
void assignor_prepare_graph(Assignor *a, int64_t max_n, cudaStream_t s);
void assignor_enqueue_graph(Assignor *a, const double *posw, int64_t n,
                            cudaStream_t s);
const double *assignor_totals(const Assignor *a);  // device [totw, totwsq]
const unsigned long long *assignor_counts(const Assignor *a);  // [num_added]

// One chunk of a deterministic histogram reduction (see fc_hist.cuh): the
// sum of values[perm[start .. start+len)] goes to partials[index].
struct HistItem {
  const double *values;
  const uint32_t *perm;
  uint32_t start;
  int len;
};
// One bin: dest = sum of partials[first .. first+count) in order.
struct FoldItem {
  int first;
  int count;
  double *dest;
};

struct Correlator;
Correlator *correlator_new_periodic(const int shape[3], double cell, int window,
                                    double rmax, double dr, double kmax,
                                    double dk, int maxell, int precision);
void correlator_delete(Correlator *c);
// Enqueues a periodic autocorrelation of rho on s with the histograms
// deferred (every multipole keeps its own subgrids).
void correlator_enqueue_deferred(Correlator *c, const double *rho,
                                 cudaStream_t s);
// Appends the histogram work of the last deferred run.
void correlator_hist_work(Correlator *c, std::vector<HistItem> &items,
                          std::vector<FoldItem> &folds);
void correlator_results(Correlator *c, double *rbins, int *rcounts,
                        double *rhist, double *kbins, int *kcounts,
                        double *khist, double *zerolag);
void correlator_dims(const Correlator *c, int *nrows, int *nr, int *nk);

}  // namespace fc
