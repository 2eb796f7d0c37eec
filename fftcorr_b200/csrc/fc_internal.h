// fc_internal.h -- objects behind the opaque C handles of fc_api.h.
#pragma once

#include <memory>
#include <atomic>
#include <vector>

#include "fc_common.cuh"
#include "fc_hist.cuh"

namespace fc {

// Blocks of the deterministic two-pass grid reductions (8 waves of 148).
constexpr int kSumBlocks = 1184;

const char *last_error_cstr();
std::atomic<unsigned long long> &launch_counter();

// ConfigSpaceGrid (cc/grid/config_space_grid.h:10-57): an N0 x N1 x N2
// row-major grid resident in HBM, with the geometry that maps survey
// coordinates onto it.  Work on the grid is ordered on its stream.  Cells
// are FP64 (the reference's type) or, for grids made for the FP32-mixed
// correlators, FP32: mass assignment still sums in FP64 and rounds once per
// update of a cell, and arithmetic on the grid is done in FP64 per cell.
struct Grid {
  int shape[3];
  double posmin[3];
  double cell_size;
  int precision = FC_FP64;  // FC_FP64 or FC_FP32_MIXED (FP32 cells)
  int device = 0;
  cudaStream_t stream = nullptr;
  DeviceBuffer data;
  DeviceBuffer scratch;
  // Expires with the grid, so objects that use it can tell it has gone.
  std::shared_ptr<int> alive = std::make_shared<int>(0);

  Grid(const int shp[3], const double pmin[3], double cell,
       int precision = FC_FP64);
  ~Grid();
  void clear();
  size_t size() const { return (size_t)shape[0] * shape[1] * shape[2]; }
  bool fp32() const { return precision == FC_FP32_MIXED; }
  size_t cell_bytes() const { return fp32() ? sizeof(float) : sizeof(double); }
  void *raw() const { return data.get(); }
  // The cells of an FP64 grid.
  double *ptr() const {
    FC_REQUIRE(!fp32(), FC_ERR_INVALID, "this operation needs an FP64 grid");
    return data.as<double>();
  }
};

// A density on the device as a correlator takes it: FP64 cells, or the FP32
// cells of an FP32 grid.
struct Density {
  const void *p;
  bool f32;
};
inline Density density_of(const Grid *g) { return {g->raw(), g->fp32()}; }

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
void device_sum_sumsq(const float *a, size_t n, double *scratch,
                      cudaStream_t s);
// out[i] = (double)in[i].
void device_widen(const float *in, double *out, size_t n, cudaStream_t s);

// Makes stream `waiter` wait for all work queued so far on `producer`.
inline void stream_after(cudaStream_t waiter, cudaStream_t producer) {
  if (waiter == producer) return;
  cudaEvent_t ev;
  FC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  FC_CUDA(cudaEventRecord(ev, producer));
  FC_CUDA(cudaStreamWaitEvent(waiter, ev, 0));
  cudaEventDestroy(ev);
}

// ------------------------------------------------------ device catalogs
// Grid geometry for the displacement kernel.
struct AssignGeomLite {
  int n[3];
  double posmin[3];
  double cell;
  int periodic;
};
// Particles first .. first+n of the counter-based uniform catalog (seed) into
// posw[0 .. n): positions uniform in [lo, hi), weights w0 + (w1 - w0) u.
void catalog_uniform(double *posw, int64_t first, int64_t n, const double lo[3],
                     const double hi[3], double w0, double w1, uint64_t seed,
                     cudaStream_t s);
// Writes the catalog a spec describes into posw (n rows of x, y, z, w).
// scratch (optional): device memory for cluster centres, at least
// catalog_scratch_bytes(c), so the call allocates nothing.
void catalog_generate(const fc_catalog_spec &c, double *posw, cudaStream_t s,
                      double *scratch = nullptr, size_t scratch_bytes = 0);
size_t catalog_scratch_bytes(const fc_catalog_spec &c);
// out[i] = pos[i] + disp[cell of pos[i]]; *flag = 1 if some position has no
// cell.  Rows of pos and out are `stride` / `out_stride` doubles apart.
void displace(const double *pos, int stride, int64_t n, const double *disp,
              const AssignGeomLite &g, double *out, int out_stride, int *flag,
              cudaStream_t s);

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
// Assigns n particles from a device array and waits (MassAssignor::
// add_particles_to_buffer + flush).
void assignor_add_device(Assignor *a, const double *posw, int64_t n);
void assignor_clear(Assignor *a);
bool assignor_has_d12();
void assignor_stats(Assignor *a, fc_assign_stats *s);
// Device bytes an assignor holds after assigning n particles at once.
size_t assignor_bytes(const int shape[3], int64_t n);
const double *assignor_totals(const Assignor *a);  // device [totw, totwsq]
const unsigned long long *assignor_counts(const Assignor *a);  // [num_added]

struct Correlator;
Correlator *correlator_new(int kind, const int shape[3], double cell,
                           const double posmin[3], int window, double rmax,
                           double dr, double kmax, double dk, int maxell,
                           int precision);
void correlator_delete(Correlator *c);
// Autocorrelation of a device grid (waits for the result).
void correlator_autocorrelate(Correlator *c, const Grid *g);
size_t correlator_footprint(int kind, const int shape[3], double cell,
                            double rmax, double kmax, int maxell, int precision);
// Periodic correlators only: every multipole keeps its own subgrids and the
// histograms are left to the caller (correlator_hist_work).
void correlator_make_deferred(Correlator *c);
// The padded real work grid [N0][N1][2(N2/2+1)] in the correlator's
// precision.
void *correlator_work(Correlator *c);
void correlator_set_stream(Correlator *c, cudaStream_t s);
// Enqueues a periodic autocorrelation of the density already in the work
// grid (deferred mode; no allocation or host synchronisation).
void correlator_enqueue_prepared(Correlator *c);
// Appends the histogram reductions of the last deferred run.
void correlator_hist_work(Correlator *c, std::vector<HistItem> &items,
                          std::vector<FoldItem> &folds);
void correlator_results(Correlator *c, double *rbins, int *rcounts,
                        double *rhist, double *kbins, int *kcounts,
                        double *khist, double *zerolag);
void correlator_dims(const Correlator *c, int *nrows, int *nr, int *nk);
struct CorrShapes {
  LaunchShape *abs2, *ksub, *rsub;
};
CorrShapes correlator_shapes(Correlator *c);
// Launches one of the tunable kernels (0 |F|^2, 1 k-subgrid, 2 r-subgrid)
// on s, for timing.
void correlator_time_kernels(Correlator *c, int which, cudaStream_t s);

}  // namespace fc
