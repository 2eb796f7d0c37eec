// fc_internal.h -- objects behind the opaque C handles of fc_api.h.
#pragma once

#include "fc_common.cuh"

namespace fc {

// Blocks of the deterministic two-pass grid reductions (8 waves of 148).
constexpr int kSumBlocks = 1184;

const char *last_error_cstr();

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

}  // namespace fc
