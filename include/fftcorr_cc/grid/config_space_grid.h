// config_space_grid.h -- ConfigSpaceGrid over the B200 library.
//
// Interface of the reference's cc/grid/config_space_grid.h:10-57 as bound by
// fftcorr/grid/config_space_grid.pxd:9-14:
//   ConfigSpaceGrid(std::array<int, 3> shape, std::array<Float, 3> posmin,
//                   Float cell_size)
//   cell_size(), shape(), posmin(), size(), data(), clear(),
//   get_grid_coords(const Float *survey, bool periodic_wrap, Float *grid)
//
// data() is a host array (the Cython package wraps it as the grid's numpy
// view and users may edit it), registered as pinned memory.  A device copy
// behind fc_grid_* is what MassAssignor scatters into: every flush uploads
// the host array, scatters on the GPU and downloads the result, so the host
// array always holds the grid between calls, as in the reference.
#ifndef FFTCORR_CC_CONFIG_SPACE_GRID_H
#define FFTCORR_CC_CONFIG_SPACE_GRID_H

#include <algorithm>
#include <array>

#include "../array/row_major_array.h"
#include "../fc_check.h"
#include "../types.h"

class ConfigSpaceGrid {
 public:
  ConfigSpaceGrid(std::array<int, 3> shape, std::array<Float, 3> posmin,
                  Float cell_size)
      : posmin_(posmin), cell_size_(cell_size) {
    const int s[3] = {shape[0], shape[1], shape[2]};
    fftcorr_cc::fc_check(fc_grid_create(s, posmin.data(), cell_size, &grid_),
                         "ConfigSpaceGrid");
    data_.allocate(shape);
    if (data_.size() > 0 &&
        fc_host_register(data_.data(), data_.size() * sizeof(Float)) == FC_OK)
      registered_ = true;
  }
  ~ConfigSpaceGrid() {
    if (registered_) fc_host_unregister(data_.data());
    fc_grid_destroy(grid_);
  }
  ConfigSpaceGrid(const ConfigSpaceGrid &) = delete;
  ConfigSpaceGrid &operator=(const ConfigSpaceGrid &) = delete;

  const std::array<int, 3> &shape() const { return data_.shape(); }
  int shape(int i) const { return data_.shape(i); }
  uint64 size() const { return data_.size(); }
  const std::array<Float, 3> &posmin() const { return posmin_; }
  Float cell_size() const { return cell_size_; }

  RowMajorArrayPtr<Float, 3> &data() { return data_; }
  const RowMajorArrayPtr<Float, 3> &data() const { return data_; }

  void clear() {
    std::fill(data_.data(), data_.data() + data_.size(), 0.0);
    fftcorr_cc::fc_check(fc_grid_clear(grid_), "ConfigSpaceGrid::clear");
  }

  // Survey coordinates -> grid coordinates; false when outside the grid and
  // periodic_wrap is false (config_space_grid.h:31-46).
  bool get_grid_coords(const Float *survey, bool periodic_wrap,
                       Float *grid_coords) const {
    int inside = 0;
    fftcorr_cc::fc_check(fc_grid_coords(grid_, survey, periodic_wrap ? 1 : 0,
                                        grid_coords, &inside),
                         "ConfigSpaceGrid::get_grid_coords");
    return inside != 0;
  }

  // The library handle and the host <-> device copies used by MassAssignor.
  fc_grid *fc_handle() { return grid_; }
  void upload() {
    fftcorr_cc::fc_check(fc_grid_upload(grid_, data_.data()), "grid upload");
  }
  void download() {
    fftcorr_cc::fc_check(fc_grid_download(grid_, data_.data()), "grid download");
  }

 private:
  std::array<Float, 3> posmin_;
  Float cell_size_;
  fc_grid *grid_ = nullptr;
  RowMajorArray<Float, 3> data_;
  bool registered_ = false;
};

#endif  // FFTCORR_CC_CONFIG_SPACE_GRID_H
