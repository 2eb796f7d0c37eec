// mass_assignor.h -- MassAssignor over the B200 library.
//
// Interface of the reference's cc/particle_mesh/mass_assignor.h:30-125 as
// bound by fftcorr/particle_mesh/mass_assignor.pxd:10-29:
//   MassAssignor(ConfigSpaceGrid &grid, DistributionScheme scheme,
//                bool periodic_wrap, int buffer_size)
//   add_particles_to_buffer(posw (n, 4))
//   add_particles_to_buffer(pos (n, 3), weights (n))
//   add_particles_to_buffer(pos (n, 3), Float weight)
//   add_particle_to_buffer(const Float *pos, Float w)
//   flush(), clear(), buffer_size(), num_added(), num_skipped(), totw(),
//   totwsq(), sort_time(), window_time()
// with the reference's argument checks (std::invalid_argument for rows
// that are not 4-D / 3-D or weights of another length).
//
// Particles go to the library's device buffer (counted as they are added,
// as the reference counts them) and reach the grid when flush() runs:
// the host grid is uploaded, the GPU sorts and scatters the buffered
// particles, and the grid is downloaded again.  With buffer_size 0 (the
// reference's "add directly to the grid" mode) each array add ends with
// that step.  buffer_size > 0 does not trigger flushes part way: the grid
// is complete after flush(), as in the reference, without a transfer per
// buffer's worth of particles.  Particles added one at a time are staged
// on the host and passed to the device in batches.
#ifndef FFTCORR_CC_MASS_ASSIGNOR_H
#define FFTCORR_CC_MASS_ASSIGNOR_H

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "../array/row_major_array.h"
#include "../fc_check.h"
#include "../grid/config_space_grid.h"
#include "../types.h"
#include "distribution_functions.h"

class MassAssignor {
 public:
  MassAssignor(ConfigSpaceGrid &grid, DistributionScheme distribution_scheme,
               bool periodic_wrap, int buffer_size)
      : grid_(grid), buffer_size_(buffer_size) {
    if (buffer_size < 0) throw std::invalid_argument("buffer_size must be >= 0");
    fftcorr_cc::fc_check(
        fc_assignor_create(grid.fc_handle(), (int)distribution_scheme,
                           periodic_wrap ? 1 : 0, kDeviceBuffer, &ma_),
        "MassAssignor");
  }
  ~MassAssignor() { fc_assignor_destroy(ma_); }
  MassAssignor(const MassAssignor &) = delete;
  MassAssignor &operator=(const MassAssignor &) = delete;

  int buffer_size() const { return buffer_size_; }
  uint64 num_added() { return stats().num_added; }
  uint64 num_skipped() { return stats().num_skipped; }
  Float totw() { return stats().totw; }
  Float totwsq() { return stats().totwsq; }
  Float sort_time() { return stats().sort_time; }
  Float window_time() { return stats().window_time; }

  void clear() {
    staged_.clear();
    pending_ = 0;
    fftcorr_cc::fc_check(fc_assignor_clear(ma_), "MassAssignor::clear");
  }

  void add_particles_to_buffer(const RowMajorArrayPtr<Float, 2> &posw) {
    if (posw.shape(1) != 4) throw std::invalid_argument("Rows must be 4D.");
    add_rows(posw.data(), nullptr, 0.0, posw.shape(0), 4);
  }
  void add_particles_to_buffer(const RowMajorArrayPtr<Float, 2> &pos,
                               const RowMajorArrayPtr<Float, 1> &weights) {
    if (pos.shape(1) != 3) throw std::invalid_argument("Rows must be 3D.");
    if (pos.shape(0) != weights.shape(0))
      throw std::invalid_argument("Positions and weights must be same length");
    add_rows(pos.data(), weights.data(), 0.0, pos.shape(0), 3);
  }
  void add_particles_to_buffer(const RowMajorArrayPtr<Float, 2> &pos,
                               Float weight) {
    if (pos.shape(1) != 3) throw std::invalid_argument("Rows must be 3D.");
    add_rows(pos.data(), nullptr, weight, pos.shape(0), 3);
  }
  void add_particle_to_buffer(const Float *pos, Float w) {
    staged_.insert(staged_.end(), {pos[0], pos[1], pos[2], w});
    if (staged_.size() >= 4 * kStageRows) push_staged();
  }

  // Applies every buffered particle to the grid (mass_assignor.h:127-191).
  void flush() {
    push_staged();
    if (pending_ == 0) return;
    grid_.upload();
    fftcorr_cc::fc_check(fc_assignor_flush(ma_), "MassAssignor::flush");
    grid_.download();
    pending_ = 0;
  }

 private:
  // Particles the device buffer holds between flushes (the library then
  // never flushes on its own, so the host grid stays in step).
  static constexpr int64_t kDeviceBuffer = int64_t(1) << 28;
  static constexpr int64_t kPiece = int64_t(1) << 26;
  static constexpr size_t kStageRows = size_t(1) << 20;

  // Rows of (x, y, z[, w]) with per-row weights, a weight array or one
  // weight for all, passed to the device buffer in pieces.
  void add_rows(const Float *rows, const Float *weights, Float weight,
                int64_t n, int cols) {
    push_staged();
    for (int64_t done = 0; done < n;) {
      const int64_t m = n - done < kPiece ? n - done : kPiece;
      reserve(m);
      const Float *r = rows + (size_t)done * cols;
      int rc;
      if (cols == 4)
        rc = fc_assignor_add_posw(ma_, r, m);
      else if (weights)
        rc = fc_assignor_add_pos_weights(ma_, r, weights + done, m);
      else
        rc = fc_assignor_add_pos_weight(ma_, r, weight, m);
      fftcorr_cc::fc_check(rc, "MassAssignor::add_particles_to_buffer");
      pending_ += m;
      done += m;
    }
    if (buffer_size_ == 0) flush();
  }

  void push_staged() {
    if (staged_.empty()) return;
    const int64_t m = (int64_t)(staged_.size() / 4);
    reserve(m);
    fftcorr_cc::fc_check(fc_assignor_add_posw(ma_, staged_.data(), m),
                         "MassAssignor::add_particle_to_buffer");
    pending_ += m;
    staged_.clear();
  }

  // Flushes first if m more particles would fill the device buffer.
  void reserve(int64_t m) {
    if (pending_ > 0 && pending_ + m >= kDeviceBuffer) {
      grid_.upload();
      fftcorr_cc::fc_check(fc_assignor_flush(ma_), "MassAssignor::flush");
      grid_.download();
      pending_ = 0;
    }
  }

  fc_assign_stats stats() {
    push_staged();
    fc_assign_stats s;
    fftcorr_cc::fc_check(fc_assignor_stats(ma_, &s), "MassAssignor stats");
    return s;
  }

  ConfigSpaceGrid &grid_;
  int buffer_size_;
  fc_assignor *ma_ = nullptr;
  int64_t pending_ = 0;         // particles in the device buffer
  std::vector<Float> staged_;   // single particles not yet on the device
};

#endif  // FFTCORR_CC_MASS_ASSIGNOR_H
