// row_major_array.h -- N-dimensional row-major views and owning arrays.
//
// The interface of the reference's cc/array/row_major_array.h and
// cc/array/array_nd.h that the Cython package binds to
// (fftcorr/array/row_major_array.pxd:5-10, fftcorr/array/numpy_adaptor.h):
//   RowMajorArrayPtr<dtype, N>()                     empty view
//   RowMajorArrayPtr<dtype, N>(std::array<int, N>, dtype *)
//   set_data(shape, data), shape(), shape(i), size(), data(), at(i, ...),
//   get_row(i, ...) and, for N = 1, operator[].
// RowMajorArray<dtype, N> owns its storage (zero-initialised).  These are
// host arrays: the device side lives behind the C ABI (fc_api.h).
#ifndef FFTCORR_CC_ROW_MAJOR_ARRAY_H
#define FFTCORR_CC_ROW_MAJOR_ARRAY_H

#include <array>
#include <stdexcept>
#include <vector>

#include "../types.h"
#include "array.h"

template <typename dtype, std::size_t N>
class RowMajorArrayPtr : public Array<dtype> {
 public:
  RowMajorArrayPtr() : data_(nullptr), size_(0) { shape_.fill(0); }
  RowMajorArrayPtr(const std::array<int, N> &shape, dtype *data) {
    set_data(shape, data);
  }

  void set_data(const std::array<int, N> &shape, dtype *data) {
    shape_ = shape;
    size_ = 1;
    for (int n : shape_) {
      if (n < 0) throw std::invalid_argument("negative array dimension");
      size_ *= (uint64)n;
    }
    data_ = data;
  }

  const std::array<int, N> &shape() const { return shape_; }
  int shape(int i) const { return shape_[i]; }
  uint64 size() const override { return size_; }
  dtype *data() override { return data_; }
  const dtype *data() const override { return data_; }

  // Row-major element access: at(i0, ..., i{N-1}).
  template <typename... I>
  dtype &at(I... idx) {
    return data_[index(idx...)];
  }
  template <typename... I>
  const dtype &at(I... idx) const {
    return data_[index(idx...)];
  }
  // First element of the row with the leading N-1 indices given.
  template <typename... I>
  dtype *get_row(I... idx) {
    return &data_[index(idx..., 0)];
  }
  template <typename... I>
  const dtype *get_row(I... idx) const {
    return &data_[index(idx..., 0)];
  }
  dtype &operator[](uint64 i) { return data_[i]; }
  const dtype &operator[](uint64 i) const { return data_[i]; }

 protected:
  template <typename... I>
  uint64 index(I... idx) const {
    static_assert(sizeof...(I) == N, "one index per dimension");
    const int ii[] = {static_cast<int>(idx)...};
    uint64 k = 0;
    for (std::size_t d = 0; d < N; ++d) k = k * (uint64)shape_[d] + (uint64)ii[d];
    return k;
  }

  std::array<int, N> shape_;
  dtype *data_;
  uint64 size_;
};

template <typename dtype, std::size_t N>
class RowMajorArray : public RowMajorArrayPtr<dtype, N> {
 public:
  RowMajorArray() = default;
  explicit RowMajorArray(const std::array<int, N> &shape) { allocate(shape); }
  RowMajorArray(const RowMajorArray &) = delete;
  RowMajorArray &operator=(const RowMajorArray &) = delete;

  void allocate(const std::array<int, N> &shape) {
    uint64 n = 1;
    for (int d : shape) n *= (uint64)(d > 0 ? d : 0);
    store_.assign(n, dtype());
    this->set_data(shape, store_.data());
  }

 private:
  std::vector<dtype> store_;
};

template <typename dtype>
class Array1D : public RowMajorArray<dtype, 1> {
 public:
  Array1D() = default;
  explicit Array1D(int n) { this->allocate({n}); }
};

#endif  // FFTCORR_CC_ROW_MAJOR_ARRAY_H
