// fc_hist.cuh -- deterministic FP64 histograms over fixed bin assignments.
//
// HistogramList::accumulate (cc/histogram/histogram_list.h:33-45) adds y to
// bin floor((x - min)/binsize) and counts it.  On the GPU the bin of every
// element is known before the values are (for the correlator subgrids it
// depends only on the geometry), so a BinIndex sorts element indices by bin
// once with a stable radix sort and splits each bin into fixed chunks.  A
// histogram pass is then a gather through that permutation, one fixed-shape
// tree reduction per chunk (warp shuffles + shared memory), and a per-bin
// fold of the chunk partials in chunk order: no floating-point atomics, the
// same bits on every run, and exact integer counts.
#pragma once

#include <vector>

#include "fc_common.cuh"

namespace fc {

// Values per histogram chunk (one CTA each).
constexpr int kHistChunk = 2048;
// Threads of a chunk reduction: part of the summation order, so fixed.
constexpr int kHistThreads = 256;

// One chunk of a histogram reduction: the sum of values[perm[start ..
// start + len)] (k_chunk_sums' fixed tree) goes to partials[item index].
struct HistItem {
  const double *values;
  const uint32_t *perm;
  uint32_t start;
  int len;
};
// One bin: *dest = sum of partials[first .. first + count) in order.
struct FoldItem {
  int first;
  int count;
  double *dest;
};

struct BinIndex {
  int nbins = 0;
  int64_t nelems = 0;     // elements indexed (all, in range or not)
  int64_t ninrange = 0;   // elements whose bin is in [0, nbins)
  int nchunks = 0;
  std::vector<int> counts;          // elements per bin
  DeviceBuffer perm;                // uint32 element ids sorted by bin
  DeviceBuffer chunk_start;         // uint32 offset into perm per chunk
  DeviceBuffer chunk_len;           // int per chunk
  DeviceBuffer chunk_first;         // int per bin + 1: first chunk of bin
  DeviceBuffer partials;            // double per chunk
  std::vector<uint32_t> h_chunk_start;  // host copies of the chunk table
  std::vector<int> h_chunk_len, h_chunk_first;

  // Builds the index from device bin ids (values outside [0, nbins) are
  // excluded).  bins_dev is clobbered.  Synchronises the stream.
  void build(int *bins_dev, int64_t n, int nbins_, cudaStream_t s);

  // hist_row[b] = sum over elements e of bin b of values[e] (overwrites).
  void reduce(const double *values, double *hist_row, cudaStream_t s) const;
  // hist_row[b] += that sum.
  void reduce_add(const double *values, double *hist_row,
                  cudaStream_t s) const;
  // Appends the work of reduce(values, hist_row) as chunk and fold items
  // (the same sums in the same order).
  void append_work(const double *values, double *hist_row,
                   std::vector<HistItem> &items,
                   std::vector<FoldItem> &folds) const;
};

// Bin index of value v for HistogramList(minval, binsize, nbins); -1 when
// outside [0, nbins).  Uses explicitly rounded FP64 operations so the result
// is the reference's floor((v - minval) / binsize) bit for bit.
__device__ __forceinline__ int bin_of(double v, double minval, double binsize,
                                      int nbins) {
  const double q = __ddiv_rn(__dsub_rn(v, minval), binsize);
  const double f = floor(q);
  if (!(f >= 0.0) || f >= (double)nbins) return -1;
  return (int)f;
}

// sqrt(a*a + b*b + c*c) rounded as the reference's row[k] = sqrt(...)
// (correlator.h:131, 184): products, then left-to-right sums, then sqrt.
__device__ __forceinline__ double norm3(double a, double b, double c) {
  return __dsqrt_rn(
      __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c)));
}

}  // namespace fc
