// fc_hist.cu -- BinIndex (deterministic segmented histogram reduction) and
// the HistogramList C entry points (cc/histogram/histogram_list.h:10-68).
#include <cub/cub.cuh>

#include <cmath>

#include "fc_hist.cuh"
#include "fc_internal.h"

namespace fc {
namespace {

__global__ void k_iota_and_key(int *bins, uint32_t *ids, int64_t n,
                               int nbins) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int b = bins[i];
    bins[i] = (b < 0 || b >= nbins) ? nbins : b;  // out of range sorts last
    ids[i] = (uint32_t)i;
  }
}

// first[b] = lower_bound(sorted_bins, b) for b in [0, nbins].
__global__ void k_bin_starts(const int *sorted_bins, int64_t n, int nbins,
                             int64_t *first) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= nbins;
       b += gridDim.x * blockDim.x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (sorted_bins[mid] < b)
        lo = mid + 1;
      else
        hi = mid;
    }
    first[b] = lo;
  }
}

// One CTA per chunk: fixed-tree sum of the chunk's gathered values.
__global__ void __launch_bounds__(256)
    k_chunk_sums(const double *__restrict__ values,
                 const uint32_t *__restrict__ perm,
                 const uint32_t *__restrict__ chunk_start,
                 const int *__restrict__ chunk_len, double *partials) {
  __shared__ double red[32];
  const uint32_t s = chunk_start[blockIdx.x];
  const int len = chunk_len[blockIdx.x];
  double acc = 0.0;
  for (int i = threadIdx.x; i < len; i += blockDim.x) acc += values[perm[s + i]];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

// One thread per bin: chunk partials folded in chunk order.
__global__ void k_bin_fold(const double *partials, const int *chunk_first,
                           int nbins, double *hist_row, int add) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbins;
       b += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int c = chunk_first[b]; c < chunk_first[b + 1]; ++c) s += partials[c];
    hist_row[b] = add ? hist_row[b] + s : s;
  }
}

__global__ void k_value_bins(const double *x, int64_t n, double minval,
                             double binsize, int nbins, int *bins) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    bins[i] = bin_of(x[i], minval, binsize, nbins);
}

}  // namespace

void BinIndex::build(int *bins_dev, int64_t n, int nbins_, cudaStream_t s) {
  nbins = nbins_;
  nelems = n;
  FC_REQUIRE(n < (int64_t)0xffffffffll, FC_ERR_INVALID,
             "histogram input too large (limit 2^32-1 values)");
  DeviceBuffer ids(n * sizeof(uint32_t) + 16);
  DeviceBuffer bins_alt(n * sizeof(int) + 16);
  DeviceBuffer ids_alt(n * sizeof(uint32_t) + 16);
  if (n > 0) {
    k_iota_and_key<<<grid_for(n, 256), 256, 0, s>>>(bins_dev, ids.as<uint32_t>(),
                                                    n, nbins);
    FC_LAUNCH_CHECK();
  }
  int end_bit = 1;
  while ((nbins >> end_bit) != 0) ++end_bit;
  // Bins are non-negative after k_iota_and_key; sort them as unsigned.
  cub::DoubleBuffer<uint32_t> dk(reinterpret_cast<uint32_t *>(bins_dev),
                                 bins_alt.as<uint32_t>());
  cub::DoubleBuffer<uint32_t> dv(ids.as<uint32_t>(), ids_alt.as<uint32_t>());
  size_t temp = 0;
  if (n > 0) {
    FC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, dk, dv, n, 0,
                                            end_bit, s));
    DeviceBuffer tmp(temp + 16);
    FC_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), temp, dk, dv, n, 0,
                                            end_bit, s));
  }
  DeviceBuffer first((nbins + 1) * sizeof(int64_t));
  k_bin_starts<<<grid_for(nbins + 1, 128), 128, 0, s>>>(
      n > 0 ? reinterpret_cast<const int *>(dk.Current()) : bins_dev, n, nbins,
      first.as<int64_t>());
  FC_LAUNCH_CHECK();
  std::vector<int64_t> h_first(nbins + 1);
  FC_CUDA(cudaMemcpyAsync(h_first.data(), first.get(),
                          (nbins + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                          s));
  FC_CUDA(cudaStreamSynchronize(s));
  ninrange = h_first[nbins];
  counts.assign(nbins, 0);
  std::vector<uint32_t> cs;
  std::vector<int> cl;
  std::vector<int> cf(nbins + 1, 0);
  for (int b = 0; b < nbins; ++b) {
    counts[b] = (int)(h_first[b + 1] - h_first[b]);
    cf[b] = (int)cs.size();
    for (int64_t o = h_first[b]; o < h_first[b + 1]; o += kHistChunk) {
      cs.push_back((uint32_t)o);
      cl.push_back((int)std::min<int64_t>(kHistChunk, h_first[b + 1] - o));
    }
  }
  cf[nbins] = (int)cs.size();
  nchunks = (int)cs.size();
  h_chunk_start = cs;
  h_chunk_len = cl;
  h_chunk_first = cf;
  perm.resize(std::max<int64_t>(ninrange, 1) * sizeof(uint32_t));
  if (ninrange > 0)
    FC_CUDA(cudaMemcpyAsync(perm.get(), dv.Current(),
                            ninrange * sizeof(uint32_t),
                            cudaMemcpyDeviceToDevice, s));
  chunk_start.resize(std::max(nchunks, 1) * sizeof(uint32_t));
  chunk_len.resize(std::max(nchunks, 1) * sizeof(int));
  chunk_first.resize((nbins + 1) * sizeof(int));
  partials.resize(std::max(nchunks, 1) * sizeof(double));
  if (nchunks > 0) {
    FC_CUDA(cudaMemcpyAsync(chunk_start.get(), cs.data(),
                            nchunks * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            s));
    FC_CUDA(cudaMemcpyAsync(chunk_len.get(), cl.data(), nchunks * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  }
  FC_CUDA(cudaMemcpyAsync(chunk_first.get(), cf.data(), (nbins + 1) * sizeof(int),
                          cudaMemcpyHostToDevice, s));
  FC_CUDA(cudaStreamSynchronize(s));
}

void BinIndex::reduce(const double *values, double *hist_row,
                      cudaStream_t s) const {
  if (nchunks > 0) {
    k_chunk_sums<<<nchunks, kHistThreads, 0, s>>>(values, perm.as<uint32_t>(),
                                         chunk_start.as<uint32_t>(),
                                         chunk_len.as<int>(),
                                         partials.as<double>());
    FC_LAUNCH_CHECK();
  }
  if (nbins > 0) {
    k_bin_fold<<<grid_for(nbins, 128), 128, 0, s>>>(
        partials.as<double>(), chunk_first.as<int>(), nbins, hist_row, 0);
    FC_LAUNCH_CHECK();
  }
}

void BinIndex::reduce_add(const double *values, double *hist_row,
                          cudaStream_t s) const {
  if (nchunks > 0) {
    k_chunk_sums<<<nchunks, kHistThreads, 0, s>>>(values, perm.as<uint32_t>(),
                                         chunk_start.as<uint32_t>(),
                                         chunk_len.as<int>(),
                                         partials.as<double>());
    FC_LAUNCH_CHECK();
  }
  if (nbins > 0) {
    k_bin_fold<<<grid_for(nbins, 128), 128, 0, s>>>(
        partials.as<double>(), chunk_first.as<int>(), nbins, hist_row, 1);
    FC_LAUNCH_CHECK();
  }
}

void BinIndex::append_work(const double *values, double *hist_row,
                           std::vector<HistItem> &items,
                           std::vector<FoldItem> &folds) const {
  const int base = (int)items.size();
  for (int c = 0; c < nchunks; ++c)
    items.push_back(HistItem{values, perm.as<uint32_t>(), h_chunk_start[c],
                             h_chunk_len[c]});
  for (int b = 0; b < nbins; ++b)
    folds.push_back(FoldItem{base + h_chunk_first[b],
                             h_chunk_first[b + 1] - h_chunk_first[b],
                             hist_row + b});
}

// HistogramList with its counts and sums in device memory.
struct Hist {
  int n;
  double minval, binsize;
  int nbins;
  std::vector<double> bins;
  std::vector<int> counts;  // host, exact
  DeviceBuffer hist;        // n x nbins doubles
  cudaStream_t stream = nullptr;

  Hist(int n_, double minval_, double maxval, double binsize_)
      : n(n_), minval(minval_), binsize(binsize_) {
    // histogram_list.h:12-26 (validated before the bin count is formed).
    FC_REQUIRE(n > 0, FC_ERR_INVALID, "n must be positive.");
    FC_REQUIRE(minval < maxval, FC_ERR_INVALID,
               "maxval must be greater than minval.");
    FC_REQUIRE(binsize > 0, FC_ERR_INVALID, "binsize must be positive.");
    nbins = (int)floor((maxval - minval) / binsize);
    bins.resize(nbins);
    for (int i = 0; i < nbins; ++i) bins[i] = minval + (i + 0.5) * binsize;
    counts.assign((size_t)n * nbins, 0);
    FC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    hist.resize(std::max<size_t>((size_t)n * nbins, 1) * sizeof(double));
    reset();
  }
  ~Hist() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
  }
  void reset() {
    std::fill(counts.begin(), counts.end(), 0);
    FC_CUDA(cudaMemsetAsync(hist.get(), 0, hist.bytes(), stream));
    FC_CUDA(cudaStreamSynchronize(stream));
  }
  void accumulate(int ih, const double *x, const double *y, int64_t len) {
    FC_REQUIRE(ih >= 0 && ih < n, FC_ERR_RANGE, "ih out of range.");
    if (len == 0) return;
    DeviceBuffer dx(len * sizeof(double)), dy(len * sizeof(double));
    DeviceBuffer db(len * sizeof(int) + 16);
    FC_CUDA(cudaMemcpyAsync(dx.get(), x, len * sizeof(double),
                            cudaMemcpyHostToDevice, stream));
    FC_CUDA(cudaMemcpyAsync(dy.get(), y, len * sizeof(double),
                            cudaMemcpyHostToDevice, stream));
    k_value_bins<<<grid_for(len, 256), 256, 0, stream>>>(
        dx.as<double>(), len, minval, binsize, nbins, db.as<int>());
    FC_LAUNCH_CHECK();
    BinIndex idx;
    idx.build(db.as<int>(), len, nbins, stream);
    idx.reduce_add(dy.as<double>(), hist.as<double>() + (size_t)ih * nbins,
                   stream);
    FC_CUDA(cudaStreamSynchronize(stream));
    for (int b = 0; b < nbins; ++b) counts[(size_t)ih * nbins + b] += idx.counts[b];
  }
};

}  // namespace fc

using namespace fc;

extern "C" {

int fc_hist_create(int n, double minval, double maxval, double binsize,
                   fc_hist **out) {
  return guard([&] {
    FC_REQUIRE(out, FC_ERR_INVALID, "null argument");
    *out = reinterpret_cast<fc_hist *>(new Hist(n, minval, maxval, binsize));
  });
}

int fc_hist_destroy(fc_hist *h) {
  return guard([&] { delete reinterpret_cast<Hist *>(h); });
}

int fc_hist_nbins(const fc_hist *h, int *nbins) {
  return guard([&] {
    FC_REQUIRE(h && nbins, FC_ERR_INVALID, "null argument");
    *nbins = reinterpret_cast<const Hist *>(h)->nbins;
  });
}

int fc_hist_accumulate(fc_hist *h, int ih, const double *x, const double *y,
                       int64_t len) {
  return guard([&] {
    FC_REQUIRE(h, FC_ERR_INVALID, "null histogram handle");
    FC_REQUIRE((x && y) || len == 0, FC_ERR_INVALID, "null value array");
    reinterpret_cast<Hist *>(h)->accumulate(ih, x, y, len);
  });
}

int fc_hist_reset(fc_hist *h) {
  return guard([&] {
    FC_REQUIRE(h, FC_ERR_INVALID, "null histogram handle");
    reinterpret_cast<Hist *>(h)->reset();
  });
}

int fc_hist_get(const fc_hist *h, double *bins, int *counts, double *hist) {
  return guard([&] {
    FC_REQUIRE(h, FC_ERR_INVALID, "null histogram handle");
    const Hist *H = reinterpret_cast<const Hist *>(h);
    if (bins) std::copy(H->bins.begin(), H->bins.end(), bins);
    if (counts) std::copy(H->counts.begin(), H->counts.end(), counts);
    if (hist) {
      FC_CUDA(cudaMemcpyAsync(hist, H->hist.get(),
                              (size_t)H->n * H->nbins * sizeof(double),
                              cudaMemcpyDeviceToHost, H->stream));
      FC_CUDA(cudaStreamSynchronize(H->stream));
    }
  });
}

}  // extern "C"
