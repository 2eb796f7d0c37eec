// fc_core.cu -- error state, device selection, ConfigSpaceGrid and the
// array_ops reductions of the fftcorr_b200 library.
//
// ConfigSpaceGrid mirrors cc/grid/config_space_grid.h:10-57 with the grid in
// HBM; sum/sumsq/add_scalar/multiply_by mirror cc/array/array_ops.cc:55-137.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>

#include <cuda_profiler_api.h>

#include "fc_common.cuh"
#include "fc_internal.h"

namespace fc {

namespace {
thread_local std::string t_last_error;
}

void set_last_error(const std::string &msg) { t_last_error = msg; }

const char *last_error_cstr() { return t_last_error.c_str(); }

std::atomic<unsigned long long> &launch_counter() {
  static std::atomic<unsigned long long> n{0};
  return n;
}

void note_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }

int sm_count() {
  int dev = 0;
  cudaGetDevice(&dev);
  static int cached[64] = {0};
  if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
  int n = 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
      cudaSuccess)
    n = 148;
  if (dev >= 0 && dev < 64) cached[dev] = n;
  return n;
}

YlmParams make_ylm_params(int ell, int m, double coeff) {
  // spherical_harmonics.h:36-38 validity checks.
  if (!(ell == 0 || ell == 2 || ell == 4))
    FC_THROW(FC_ERR_INVALID, "Unsupported ell");
  if (m < -ell || m > ell) FC_THROW(FC_ERR_INVALID, "Illegal (ell, m)");
  YlmParams p;
  p.ell = ell;
  p.m = m;
  // spherical_harmonics.h:52 (ell = 0 shortcut) and :85-87.
  p.value0 = coeff / sqrt(4.0 * M_PI);
  double isqpi = sqrt(1.0 / M_PI);
  isqpi *= coeff;
  if (m != 0) isqpi *= sqrt(2.0);
  p.isqpi = isqpi;
  // The (ell, m) constant of each real-form Y_lm (spherical_harmonics.h:
  // 107-176), folded with isqpi for the FP32 evaluator.
  double c = 1.0;
  if (ell == 2) {
    c = m == 2 ? sqrt(15.0 / 32.0) : m == 0 ? sqrt(5.0 / 16.0) : sqrt(15.0 / 8.0);
  } else if (ell == 4) {
    switch (m < 0 ? -m : m) {
      case 4: c = 3.0 / 16.0 * sqrt(35.0 / 2.0); break;
      case 3: c = 3.0 / 8.0 * sqrt(35.0); break;
      case 2: c = 3.0 / 8.0 * sqrt(5.0 / 2.0); break;
      case 1: c = 3.0 / 8.0 * sqrt(5.0) * 3.0; break;
      default: c = 3.0 / 16.0 * 8.0; break;
    }
  }
  p.norm = isqpi * c;
  return p;
}

// --------------------------------------------------------------- kernels

namespace {

__global__ void k_fill(double *a, size_t n, double v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = v;
}

// Grid arithmetic in FP64 per cell, rounded once to the cell type.
template <typename T>
__global__ void k_add_scalar(T *a, size_t n, double s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = (T)((double)a[i] + s);
}

template <typename T>
__global__ void k_multiply_by(T *a, size_t n, double s) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    a[i] = (T)((double)a[i] * s);
}

template <typename TY, typename TX>
__global__ void k_axpy(TY *y, const TX *x, size_t n, double a) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (TY)((double)y[i] + a * (double)x[i]);
}

__global__ void k_widen(const float *in, double *out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// Pass 1 of the deterministic sum/sumsq: block b reduces the grid-stride
// subsequence it owns in a fixed order.
template <typename T>
__global__ void k_sum_partials(const T *a, size_t n, double *partials) {
  __shared__ double red[32];
  double s = 0.0, q = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double v = (double)a[i];
    s += v;
    q += v * v;
  }
  s = block_sum(s, red);
  q = block_sum(q, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = s;
    partials[2 * blockIdx.x + 1] = q;
  }
}

// Pass 2: one block folds the partials in block order.
__global__ void k_sum_final(const double *partials, int nparts, double *out) {
  __shared__ double red[32];
  double s = 0.0, q = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    s += partials[2 * i];
    q += partials[2 * i + 1];
  }
  s = block_sum(s, red);
  q = block_sum(q, red);
  if (threadIdx.x == 0) {
    out[0] = s;
    out[1] = q;
  }
}

}  // namespace

void device_fill(double *a, size_t n, double v, cudaStream_t s) {
  if (n == 0) return;
  k_fill<<<grid_for(n, 256), 256, 0, s>>>(a, n, v);
  FC_LAUNCH_CHECK();
}

template <typename T>
static void sum_sumsq(const T *a, size_t n, double *scratch, cudaStream_t s) {
  // scratch: 2 * kSumBlocks partials followed by the 2 results.
  k_sum_partials<T><<<kSumBlocks, 256, 0, s>>>(a, n, scratch);
  FC_LAUNCH_CHECK();
  k_sum_final<<<1, 256, 0, s>>>(scratch, kSumBlocks, scratch + 2 * kSumBlocks);
  FC_LAUNCH_CHECK();
}
void device_sum_sumsq(const double *a, size_t n, double *scratch,
                      cudaStream_t s) {
  sum_sumsq(a, n, scratch, s);
}
void device_sum_sumsq(const float *a, size_t n, double *scratch,
                      cudaStream_t s) {
  sum_sumsq(a, n, scratch, s);
}

void device_widen(const float *in, double *out, size_t n, cudaStream_t s) {
  if (n == 0) return;
  k_widen<<<grid_for(n, 256), 256, 0, s>>>(in, out, n);
  FC_LAUNCH_CHECK();
}

// ------------------------------------------------------- fault injection

namespace {
std::atomic<long long> g_fault_countdown[3];  // by FaultKind; <= 0: disarmed
std::atomic<long long> g_device_bytes{0};
std::atomic<unsigned long long> g_device_budget{0};  // 0: no budget
}  // namespace

bool fault_fires(int kind) {
  std::atomic<long long> &c = g_fault_countdown[kind];
  long long v = c.load();
  while (v > 0) {
    if (c.compare_exchange_weak(v, v - 1)) return v == 1;
  }
  return false;
}

void device_alloc_check(size_t bytes) {
  if (fault_fires(kFaultDeviceAlloc))
    FC_THROW(FC_ERR_ALLOC, "injected device allocation failure");
  const unsigned long long budget = g_device_budget.load();
  if (budget && (unsigned long long)g_device_bytes.load() + bytes > budget)
    FC_THROW(FC_ERR_ALLOC, "device memory budget exceeded (" +
                               std::to_string(bytes) + " more bytes)");
}

void device_bytes_add(long long delta) { g_device_bytes += delta; }

// ------------------------------------------------------------- the grid

Grid::Grid(const int shp[3], const double pmin[3], double cell, int prec) {
  FC_REQUIRE(prec == FC_FP64 || prec == FC_FP32_MIXED, FC_ERR_INVALID,
             "grid precision must be FC_FP64 or FC_FP32_MIXED");
  precision = prec;
  for (int i = 0; i < 3; ++i) {
    FC_REQUIRE(shp[i] > 0, FC_ERR_INVALID, "grid shape must be positive");
    shape[i] = shp[i];
    posmin[i] = pmin[i];
  }
  FC_REQUIRE(cell > 0, FC_ERR_INVALID, "cell_size must be positive");
  cell_size = cell;
  FC_CUDA(cudaGetDevice(&device));
  FC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  try {
    data.resize(size() * cell_bytes());
    scratch.resize((2 * kSumBlocks + 2) * sizeof(double));
    clear();
  } catch (...) {
    cudaStreamDestroy(stream);
    stream = nullptr;
    throw;
  }
}

Grid::~Grid() {
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
}

void Grid::clear() {
  FC_CUDA(cudaMemsetAsync(data.get(), 0, size() * cell_bytes(), stream));
}

}  // namespace fc

// ============================================================== C entry

using namespace fc;

extern "C" {

const char *fc_last_error(void) { return fc::last_error_cstr(); }

int fc_version(void) { return 10000 * 0 + 100 * 9 + 0; }

int fc_launch_count(unsigned long long *count) {
  return guard([&] {
    FC_REQUIRE(count, FC_ERR_INVALID, "null argument");
    *count = fc::launch_counter().load(std::memory_order_relaxed);
  });
}

int fc_profiler_range(int on) {
  return guard([&] {
    if (on)
      FC_CUDA(cudaProfilerStart());
    else
      FC_CUDA(cudaProfilerStop());
  });
}

int fc_set_device(int device) {
  return guard([&] { FC_CUDA(cudaSetDevice(device)); });
}

int fc_grid_create_precision(const int shape[3], const double posmin[3],
                             double cell_size, int precision, fc_grid **out) {
  return guard([&] {
    FC_REQUIRE(shape && posmin && out, FC_ERR_INVALID, "null argument");
    *out = nullptr;
    std::unique_ptr<Grid> g(new Grid(shape, posmin, cell_size, precision));
    FC_CUDA(cudaStreamSynchronize(g->stream));
    *out = reinterpret_cast<fc_grid *>(g.release());
  });
}

int fc_grid_create(const int shape[3], const double posmin[3],
                   double cell_size, fc_grid **out) {
  return fc_grid_create_precision(shape, posmin, cell_size, FC_FP64, out);
}

int fc_grid_precision(const fc_grid *grid, int *precision) {
  return guard([&] {
    FC_REQUIRE(precision, FC_ERR_INVALID, "null argument");
    *precision = as_grid(grid)->precision;
  });
}

int fc_grid_destroy(fc_grid *grid) {
  return guard([&] { delete reinterpret_cast<Grid *>(grid); });
}

int fc_grid_clear(fc_grid *grid) {
  return guard([&] {
    Grid *g = as_grid(grid);
    g->clear();
    FC_CUDA(cudaStreamSynchronize(g->stream));
  });
}

int fc_grid_upload(fc_grid *grid, const double *host) {
  return guard([&] {
    Grid *g = as_grid(grid);
    FC_REQUIRE(host, FC_ERR_INVALID, "null host pointer");
    if (g->fp32()) {
      // Rounded once per cell on the host, then copied.
      std::vector<float> tmp(g->size());
      for (size_t i = 0; i < tmp.size(); ++i) tmp[i] = (float)host[i];
      FC_CUDA(cudaMemcpyAsync(g->raw(), tmp.data(), tmp.size() * sizeof(float),
                              cudaMemcpyHostToDevice, g->stream));
      FC_CUDA(cudaStreamSynchronize(g->stream));
      return;
    }
    FC_CUDA(cudaMemcpyAsync(g->ptr(), host, g->size() * sizeof(double),
                            cudaMemcpyHostToDevice, g->stream));
    FC_CUDA(cudaStreamSynchronize(g->stream));
  });
}

int fc_grid_download(const fc_grid *grid, double *host) {
  return guard([&] {
    const Grid *g = as_grid(grid);
    FC_REQUIRE(host, FC_ERR_INVALID, "null host pointer");
    if (g->fp32()) {
      std::vector<float> tmp(g->size());
      FC_CUDA(cudaMemcpyAsync(tmp.data(), g->raw(), tmp.size() * sizeof(float),
                              cudaMemcpyDeviceToHost, g->stream));
      FC_CUDA(cudaStreamSynchronize(g->stream));
      for (size_t i = 0; i < tmp.size(); ++i) host[i] = (double)tmp[i];
      return;
    }
    FC_CUDA(cudaMemcpyAsync(host, g->ptr(), g->size() * sizeof(double),
                            cudaMemcpyDeviceToHost, g->stream));
    FC_CUDA(cudaStreamSynchronize(g->stream));
  });
}

int fc_grid_device_ptr(const fc_grid *grid, double **device_ptr) {
  return guard([&] {
    FC_REQUIRE(device_ptr, FC_ERR_INVALID, "null argument");
    *device_ptr = as_grid(grid)->ptr();
  });
}

int fc_grid_device_data(const fc_grid *grid, void **device_ptr) {
  return guard([&] {
    FC_REQUIRE(device_ptr, FC_ERR_INVALID, "null argument");
    *device_ptr = as_grid(grid)->raw();
  });
}

int fc_grid_coords(const fc_grid *grid, const double survey[3], int periodic,
                   double grid_coords[3], int *inside) {
  return guard([&] {
    const Grid *g = as_grid(grid);
    FC_REQUIRE(survey && grid_coords && inside, FC_ERR_INVALID,
               "null argument");
    *inside = host_grid_coords(survey, g->posmin, g->cell_size, g->shape,
                               periodic != 0, grid_coords)
                  ? 1
                  : 0;
  });
}

int fc_grid_sum(fc_grid *grid, double *sum, double *sumsq) {
  return guard([&] {
    Grid *g = as_grid(grid);
    double *scr = g->scratch.as<double>();
    if (g->fp32())
      device_sum_sumsq(static_cast<const float *>(g->raw()), g->size(), scr,
                       g->stream);
    else
      device_sum_sumsq(g->ptr(), g->size(), scr, g->stream);
    double res[2];
    FC_CUDA(cudaMemcpyAsync(res, scr + 2 * kSumBlocks, sizeof(res),
                            cudaMemcpyDeviceToHost, g->stream));
    FC_CUDA(cudaStreamSynchronize(g->stream));
    if (sum) *sum = res[0];
    if (sumsq) *sumsq = res[1];
  });
}

int fc_grid_add_scalar(fc_grid *grid, double s) {
  return guard([&] {
    Grid *g = as_grid(grid);
    if (g->fp32())
      k_add_scalar<<<grid_for(g->size(), 256), 256, 0, g->stream>>>(
          static_cast<float *>(g->raw()), g->size(), s);
    else
      k_add_scalar<<<grid_for(g->size(), 256), 256, 0, g->stream>>>(
          g->ptr(), g->size(), s);
    FC_LAUNCH_CHECK();
    FC_CUDA(cudaStreamSynchronize(g->stream));
  });
}

int fc_grid_multiply_by(fc_grid *grid, double s) {
  return guard([&] {
    Grid *g = as_grid(grid);
    if (g->fp32())
      k_multiply_by<<<grid_for(g->size(), 256), 256, 0, g->stream>>>(
          static_cast<float *>(g->raw()), g->size(), s);
    else
      k_multiply_by<<<grid_for(g->size(), 256), 256, 0, g->stream>>>(
          g->ptr(), g->size(), s);
    FC_LAUNCH_CHECK();
    FC_CUDA(cudaStreamSynchronize(g->stream));
  });
}

int fc_grid_axpy(fc_grid *y, double a, const fc_grid *x) {
  return guard([&] {
    Grid *gy = as_grid(y);
    const Grid *gx = as_grid(x);
    for (int i = 0; i < 3; ++i)
      FC_REQUIRE(gy->shape[i] == gx->shape[i], FC_ERR_INVALID,
                 "Incompatible shapes for axpy.");
    // Order after any pending work on x's stream.
    cudaEvent_t ev;
    FC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaEventRecord(ev, gx->stream);
    cudaStreamWaitEvent(gy->stream, ev, 0);
    cudaEventDestroy(ev);
    const unsigned nb = grid_for(gy->size(), 256);
    const size_t n = gy->size();
    float *y32 = static_cast<float *>(gy->raw());
    const float *x32 = static_cast<const float *>(gx->raw());
    double *y64 = static_cast<double *>(gy->raw());
    const double *x64 = static_cast<const double *>(gx->raw());
    if (gy->fp32() && gx->fp32())
      k_axpy<<<nb, 256, 0, gy->stream>>>(y32, x32, n, a);
    else if (gy->fp32())
      k_axpy<<<nb, 256, 0, gy->stream>>>(y32, x64, n, a);
    else if (gx->fp32())
      k_axpy<<<nb, 256, 0, gy->stream>>>(y64, x32, n, a);
    else
      k_axpy<<<nb, 256, 0, gy->stream>>>(y64, x64, n, a);
    FC_LAUNCH_CHECK();
    FC_CUDA(cudaStreamSynchronize(gy->stream));
  });
}

}  // extern "C"

// ============================================= allocation-free reduction

namespace fc {
namespace {

// Elements per block of the allocation-free reduction: block b sums
// [b * kStaticSeg, (b + 1) * kStaticSeg) in a fixed order.
constexpr int64_t kStaticSeg = 1 << 18;
constexpr int kStaticParts = 4096;  // FC_SUM_STATIC_MAX_N / kStaticSeg

// Scratch of fc_sum_sumsq_static: kStaticParts (sum, sumsq) partials and
// the two results, 64 KiB + 16 B.  Host code must not use this name as an
// address; it uses the device address looked up below.
static __device__ __align__(256) double g_static_scratch[2 * kStaticParts + 2];

__global__ void k_seg_partials(const double *a, int64_t n, double *partials) {
  __shared__ double red[32];
  const int64_t lo = (int64_t)blockIdx.x * kStaticSeg;
  const int64_t hi = lo + kStaticSeg < n ? lo + kStaticSeg : n;
  double s = 0.0, q = 0.0;
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    const double v = a[i];
    s += v;
    q += v * v;
  }
  s = block_sum(s, red);
  q = block_sum(q, red);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = s;
    partials[2 * blockIdx.x + 1] = q;
  }
}

// Device address of g_static_scratch in the current device's context, looked
// up on every call (a cheap query): a cached address would go stale if the
// context were torn down and created again (cudaDeviceReset), which reloads
// the module.
double *static_scratch() {
  void *p = nullptr;
  FC_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
  return static_cast<double *>(p);
}

}  // namespace
}  // namespace fc

extern "C" int fc_sum_sumsq_static(const double *device_data, int64_t n,
                                   double *sum, double *sumsq) {
  using namespace fc;
  return guard([&] {
    FC_REQUIRE(n >= 0, FC_ERR_INVALID, "n must be non-negative");
    FC_REQUIRE(n <= FC_SUM_STATIC_MAX_N, FC_ERR_RANGE,
               "n exceeds FC_SUM_STATIC_MAX_N (2^30 values), the capacity of "
               "the fixed scratch array");
    FC_REQUIRE(device_data || n == 0, FC_ERR_INVALID, "null device pointer");
    double *scr = static_scratch();
    const int blocks = (int)((n + kStaticSeg - 1) / kStaticSeg);
    cudaStream_t s = 0;
    if (blocks > 0) {
      k_seg_partials<<<blocks, 256, 0, s>>>(device_data, n, scr);
      FC_LAUNCH_CHECK();
      k_sum_final<<<1, 256, 0, s>>>(scr, blocks, scr + 2 * kStaticParts);
      FC_LAUNCH_CHECK();
    } else {
      FC_CUDA(cudaMemsetAsync(scr + 2 * kStaticParts, 0, 2 * sizeof(double), s));
    }
    double res[2];
    FC_CUDA(cudaMemcpyAsync(res, scr + 2 * kStaticParts, sizeof(res),
                            cudaMemcpyDeviceToHost, s));
    FC_CUDA(cudaStreamSynchronize(s));
    if (sum) *sum = res[0];
    if (sumsq) *sumsq = res[1];
  });
}

// ============================================================ utilities

namespace {
struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
};
}  // namespace

extern "C" {

int fc_device_synchronize(void) {
  return guard([&] { FC_CUDA(cudaDeviceSynchronize()); });
}

int fc_host_register(void *ptr, size_t bytes) {
  return guard([&] {
    FC_REQUIRE(ptr, FC_ERR_INVALID, "null pointer");
    FC_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  });
}

int fc_host_unregister(void *ptr) {
  return guard([&] { FC_CUDA(cudaHostUnregister(ptr)); });
}

int fc_device_malloc(size_t bytes, void **ptr) {
  return guard([&] {
    FC_REQUIRE(ptr, FC_ERR_INVALID, "null pointer");
    *ptr = nullptr;
    FC_CUDA(cudaMalloc(ptr, bytes));
  });
}

int fc_fault_inject(int kind, int64_t n) {
  return guard([&] {
    FC_REQUIRE(kind == FC_FAULT_DEVICE_ALLOC || kind == FC_FAULT_FFT_PLAN,
               FC_ERR_INVALID, "unknown fault kind");
    g_fault_countdown[kind].store(n > 0 ? (long long)n : 0);
  });
}

int fc_set_device_budget(size_t bytes) {
  return guard([&] { g_device_budget.store(bytes); });
}

int fc_device_bytes(size_t *bytes) {
  return guard([&] {
    FC_REQUIRE(bytes, FC_ERR_INVALID, "null argument");
    const long long b = g_device_bytes.load();
    *bytes = b > 0 ? (size_t)b : 0;
  });
}

int fc_device_free(void *ptr) {
  return guard([&] { FC_CUDA(cudaFree(ptr)); });
}

int fc_memcpy_htod(void *dst, const void *src, size_t bytes) {
  return guard([&] {
    FC_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  });
}

int fc_device_memory(size_t *free_bytes, size_t *total_bytes) {
  return guard([&] {
    size_t f = 0, t = 0;
    FC_CUDA(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
  });
}

int fc_memcpy_dtoh(void *dst, const void *src, size_t bytes) {
  return guard([&] {
    FC_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
  });
}

int fc_timer_create(fc_timer **t) {
  return guard([&] {
    FC_REQUIRE(t, FC_ERR_INVALID, "null pointer");
    Timer *x = new Timer;
    FC_CUDA(cudaEventCreate(&x->a));
    FC_CUDA(cudaEventCreate(&x->b));
    *t = reinterpret_cast<fc_timer *>(x);
  });
}

int fc_timer_start(fc_timer *t) {
  return guard([&] {
    FC_REQUIRE(t, FC_ERR_INVALID, "null timer");
    Timer *x = reinterpret_cast<Timer *>(t);
    FC_CUDA(cudaDeviceSynchronize());
    FC_CUDA(cudaEventRecord(x->a, 0));
  });
}

int fc_timer_stop(fc_timer *t, double *seconds) {
  return guard([&] {
    FC_REQUIRE(t && seconds, FC_ERR_INVALID, "null argument");
    Timer *x = reinterpret_cast<Timer *>(t);
    FC_CUDA(cudaDeviceSynchronize());
    FC_CUDA(cudaEventRecord(x->b, 0));
    FC_CUDA(cudaEventSynchronize(x->b));
    float ms = 0.f;
    FC_CUDA(cudaEventElapsedTime(&ms, x->a, x->b));
    *seconds = ms * 1e-3;
  });
}

int fc_timer_destroy(fc_timer *t) {
  return guard([&] {
    Timer *x = reinterpret_cast<Timer *>(t);
    if (!x) return;
    if (x->a) cudaEventDestroy(x->a);
    if (x->b) cudaEventDestroy(x->b);
    delete x;
  });
}

}  // extern "C"
