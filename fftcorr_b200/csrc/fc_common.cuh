// fc_common.cuh -- shared plumbing of the fftcorr_b200 CUDA library:
// status/error handling, device buffers, deterministic block reductions and
// the FP64 spherical-harmonic evaluator used by every kernel that weights a
// grid by Y_lm.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fc_api.h"

namespace fc {

// ----------------------------------------------------------------- errors

// Exception carrying an fc_status; every C entry point catches it and turns
// it into the return code plus the thread's last-error message.
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string &msg) : std::runtime_error(msg), code(c) {}
};

void set_last_error(const std::string &msg);

#define FC_THROW(code, msg) throw ::fc::Error((code), (msg))

#define FC_CUDA(call)                                                     \
  do {                                                                    \
    cudaError_t fc_e_ = (call);                                           \
    if (fc_e_ != cudaSuccess) {                                           \
      FC_THROW(fc_e_ == cudaErrorMemoryAllocation ? FC_ERR_ALLOC          \
                                                  : FC_ERR_CUDA,          \
               std::string(#call) + ": " + cudaGetErrorString(fc_e_));    \
    }                                                                     \
  } while (0)

#define FC_CUFFT(call)                                                    \
  do {                                                                    \
    cufftResult fc_r_ = (call);                                           \
    if (fc_r_ != CUFFT_SUCCESS) {                                         \
      FC_THROW(fc_r_ == CUFFT_ALLOC_FAILED ? FC_ERR_ALLOC : FC_ERR_CUFFT, \
               std::string(#call) + ": cufft error " +                    \
                   std::to_string((int)fc_r_));                           \
    }                                                                     \
  } while (0)

// Host-side count of this library's own kernel launches (every launch site
// is followed by FC_LAUNCH_CHECK).
void note_launch();
#define FC_LAUNCH_CHECK()            \
  do {                               \
    ::fc::note_launch();             \
    FC_CUDA(cudaGetLastError());     \
  } while (0)

#define FC_REQUIRE(cond, code, msg) \
  do {                              \
    if (!(cond)) FC_THROW((code), (msg)); \
  } while (0)

// Runs f and maps exceptions to fc_status codes.
template <typename F>
int guard(F &&f) {
  try {
    f();
    return FC_OK;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc &e) {
    set_last_error("host allocation failed");
    return FC_ERR_ALLOC;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FC_ERR_INVALID;
  }
}

// ------------------------------------------------------- fault injection

// Test hooks behind fc_fault_inject and fc_set_device_budget.  A planned
// failure is raised on the host where the real one would surface, before
// the CUDA or cuFFT call is made, so nothing ever faults on the GPU.
enum FaultKind { kFaultDeviceAlloc = 1, kFaultFftPlan = 2 };
// True when an armed fault of this kind fires now (it then disarms).
bool fault_fires(int kind);
// Called before every device allocation of the library: throws
// FC_ERR_ALLOC for an injected failure or when the bytes would exceed the
// budget.
void device_alloc_check(size_t bytes);
// Running total of the library's device bytes (for the budget).
void device_bytes_add(long long delta);

// ---------------------------------------------------------------- buffers

// Owning device allocation (cudaMalloc / cudaFree).
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { resize(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : ptr_(o.ptr_), bytes_(o.bytes_) {
    o.ptr_ = nullptr;
    o.bytes_ = 0;
  }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
      release();
      ptr_ = o.ptr_;
      bytes_ = o.bytes_;
      o.ptr_ = nullptr;
      o.bytes_ = 0;
    }
    return *this;
  }
  // Reallocates (contents are not preserved) when bytes exceeds capacity.
  void resize(size_t bytes) {
    if (bytes <= bytes_) return;
    release();
    if (bytes == 0) return;
    device_alloc_check(bytes);
    FC_CUDA(cudaMalloc(&ptr_, bytes));
    bytes_ = bytes;
    device_bytes_add((long long)bytes);
  }
  void release() {
    if (ptr_) {
      cudaFree(ptr_);
      device_bytes_add(-(long long)bytes_);
    }
    ptr_ = nullptr;
    bytes_ = 0;
  }
  template <typename T>
  T *as() const {
    return static_cast<T *>(ptr_);
  }
  void *get() const { return ptr_; }
  size_t bytes() const { return bytes_; }

 private:
  void *ptr_ = nullptr;
  size_t bytes_ = 0;
};

// Event pair measuring device time of a phase on one stream, accumulated.
class PhaseTimer {
 public:
  PhaseTimer() {
    FC_CUDA(cudaEventCreate(&a_));
    FC_CUDA(cudaEventCreate(&b_));
  }
  ~PhaseTimer() {
    cudaEventDestroy(a_);
    cudaEventDestroy(b_);
  }
  void start(cudaStream_t s) { cudaEventRecord(a_, s); }
  // Records the end and folds the elapsed time in once it is known.
  void stop(cudaStream_t s) {
    cudaEventRecord(b_, s);
    pending_ = true;
  }
  double seconds() {
    settle();
    return total_;
  }
  void clear() {
    settle();
    total_ = 0.0;
  }
  // Folds a finished interval into the total (waits for the end event).
  void settle() {
    if (!pending_) return;
    cudaEventSynchronize(b_);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a_, b_) == cudaSuccess) total_ += ms * 1e-3;
    pending_ = false;
  }

 private:
  cudaEvent_t a_, b_;
  bool pending_ = false;
  double total_ = 0.0;
};

// Number of SMs on the current device (148 on B200).
int sm_count();

inline unsigned grid_for(size_t n, int block, int waves = 8) {
  size_t blocks = (n + block - 1) / block;
  size_t cap = (size_t)sm_count() * waves;
  if (blocks > cap) blocks = cap;
  if (blocks == 0) blocks = 1;
  return (unsigned)blocks;
}

// Launch shape of a grid-stride kernel: threads per block and at most
// `waves` blocks per SM.
struct LaunchShape {
  int threads;
  int waves;
  unsigned grid(size_t n) const { return grid_for(n, threads, waves); }
};

// ------------------------------------------------------------ reductions

// Deterministic block sum: fixed shuffle tree inside each warp, then warp
// partials combined in warp order by warp 0.  Every thread must call it;
// the result is valid in thread 0.  blockDim.x must be a multiple of 32
// and at most 1024.
// Asynchronous global -> shared copies (no registers held while they fly);
// a thread waits for its own with cp_async_wait_all.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src)
               : "memory");
}
// One grid cell of either type.
__device__ __forceinline__ void cp_async_cell(double *dst, const double *src) {
  cp_async8(dst, src);
}
__device__ __forceinline__ void cp_async_cell(float *dst, const float *src) {
  cp_async4(dst, src);
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

__device__ __forceinline__ double block_sum(double v, double *smem32) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (lane == 0) smem32[warp] = v;
  __syncthreads();
  const int nw = blockDim.x >> 5;
  if (warp == 0) {
    v = lane < nw ? smem32[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}

// ----------------------------------------------------- spherical harmonics

// Parameters of one (ell, m) evaluation: isqpi = sqrt(1/pi)*coeff*(sqrt 2
// when m != 0) and value0 = coeff/sqrt(4 pi) for the ell = 0 shortcut,
// both computed on the host exactly as spherical_harmonics.h:50-87 does.
struct YlmParams {
  int ell;
  int m;
  double isqpi;
  double value0;
  double norm;  // isqpi times the (ell, m) constant: the FP32 evaluator's
                // single normalisation factor, formed in FP64
};

YlmParams make_ylm_params(int ell, int m, double coeff);

// Y_lm(x, y, z) * coeff * D in the reference's operation order
// (spherical_harmonics.h:100-176, exponent 0 so R == 1 and D*R == D).  The
// library is compiled with -fmad=false, so no product is contracted into
// an FMA and each value rounds like the reference's FP64 code.
__device__ __forceinline__ double ylm_eval(const YlmParams &p, double D,
                                           double x, double y, double z) {
  if (p.ell == 0) return D * p.value0;
  const double x2 = x * x;
  const double y2 = y * y;
  const double y3 = y2 * y;
  const double y4 = y3 * y;
  const double z2 = z * z;
  const double ir2 = 1.0 / (x2 + y2 + z2 + 1e-20);
  const double isqpi = p.isqpi;
  if (p.ell == 2) {
    switch (p.m) {
      case 2:
        return D * isqpi * sqrt(15.0 / 32.0) *
               (x2 - y2) * ir2;
      case 1:
        return D * isqpi * sqrt(15.0 / 8.0) * x * z * ir2;
      case 0:
        return D * isqpi * sqrt(5.0 / 16.0) *
               (2.0 * z2 - x2 - y2) * ir2;
      case -1:
        return D * isqpi * sqrt(15.0 / 8.0) * y * z * ir2;
      default:
        return D * isqpi * sqrt(15.0 / 8.0) * x * y * ir2;
    }
  }
  const double z3 = z2 * z;
  const double z4 = z3 * z;
  switch (p.m) {
    case 4:
      return D * isqpi * 3.0 / 16.0 * sqrt(35.0 / 2.0) *
             (x2 * x2 - 6.0 * x2 * y2 + y4) * ir2 * ir2;
    case 3:
      return D * isqpi * 3.0 / 8.0 * sqrt(35.0) *
             (x2 - 3.0 * y2) * z * x * ir2 * ir2;
    case 2:
      return D * isqpi * 3.0 / 8.0 * sqrt(5.0 / 2.0) *
             (6.0 * z2 * (x2 - y2) - x2 * x2 + y4) * ir2 * ir2;
    case 1:
      return D * isqpi * 3.0 / 8.0 * sqrt(5.0) * 3.0 *
             (4.0 / 3.0 * z2 - x2 - y2) * x * z * ir2 * ir2;
    case 0:
      return D * isqpi * 3.0 / 16.0 * 8.0 *
             (z4 - 3.0 * z2 * (x2 + y2) +
              3.0 / 8.0 * (x2 * x2 + 2.0 * x2 * y2 + y4)) *
             ir2 * ir2;
    case -1:
      return D * isqpi * 3.0 / 8.0 * sqrt(5.0) * 3.0 *
             (4.0 / 3.0 * z2 - x2 - y2) * y * z * ir2 * ir2;
    case -2:
      return D * isqpi * 3.0 / 8.0 * sqrt(5.0 / 2.0) *
             (2.0 * x * y * (6.0 * z2 - x2 - y2)) * ir2 * ir2;
    case -3:
      return D * isqpi * 3.0 / 8.0 * sqrt(35.0) *
             (3.0 * x2 * y - y3) * z * ir2 * ir2;
    default:
      return D * isqpi * 3.0 / 16.0 * sqrt(35.0 / 2.0) *
             (4.0 * x * (x2 * y - y3)) * ir2 * ir2;
  }
}

// FP32-mixed evaluator: the same real-form Y_lm * coeff * D, with the
// observer-relative coordinates formed in FP64 by the caller and the FP64
// normalisation p.norm, but the angular polynomial and 1/r^2 in FP32 (the
// result feeds an FP32 transform).
__device__ __forceinline__ float ylm_eval_f32(const YlmParams &p, float D,
                                              double xd, double yd, double zd) {
  if (p.ell == 0) return D * (float)p.value0;
  const float x = (float)xd, y = (float)yd, z = (float)zd;
  const float x2 = x * x, y2 = y * y, z2 = z * z;
  const float ir2 = 1.0f / (x2 + y2 + z2 + 1e-20f);
  const float n = (float)p.norm;
  float poly;
  if (p.ell == 2) {
    switch (p.m) {
      case 2: poly = x2 - y2; break;
      case 1: poly = x * z; break;
      case 0: poly = 2.0f * z2 - x2 - y2; break;
      case -1: poly = y * z; break;
      default: poly = x * y; break;
    }
    return D * n * poly * ir2;
  }
  const float y4 = y2 * y2;
  switch (p.m) {
    case 4: poly = x2 * x2 - 6.0f * x2 * y2 + y4; break;
    case 3: poly = (x2 - 3.0f * y2) * z * x; break;
    case 2: poly = 6.0f * z2 * (x2 - y2) - x2 * x2 + y4; break;
    case 1: poly = (4.0f / 3.0f * z2 - x2 - y2) * x * z; break;
    case 0:
      poly = z2 * z2 - 3.0f * z2 * (x2 + y2) +
             0.375f * (x2 * x2 + 2.0f * x2 * y2 + y4);
      break;
    case -1: poly = (4.0f / 3.0f * z2 - x2 - y2) * y * z; break;
    case -2: poly = 2.0f * x * y * (6.0f * z2 - x2 - y2); break;
    case -3: poly = (3.0f * x2 * y - y2 * y) * z; break;
    default: poly = 4.0f * x * (x2 * y - y2 * y); break;
  }
  return D * n * poly * (ir2 * ir2);
}

}  // namespace fc
