// fc_fused.cu -- the survey correlator's per-(ell, m) work as five fused,
// hand-written FFT passes over HBM (no cuFFT), with the Y_lm weighting, the
// conjugate product, the k-subgrid extraction and the r-subgrid extraction
// folded into them, and the inverse transform pruned to the rows the
// r-subgrid needs.
//
// Per (ell, m), for the half-complex work array W[x][y][kz] (kz < N2/2+1):
//   zfwd   W[x][y][:] = R2C_z( Y_lm(cell) * rho[x][y][:] )   (make_ylm + r2c
//          along z; spherical_harmonics.h:32-179, fft_grid.cc:125-150)
//   yfwd   W = DFT_y(W)
//   xcorr  per (ky, kz) column: F = DFT_x(W); P = F * conj(G)
//          (array_ops.cc:139-163); ksub += Y_lm(k) W(k)^-2 4 pi Re P on the
//          k-subgrid (fft_grid.cc:215-258); Wr[ri][ky][kz] = IDFT_x(P) only
//          at the rs rows x = (N0 - rs/2 + ri) mod N0 of the r-subgrid
//   yinv   Wry[ri][rj][kz] = IDFT_y(Wr) at the rs rows of the r-subgrid
//   zinv   rsub[ri][rj][rk] += Y_lm(r) 4 pi/N * C2R_z(Wry)[rk] (fft_grid.cc:
//          182-210)
// grid2's transform G (correlator.h:53-77) is zfwd (no weighting) + yfwd +
// DFT_x.  Bytes per (ell, m) at 512^3 FP32: ~4 GB instead of ~11 GB for
// separate make_ylm / cuFFT r2c / multiply / extract / cuFFT c2r passes.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fc_common.cuh"
#include "fc_fft.cuh"
#include "fc_fused.h"
#include "fc_internal.h"

namespace fc {
namespace {

constexpr int kThreads = 256;  // threads per CTA of every fused pass

template <typename T>
using C2 = typename Vec2<T>::type;

// ------------------------------------------------------------------ zfwd
// B rows of N2 reals per CTA: (optionally Y_lm-weighted) packed as
// z_j = x_2j + i x_2j+1, length-M complex DFT, then the real-to-complex
// split X_k = E_k + e^{-2 pi i k/N2} O_k for k <= M.
template <typename T, typename TI, bool WEIGHT>
__global__ void k_zfwd(const TI *__restrict__ rho, C2<T> *__restrict__ W,
                       FusedGeom g, YlmParams p, double x0, double y0,
                       double z0, const C2<T> *__restrict__ tabz, int B) {
  using C = C2<T>;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int BP = B + 1;
  const int M = g.m;
  C *buf2 = buf + M * BP;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const int64_t row0 = (int64_t)blockIdx.x * B;
  for (int idx = threadIdx.x; idx < M * B; idx += blockDim.x) {
    const int b = idx / M;
    const int j = idx - b * M;
    const int64_t row = row0 + b;
    C z;
    z.x = 0;
    z.y = 0;
    if (row < nrows) {
      const TI *src = rho + row * g.n2 + 2 * j;
      double v0 = (double)src[0];
      double v1 = (double)src[1];
      if (WEIGHT) {
        const int x = (int)(row / g.n1);
        const int y = (int)(row - (int64_t)x * g.n1);
        const double cx = x0 + x * 1.0;
        const double cy = y0 + y * 1.0;
        v0 = ylm_eval(p, v0, cx, cy, z0 + (2 * j) * 1.0);
        v1 = ylm_eval(p, v1, cx, cy, z0 + (2 * j + 1) * 1.0);
      }
      z.x = (T)v0;
      z.y = (T)v1;
    }
    buf[j * BP + b] = z;
  }
  __syncthreads();
  buf = fft_columns(buf, buf2, g.pz, B, BP, tabz, -1);
  const int H = M + 1;
  for (int idx = threadIdx.x; idx < H * B; idx += blockDim.x) {
    const int b = idx / H;
    const int k = idx - b * H;
    const int64_t row = row0 + b;
    if (row >= nrows) continue;
    const C a = buf[(k % M) * BP + b];
    const C c = cconj(buf[((M - k) % M) * BP + b]);
    C e, d, o;
    e.x = (T)0.5 * (a.x + c.x);
    e.y = (T)0.5 * (a.y + c.y);
    d = csub(a, c);
    o.x = (T)0.5 * d.y;  // -i (a - c) / 2
    o.y = (T)-0.5 * d.x;
    W[row * g.h + k] = cadd(e, cmul(tabz[k], o));
  }
}

// Loads a B-column tile of a strided axis into shared memory.
template <typename C>
__device__ __forceinline__ void load_columns(C *buf, const C *__restrict__ src,
                                             int64_t base, int64_t stride,
                                             int L, int B, int BP, int kz0,
                                             int h) {
  for (int idx = threadIdx.x; idx < L * B; idx += blockDim.x) {
    const int i = idx / B;
    const int b = idx - i * B;
    C v;
    v.x = 0;
    v.y = 0;
    if (kz0 + b < h) v = src[base + i * stride + kz0 + b];
    buf[i * BP + b] = v;
  }
  __syncthreads();
}

// ------------------------------------------------------------------ yfwd
template <typename T>
__global__ void k_yfwd(C2<T> *__restrict__ W, FusedGeom g,
                       const C2<T> *__restrict__ taby, int B) {
  using C = C2<T>;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int BP = B + 1;
  const int kz0 = blockIdx.x * B;
  const int x = blockIdx.y;
  const int64_t base = (int64_t)x * g.n1 * g.h;
  load_columns(buf, W, base, g.h, g.n1, B, BP, kz0, g.h);
  buf = fft_columns(buf, buf + g.n1 * BP, g.py, B, BP, taby, -1);
  for (int idx = threadIdx.x; idx < g.n1 * B; idx += blockDim.x) {
    const int i = idx / B;
    const int b = idx - i * B;
    if (kz0 + b < g.h) W[base + (int64_t)i * g.h + kz0 + b] = buf[i * BP + b];
  }
}

// ----------------------------------------------------------------- xcorr
// MODE 0: G = DFT_x(W) (grid2's transform).  MODE 1: the fused product,
// k-subgrid extraction, inverse and pruning described at the top.
template <typename T, int MODE>
__global__ void k_xcorr(const C2<T> *__restrict__ W,
                        const C2<T> *__restrict__ G, C2<T> *__restrict__ out,
                        double *__restrict__ ksub, FusedGeom g,
                        const C2<T> *__restrict__ tabx,
                        const double *__restrict__ kx,
                        const double *__restrict__ ky,
                        const double *__restrict__ kz,
                        const double *__restrict__ wx,
                        const double *__restrict__ wy,
                        const double *__restrict__ wz, YlmParams pk, int B) {
  using C = C2<T>;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int BP = B + 1;
  const int kz0 = blockIdx.x * B;
  const int yy = blockIdx.y;
  const int64_t stride = (int64_t)g.n1 * g.h;
  const int64_t base = (int64_t)yy * g.h;
  C *other = buf + g.n0 * BP;
  load_columns(buf, W, base, stride, g.n0, B, BP, kz0, g.h);
  {
    C *res = fft_columns(buf, other, g.px, B, BP, tabx, -1);
    other = res == buf ? other : buf;
    buf = res;
  }
  if constexpr (MODE == 0) {
    for (int idx = threadIdx.x; idx < g.n0 * B; idx += blockDim.x) {
      const int i = idx / B;
      const int b = idx - i * B;
      if (kz0 + b < g.h) out[base + i * stride + kz0 + b] = buf[i * BP + b];
    }
    return;
  } else {
  // P = F * conj(G).
  for (int idx = threadIdx.x; idx < g.n0 * B; idx += blockDim.x) {
    const int i = idx / B;
    const int b = idx - i * B;
    if (kz0 + b < g.h)
      buf[i * BP + b] = cmulc(buf[i * BP + b], G[base + i * stride + kz0 + b]);
  }
  __syncthreads();
  // k-subgrid: this CTA owns the sources with ky index yy and kz in its
  // block.  Direct targets k = kz + oz read P[(i - ox) mod N0][yy][kz];
  // reflected targets k = oz - kz (kz >= 1) read P[(ox - i) mod N0][yy][kz]
  // for j with (oy - j) mod N1 == yy.  Every ksub cell has exactly one
  // source element, so these read-modify-writes never collide.
  if (ksub != nullptr) {
    const int ox = g.ks0 / 2, oy = g.ks1 / 2, oz = g.ks2 / 2;
    for (int refl = 0; refl < 2; ++refl) {
      int j = refl == 0 ? (yy + oy) % g.n1 : ((oy - yy) % g.n1 + g.n1) % g.n1;
      for (; j < g.ks1; j += g.n1) {
        for (int idx = threadIdx.x; idx < g.ks0 * B; idx += blockDim.x) {
          const int i = idx / B;
          const int b = idx - i * B;
          const int kzi = kz0 + b;
          if (kzi >= g.h || kzi > oz || (refl == 1 && kzi == 0)) continue;
          const int k = refl == 0 ? kzi + oz : oz - kzi;
          const int x = refl == 0 ? ((i - ox) % g.n0 + g.n0) % g.n0
                                  : ((ox - i) % g.n0 + g.n0) % g.n0;
          const double re = (double)buf[x * BP + b].x;
          const double inv_w = 1.0 / (wx[i] * wy[j] * wz[k]);
          const double yv = ylm_eval(pk, inv_w, kx[i], ky[j], kz[k]);
          double *dst = ksub + ((size_t)i * g.ks1 + j) * g.ks2 + k;
          *dst += yv * re;
        }
      }
    }
    __syncthreads();
  }
  buf = fft_columns(buf, other, g.px, B, BP, tabx, +1);
  const int64_t obase = (int64_t)yy * g.h;
  const int64_t ostride = (int64_t)g.n1 * g.h;
  for (int idx = threadIdx.x; idx < g.rs * B; idx += blockDim.x) {
    const int ri = idx / B;
    const int b = idx - ri * B;
    if (kz0 + b >= g.h) continue;
    const int x = ((ri - g.ro) % g.n0 + g.n0) % g.n0;
    out[obase + ri * ostride + kz0 + b] = buf[x * BP + b];
  }
  }
}

// ------------------------------------------------------------------ yinv
template <typename T>
__global__ void k_yinv(const C2<T> *__restrict__ Wr, C2<T> *__restrict__ Wry,
                       FusedGeom g, const C2<T> *__restrict__ taby, int B) {
  using C = C2<T>;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int BP = B + 1;
  const int kz0 = blockIdx.x * B;
  const int ri = blockIdx.y;
  const int64_t base = (int64_t)ri * g.n1 * g.h;
  load_columns(buf, Wr, base, g.h, g.n1, B, BP, kz0, g.h);
  buf = fft_columns(buf, buf + g.n1 * BP, g.py, B, BP, taby, +1);
  const int64_t obase = (int64_t)ri * g.rs * g.h;
  for (int idx = threadIdx.x; idx < g.rs * B; idx += blockDim.x) {
    const int rj = idx / B;
    const int b = idx - rj * B;
    if (kz0 + b >= g.h) continue;
    const int y = ((rj - g.ro) % g.n1 + g.n1) % g.n1;
    Wry[obase + (int64_t)rj * g.h + kz0 + b] = buf[y * BP + b];
  }
}

// ----------------------------------------------------------------- zinv
// B rows (ri, rj) per CTA: complex-to-real inverse along z (unnormalised,
// the imaginary parts of the DC and Nyquist terms ignored), then
// rsub[ri][rj][rk] += Y_lm(r) * value at z = (N2 - rs/2 + rk) mod N2.
template <typename T>
__global__ void k_zinv_rsub(const C2<T> *__restrict__ Wry,
                            double *__restrict__ rsub, FusedGeom g,
                            const C2<T> *__restrict__ tabz,
                            const double *__restrict__ raxis, YlmParams pr,
                            int B) {
  using C = C2<T>;
  extern __shared__ unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int BP = B + 1;
  const int M = g.m;
  const int nrows = g.rs * g.rs;
  const int row0 = blockIdx.x * B;
  C *buf2 = buf + M * BP;
  for (int idx = threadIdx.x; idx < M * B; idx += blockDim.x) {
    const int b = idx / M;
    const int k = idx - b * M;
    const int row = row0 + b;
    C z;
    z.x = 0;
    z.y = 0;
    if (row < nrows) {
      const C *X = Wry + (int64_t)row * g.h;
      C a = X[k];
      C c = cconj(X[M - k]);
      if (k == 0) {
        a.y = 0;
        c.y = 0;  // X[M] is the Nyquist term
      }
      const C e = cadd(a, c);
      const C o = cmul(csub(a, c), cconj(tabz[k]));  // times e^{+2 pi i k/N2}
      z.x = e.x - o.y;
      z.y = e.y + o.x;
    }
    buf[k * BP + b] = z;
  }
  __syncthreads();
  buf = fft_columns(buf, buf2, g.pz, B, BP, tabz, +1);
  for (int idx = threadIdx.x; idx < g.rs * B; idx += blockDim.x) {
    const int b = idx / g.rs;
    const int rk = idx - b * g.rs;
    const int row = row0 + b;
    if (row >= nrows) continue;
    const int ri = row / g.rs;
    const int rj = row - ri * g.rs;
    const int z = ((rk - g.ro) % g.n2 + g.n2) % g.n2;
    const C zz = buf[(z >> 1) * BP + b];
    const double v = (double)((z & 1) ? zz.y : zz.x);
    const double yv = ylm_eval(pr, 1.0, raxis[ri], raxis[rj], raxis[rk]);
    rsub[(size_t)row * g.rs + rk] += yv * v;
  }
}

__global__ void k_to_float(const double *__restrict__ in, float *__restrict__ out,
                           size_t n, double shift) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)(in[i] - shift);
}

// Radices of a length, largest first (8, 4, 2, 3, 5, 7); false if L has a
// prime factor above 7.
bool plan_length(int L, int tab_scale, FftPlan *p) {
  p->L = L;
  p->tab_scale = tab_scale;
  p->npass = 0;
  int n = L;
  const int radices[] = {8, 4, 2, 3, 5, 7};
  for (int r : radices) {
    while (n % r == 0) {
      if (p->npass == 12) return false;
      p->radix[p->npass++] = r;
      n /= r;
    }
  }
  if (n != 1) return false;
  int ns = 1;
  for (int s = 0; s < p->npass; ++s) {
    p->ns[s] = ns;
    ns *= p->radix[s];
  }
  return true;
}

template <typename C>
std::vector<C> root_table(int order) {
  std::vector<C> t(order);
  for (int m = 0; m < order; ++m) {
    // e^{-2 pi i m / order}, argument reduced exactly before the FP64 call.
    const double a = 2.0 * M_PI * (double)m / (double)order;
    t[m].x = (decltype(t[m].x))cos(a);
    t[m].y = (decltype(t[m].y))(-sin(a));
  }
  return t;
}

int cols_for(int L, int elem_bytes) {
  // Columns per CTA: 64-byte row segments (full 32-byte sectors) while the
  // two shared-memory tiles (2 x L x (B+1) complex) stay within 100 KB, so
  // two or more CTAs fit on an SM.
  int B = 64 / elem_bytes;
  while (B > 1 && 2 * (size_t)L * (B + 1) * elem_bytes > 100 * 1024) B /= 2;
  return B;
}

}  // namespace

bool FusedSurvey::supported(const int shape[3], int rsize) {
  if (shape[2] % 2 != 0) return false;
  FftPlan p;
  if (!plan_length(shape[0], 1, &p) || !plan_length(shape[1], 1, &p) ||
      !plan_length(shape[2] / 2, 2, &p))
    return false;
  for (int a = 0; a < 3; ++a) {
    const int L = a == 2 ? shape[2] / 2 : shape[a];
    if (L > 4096) return false;
  }
  return rsize > 0;
}

FusedSurvey::FusedSurvey(const int shape[3], int rsize, const int kshape[3],
                         bool fp64)
    : fp64_(fp64) {
  g.n0 = shape[0];
  g.n1 = shape[1];
  g.n2 = shape[2];
  g.m = shape[2] / 2;
  g.h = g.m + 1;
  g.rs = rsize;
  g.ro = rsize / 2;
  g.ks0 = kshape[0];
  g.ks1 = kshape[1];
  g.ks2 = kshape[2];
  FC_REQUIRE(plan_length(g.n0, 1, &g.px) && plan_length(g.n1, 1, &g.py) &&
                 plan_length(g.m, 2, &g.pz),
             FC_ERR_UNSUPPORTED, "grid size has a prime factor above 7");
  const size_t eb = fp64 ? 16 : 8;
  if (fp64) {
    auto tx = root_table<double2>(g.n0), ty = root_table<double2>(g.n1),
         tz = root_table<double2>(g.n2);
    upload(tabx, tx);
    upload(taby, ty);
    upload(tabz, tz);
  } else {
    auto tx = root_table<float2>(g.n0), ty = root_table<float2>(g.n1),
         tz = root_table<float2>(g.n2);
    upload(tabx, tx);
    upload(taby, ty);
    upload(tabz, tz);
  }
  bx = cols_for(g.n0, (int)eb);
  by = cols_for(g.n1, (int)eb);
  bz = cols_for(g.m, (int)eb);
  const size_t nc = (size_t)g.n0 * g.n1 * g.h;
  W.resize(nc * eb);
  G.resize(nc * eb);
  Wr.resize((size_t)g.rs * g.n1 * g.h * eb);
  Wry.resize((size_t)g.rs * g.rs * g.h * eb);
  if (!fp64) rho32.resize((size_t)g.n0 * g.n1 * g.n2 * sizeof(float));
  set_smem_limits();
}

template <typename V>
void FusedSurvey::upload(DeviceBuffer &dst, const std::vector<V> &v) {
  dst.resize(v.size() * sizeof(V));
  FC_CUDA(cudaMemcpy(dst.get(), v.data(), v.size() * sizeof(V),
                     cudaMemcpyHostToDevice));
}

size_t FusedSurvey::smem(int L, int B) const {
  return 2 * (size_t)L * (B + 1) * (fp64_ ? 16 : 8);
}

void FusedSurvey::set_smem_limits() {
  const int big = 200 * 1024;
  if (fp64_) {
    FC_CUDA(cudaFuncSetAttribute(k_zfwd<double, double, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zfwd<double, double, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_yfwd<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xcorr<double, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xcorr<double, 1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_yinv<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zinv_rsub<double>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  } else {
    FC_CUDA(cudaFuncSetAttribute(k_zfwd<float, float, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zfwd<float, float, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_yfwd<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xcorr<float, 0>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_xcorr<float, 1>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_yinv<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    FC_CUDA(cudaFuncSetAttribute(k_zinv_rsub<float>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  }
}

const void *FusedSurvey::prepare_input(const double *rho, cudaStream_t s) {
  if (fp64_) return rho;
  const size_t n = (size_t)g.n0 * g.n1 * g.n2;
  k_to_float<<<grid_for(n, 256), 256, 0, s>>>(rho, rho32.as<float>(), n, 0.0);
  FC_LAUNCH_CHECK();
  return rho32.get();
}

template <typename T>
void FusedSurvey::zfwd(const void *rho, bool weight, const YlmParams &p,
                       const double xyz0[3], cudaStream_t s) {
  const int B = bz;
  const int64_t nrows = (int64_t)g.n0 * g.n1;
  const unsigned blocks = (unsigned)((nrows + B - 1) / B);
  const int threads = kThreads;
  const size_t sm = smem(g.m, B);
  if (weight)
    k_zfwd<T, T, true><<<blocks, threads, sm, s>>>(
        (const T *)rho, W.as<C2<T>>(), g, p, xyz0[0], xyz0[1], xyz0[2],
        tabz.as<C2<T>>(), B);
  else
    k_zfwd<T, T, false><<<blocks, threads, sm, s>>>(
        (const T *)rho, W.as<C2<T>>(), g, p, xyz0[0], xyz0[1], xyz0[2],
        tabz.as<C2<T>>(), B);
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::yfwd(cudaStream_t s) {
  const int B = by;
  dim3 grid((g.h + B - 1) / B, g.n0);
  k_yfwd<T><<<grid, kThreads, smem(g.n1, B), s>>>(W.as<C2<T>>(), g,
                                                       taby.as<C2<T>>(), B);
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::xcorr(bool product, double *ksub, const KAxes &ka,
                        const YlmParams &pk, cudaStream_t s) {
  const int B = bx;
  dim3 grid((g.h + B - 1) / B, g.n1);
  const int threads = kThreads;
  const size_t sm = smem(g.n0, B);
  if (!product) {
    k_xcorr<T, 0><<<grid, threads, sm, s>>>(
        W.as<C2<T>>(), nullptr, G.as<C2<T>>(), nullptr, g, tabx.as<C2<T>>(),
        ka.kx, ka.ky, ka.kz, ka.wx, ka.wy, ka.wz, pk, B);
  } else {
    k_xcorr<T, 1><<<grid, threads, sm, s>>>(
        W.as<C2<T>>(), G.as<C2<T>>(), Wr.as<C2<T>>(), ksub, g, tabx.as<C2<T>>(),
        ka.kx, ka.ky, ka.kz, ka.wx, ka.wy, ka.wz, pk, B);
  }
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::yinv(cudaStream_t s) {
  const int B = by;
  dim3 grid((g.h + B - 1) / B, g.rs);
  k_yinv<T><<<grid, kThreads, smem(g.n1, B), s>>>(
      Wr.as<C2<T>>(), Wry.as<C2<T>>(), g, taby.as<C2<T>>(), B);
  FC_LAUNCH_CHECK();
}

template <typename T>
void FusedSurvey::zinv(double *rsub, const double *raxis, const YlmParams &pr,
                       cudaStream_t s) {
  const int B = bz;
  const int nrows = g.rs * g.rs;
  const unsigned blocks = (unsigned)((nrows + B - 1) / B);
  k_zinv_rsub<T><<<blocks, kThreads, smem(g.m, B), s>>>(
      Wry.as<C2<T>>(), rsub, g, tabz.as<C2<T>>(), raxis, pr, B);
  FC_LAUNCH_CHECK();
}

void FusedSurvey::grid2(const void *rho_in, cudaStream_t s, const KAxes &ka) {
  YlmParams none = make_ylm_params(0, 0, 1.0);
  const double zero[3] = {0, 0, 0};
  if (fp64_) {
    zfwd<double>(rho_in, false, none, zero, s);
    yfwd<double>(s);
    xcorr<double>(false, nullptr, ka, none, s);
  } else {
    zfwd<float>(rho_in, false, none, zero, s);
    yfwd<float>(s);
    xcorr<float>(false, nullptr, ka, none, s);
  }
}

void FusedSurvey::term(const void *rho_in, int ell, int m, const double xyz0[3],
                       double ncells, double *ksub, double *rsub,
                       const double *raxis, const KAxes &ka, cudaStream_t s,
                       PhaseHook *hook) {
  const YlmParams pw = make_ylm_params(ell, m, 1.0);
  const YlmParams pk = make_ylm_params(ell, m, 4.0 * M_PI);
  const YlmParams pr = make_ylm_params(ell, m, 4.0 * M_PI / ncells);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    if (hook) hook->begin("zfwd");
    zfwd<T>(rho_in, true, pw, xyz0, s);
    if (hook) hook->end();
    if (hook) hook->begin("yfwd");
    yfwd<T>(s);
    if (hook) hook->end();
    if (hook) hook->begin("xcorr");
    xcorr<T>(true, ksub, ka, pk, s);
    if (hook) hook->end();
    if (hook) hook->begin("yinv");
    yinv<T>(s);
    if (hook) hook->end();
    if (hook) hook->begin("zinv");
    zinv<T>(rsub, raxis, pr, s);
    if (hook) hook->end();
  };
  if (fp64_)
    run(double());
  else
    run(float());
}

}  // namespace fc
